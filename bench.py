#!/usr/bin/env python
"""Benchmark of the per-gulp single-pulse search (Heimdall's hd_execute).

Headline workload (default, --workload multibeam): one gulp of a 36-beam
multibeam receiver -- 36 beams x 320 channels uint8, 851 MHz top,
-0.09765625 MHz channels, 655.36 us, 2^15 samples per beam (773 beam-seconds
per gulp), DM 0-2000 (tol 1.25, 40 us), boxcars 2^0..2^9, threshold 6; seeded
synthetic data (noise N(128,16^2), 2 injected dispersed pulses per beam).

Metric: beam-seconds searched per second, batched vs plain.
  value  -- the batched form: K gulps through hd_execute_beams with the 36
            filterbanks resident in HBM; CUDA events around the K calls (each
            call ends synchronised).
  plain  -- the plain per-beam GPU form on the same resident data: each gulp
            is 36 hd_execute_device calls, one per beam.
  e2e    -- the batched form through hd_execute_beams from pinned host memory:
            the host->device copy of all 36 filterbanks is inside the timed
            region, candidate rows are read back every step.
  recall -- injected pulses with S/N >= 8 matched by a candidate of their beam.
The input (360 MiB) is larger than L2 (126 MB), so no L2 flush is needed.
--workload survey runs the plain single-beam survey gulp (1024 channels,
2^18 samples, DM 0-2000, boxcars to 2^12, clean_filterbank_rfi on) instead;
the default run also reports it as "survey_plain".

`--impl reference` times the reference's own stage code (Pipeline/*.cu rebuilt
on Thrust's OpenMP backend, oracle/_ref) with all host threads on a bounded
sample of the same workload (whole beams of the multibeam gulp; a DM-range
subset of the survey gulp, scaled by the DM count).

Multi-GPU: beams are independent, so every rank searches its own gulp
(replicas, weak scaling); the max over ranks of the device time is used.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "beam-sec searched per sec, batched vs plain; injected recall at S/N>=8"
UNIT = "beam-s/s"

# DRAM bytes per k_dedisp launch, read from the committed ncu summaries
TRAFFIC = {
    "multibeam_36x_c320_n32768": ("k_dedisp_multibeam_36x_c320_n32768.md",
                                  "traffic_bytes_per_launch:"),
}


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, gpu_index: int = 0):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:  # no nvidia-smi: the line says so
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        med = float(np.median(sm)) if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


class Work:
    """One gulp: `beams` independent filterbanks (nsamps x nchans uint8 each)
    with their injected pulses, and the search configuration `w`."""

    def __init__(self, w, fbs, pulses):
        self.w = w
        self.fbs = fbs
        self.pulses = pulses
        self.nsamps, self.nchans = fbs[0].shape
        self.units = len(fbs)
        self.beam_s = self.units * self.nsamps * w.dt


def workload(kind, nsamps=None, nbeams=None):
    import dataclasses
    from heimdall_multibeam_b200 import synth
    if kind == "survey":
        w = synth.SEARCH_C1
        b = synth.make_c1(nsamps=nsamps)
        if nsamps:
            w = dataclasses.replace(w, name=f"plain_c1024_n{nsamps}_rfi", nsamps=nsamps)
        return Work(w, [b.data], [b.pulses])
    w = synth.SEARCH_C2
    if nsamps or nbeams:
        w = dataclasses.replace(w, nsamps=nsamps or w.nsamps, nbeams=nbeams or w.nbeams)
        w = dataclasses.replace(w, name=f"multibeam_{w.nbeams}x_c320_n{w.nsamps}")
    beams = synth.make_multibeam(w, seed=2026)
    return Work(w, [b.data for b in beams], [b.pulses for b in beams])


def params_for(H, w, **kw):
    return H.default_params(nchans=w.nchans, dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min,
                            dm_max=w.dm_max, boxcar_max=w.boxcar_max, output_dir=None, **kw)


def config_for(wk, dm_trials, world):
    """The workload description both arms print (identical dicts)."""
    w = wk.w
    return {"workload": w.name, "form": "batched" if wk.units > 1 else "plain",
            "nbeams": wk.units, "nchans": wk.nchans, "nsamps_per_beam": wk.nsamps,
            "dt_s": w.dt, "dm_range": [w.dm_min, w.dm_max], "dm_trials": dm_trials,
            "boxcar_max": w.boxcar_max, "clean_filterbank_rfi": bool(w.clean),
            "beam_seconds_per_gulp": round(wk.beam_s, 4),
            "l2": f"input {wk.units * wk.nsamps * wk.nchans / 2**20:.0f} MiB > L2, no flush",
            "parallelism": f"replicas{world}"}


def recall(cands, pulses, dt, snr_min=8.0):
    """Injected pulses with S/N >= 8 matched by a candidate: |samp - t0| <=
    max(2^filter, FWHM/dt) + 2 and DM within max(5%, 2 trial steps) (fixed
    before any run)."""
    hit = 0
    strong = [p for p in pulses if p.snr >= snr_min]
    for p in strong:
        fw = p.fwhm_s / dt
        ok = False
        for c in cands:
            tol_t = max(2 ** int(c["filter"]), fw) + 2
            tol_dm = max(0.05 * p.dm, 2 * 1.25 * max(p.dm, 1.0) * 0.01)
            if abs(int(c["samp_idx"]) - p.t0) <= tol_t and abs(float(c["dm"]) - p.dm) <= tol_dm:
                ok = True
                break
        hit += ok
    return hit, len(strong)


def max_over_ranks(torch, dist, values, device):
    """Element-wise maximum over all ranks of this rank's timings (ms): a
    multi-GPU step takes as long as its slowest rank."""
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def whole_job_value(world, beam_s, ms):
    """Beam-seconds searched per second by the whole job: every rank searches
    its own gulp of beam_s beam-seconds (replicas, weak scaling) in at most
    ms milliseconds."""
    return world * beam_s / (ms / 1e3)


def _timed(torch, dev, barrier, steps, fn, stage=None, timing=None):
    """K calls of fn between CUDA events (each call ends synchronised)."""
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record()
    for _ in range(steps):
        fn()
        if stage is not None:
            t = timing()
            for k in stage:
                stage[k] += t[k]
    e1.record()
    barrier()
    return e0.elapsed_time(e1) / steps


def run_product(args):
    import torch
    import heimdall_multibeam_b200 as H

    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", local if world > 1 else 0)

    wk = workload(args.workload, args.nsamps, args.nbeams)
    w = wk.w
    U, nsamps, nchans = wk.units, wk.nsamps, wk.nchans
    p = params_for(H, w)
    p.gpu_id = dev.index
    pl = H.Pipeline(p, cleaning=w.clean)

    d_all = torch.from_numpy(np.stack(wk.fbs)).to(dev)
    h_all = torch.from_numpy(np.stack(wk.fbs)).pin_memory()
    fb_bytes = nsamps * nchans
    d_ptrs = [d_all.data_ptr() + u * fb_bytes for u in range(U)]
    h_ptrs = [h_all.data_ptr() + u * fb_bytes for u in range(U)]
    torch.cuda.synchronize(dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def batched():
        if U == 1:
            err, _ = pl.execute_device(d_ptrs[0], nsamps)
        else:
            err, _, _ = pl.execute_beams(d_ptrs, nsamps=nsamps, on_device=True)
        assert err in (H.HD_NO_ERROR, H.HD_TOO_MANY_EVENTS), H.error_string(err)

    def batched_e2e():
        if U == 1:
            pl.execute_ptr(h_ptrs[0], nsamps)
        else:
            pl.execute_beams(h_ptrs, nsamps=nsamps, on_device=False)
        return len(pl.candidates())  # every beam's rows, one call

    def plain():
        for u in range(U):
            pl.execute_device(d_ptrs[u], nsamps)

    # measured 32-bit integer add rate (the dedispersion roofline's denominator)
    int_peak = H.int_add_rate(dev.index) / 1e12

    # ---- batched form, device-resident input ---------------------------------
    for _ in range(args.warmup):
        batched()
    l0 = H.launch_count()
    r0 = pl.graph_replays()
    stage = {k: 0.0 for k in pl.timing()}
    clk = ClockSampler(dev.index)
    clk.start()
    ms = _timed(torch, dev, barrier, args.steps, batched, stage, pl.timing)
    launches = H.launch_count() - l0
    replays = pl.graph_replays() - r0
    cands = [pl.candidates(u) for u in range(U)] if U > 1 else [pl.candidates()]
    tile = pl.dedisp_tile()
    tile_source = pl.dedisp_tile_source()

    # ---- plain per-beam form on the same data ---------------------------------
    ms_plain = None
    if U > 1 and not args.batched_only:
        for _ in range(max(1, args.warmup // 2)):
            plain()
        lp = H.launch_count()
        ms_plain = _timed(torch, dev, barrier, args.steps, plain)
        launches_plain = H.launch_count() - lp

    # ---- end to end from pinned host memory ------------------------------------
    ms_e2e = None
    ncand = 0
    stage_e2e = {k: 0.0 for k in stage}
    if not args.batched_only:
        for _ in range(max(1, args.warmup // 2)):
            batched_e2e()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record()
        for _ in range(args.steps):
            ncand = batched_e2e()
            t = pl.timing()
            for k in stage_e2e:
                stage_e2e[k] += t[k]
        e1.record()
        barrier()
        ms_e2e = e0.elapsed_time(e1) / args.steps

    # ---- end to end, double-buffered ingest (hd_prefetch_beams): the copy of
    # gulp k + 1 runs on the copy stream while gulp k is searched; every
    # step's copy and result read stay inside the timed region
    ms_e2e_pf = None
    if not args.batched_only and U > 1:
        def e2e_pipelined(steps):
            n = 0
            assert pl.prefetch_beams(h_ptrs, nsamps) == H.HD_NO_ERROR
            for k in range(steps):
                if k + 1 < steps:
                    assert pl.prefetch_beams(h_ptrs, nsamps) == H.HD_NO_ERROR
                err, _, _ = pl.execute_prefetched(U)
                assert err in (H.HD_NO_ERROR, H.HD_TOO_MANY_EVENTS), err
                n = len(pl.candidates())  # every beam's rows, one call
            return n
        # the streaming form rotates three device buffers: one capture each
        e2e_pipelined(max(4, args.warmup))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record()
        ncand = e2e_pipelined(args.steps)
        e1.record()
        barrier()
        ms_e2e_pf = e0.elapsed_time(e1) / args.steps

    # clocks sampled over the timed regions (batched, plain, e2e)
    clocks = clk.stop()
    ms, ms_plain_m, ms_e2e_m, ms_e2e_pf_m = max_over_ranks(
        torch, dist, [ms, ms_plain or 0.0, ms_e2e or 0.0, ms_e2e_pf or 0.0], dev)
    value = whole_job_value(world, wk.beam_s, ms)

    clf_rec = None
    if not args.batched_only and not args.no_classifier:
        clf_rec = classifier_bench(args, H, torch, dev, pl)
    pl.close()
    uneven = None
    if args.workload == "multibeam" and not args.batched_only and args.uneven_beams > 0:
        uneven = uneven_bench(args, H, torch, dev, barrier, dist, world)
    # secondary: the plain survey-size single-beam gulp
    survey = None
    if args.workload == "multibeam" and not args.no_survey and not args.batched_only:
        survey = survey_plain(args, H, torch, dev, barrier, dist, world)

    if rank == 0:
        peaks, peak_kind = _peaks()
        # dominant kernel: brute-force dedispersion
        plan = H.DedispPlan(nchans, w.dt, w.f0, w.df)
        plan.generate_dm_list(w.dm_min, w.dm_max, 40.0, 1.25)
        D = len(plan.dm_list)
        nout = nsamps - plan.max_delay
        t_dd = stage["dedisperse"] / args.steps  # ms, events on the pipeline stream
        bytes_dd = U * (nchans * nsamps + D * nout * 4)
        adds = U * D * nout * nchans
        gbs = bytes_dd / (t_dd / 1e3) / 1e9
        add_rate = adds / (t_dd / 1e3) / 1e12  # T sample-channel adds / s
        t_hbm = bytes_dd / (peaks["hbm_gbs"] * 1e9) * 1e3
        t_int = adds / (int_peak * 1e12) * 1e3
        traffic = None
        tf = TRAFFIC.get(w.name)
        if tf:
            try:
                with open(os.path.join(ROOT, "profiles", tf[0])) as f:
                    for ln in f:
                        if ln.startswith(tf[1]):
                            traffic = int(ln.split(":")[1])
            except (OSError, ValueError, IndexError):
                traffic = None  # no committed capture: the line reports traffic null
        hit = nstrong = 0
        for u in range(U):
            h_, n_ = recall(cands[u], wk.pulses[u], w.dt)
            hit += h_
            nstrong += n_
        # roofline of the dominant kernel: t_min = max(bytes / HBM, adds /
        # integer add rate); frac = t_min / t_measured, bound = the larger
        int_bound = t_int >= t_hbm
        roof = {"kernel": "k_dedisp", "bound": "int_add" if int_bound else "hbm",
                "achieved": round(add_rate if int_bound else gbs, 3),
                "peak": round(int_peak if int_bound else peaks["hbm_gbs"], 3),
                "unit": "Tadd/s" if int_bound else "GB/s",
                "frac": round(max(t_int, t_hbm) / t_dd, 4),
                "traffic": traffic, "t_min_ms": round(max(t_int, t_hbm), 4),
                "t_measured_ms": round(t_dd, 4),
                "int_add": {"adds_per_launch": int(adds), "achieved_tadds": round(add_rate, 3),
                            "peak_tadds": round(int_peak, 3), "t_min_ms": round(t_int, 4),
                            "peak_kind": "measured (hd_measure_int_add_rate, this run)",
                            "frac": round(t_int / t_dd, 4)},
                "hbm": {"bytes_per_launch": int(bytes_dd), "achieved_gbs": round(gbs, 2),
                        "peak_gbs": peaks["hbm_gbs"], "peak_kind": f"of {peak_kind}",
                        "t_min_ms": round(t_hbm, 4), "frac": round(t_hbm / t_dd, 4)},
                "note": "adds = sample-channel terms (nbeams x trials x output samples x "
                        "channels); the kernel packs four byte-wide terms into one 32-bit add "
                        "(SWAR), so it can run above the one-add-per-term bound"}
        rec = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic",
            "config": config_for(wk, D, world),
            "dedisp_tile": {"dm_block": tile[0], "time_block": tile[1],
                            "rows_per_stage": tile[2],
                            "chosen_by": tile_source},
            "stage_ms": {k: round(v / args.steps, 4) for k, v in stage.items()},
            "roofline": roof,
            "recall": {"snr_ge_8_found": hit, "snr_ge_8_injected": nstrong},
            "gpu_launches": int(launches),
            # timed gulps served by one CUDA graph replay each (hd_get_graph_replays)
            "graph_replays": int(replays),
            "clocks": clocks,
        }
        if ms_plain is not None:
            v_plain = whole_job_value(world, wk.beam_s, ms_plain_m)
            rec["plain"] = {"value": round(v_plain, 3), "unit": UNIT,
                            "ms_per_step": round(ms_plain_m, 3),
                            "form": f"{U} hd_execute_device calls per gulp",
                            "gpu_launches": int(launches_plain)}
            rec["batched_over_plain"] = round(value / v_plain, 3)
        if ms_e2e is not None:
            sync = {"value": round(whole_job_value(world, wk.beam_s, ms_e2e_m), 3),
                    "unit": UNIT,
                    "ms_per_step": round(ms_e2e_m, 3),
                    "h2d_bytes_per_step": int(U * fb_bytes),
                    "d2h_bytes_per_step": int(ncand * 64 + 128),
                    "stage_ms": {k: round(v / args.steps, 4)
                                 for k, v in stage_e2e.items()},
                    "host_buffer": "pinned (torch pin_memory)",
                    "api": "hd_execute_beams" if U > 1 else "hd_execute"}
            if ms_e2e_pf is not None:
                rec["e2e"] = {"value": round(whole_job_value(world, wk.beam_s, ms_e2e_pf_m), 3),
                              "unit": UNIT, "ms_per_step": round(ms_e2e_pf_m, 3),
                              "h2d_bytes_per_step": int(U * fb_bytes),
                              "d2h_bytes_per_step": int(ncand * 64 + 128),
                              "host_buffer": "pinned (torch pin_memory)",
                              "api": "hd_prefetch_beams + hd_execute_prefetched "
                                     "(gulp k+1 copied while gulp k is searched)"}
                rec["e2e_sync"] = sync
            else:
                rec["e2e"] = sync
        if survey is not None:
            rec["survey_plain"] = survey
        if clf_rec is not None:
            rec["classifier"] = clf_rec
        if uneven is not None:
            rec["uneven"] = uneven
        if not args.no_cpu_baseline:
            rec["cpu_baseline"] = cpu_baseline(args, wk)
        print(json.dumps(rec), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# forward multiply-adds of the classifier per candidate: 3x3 convolutions
# (rows x cols x c_out x c_in x 9 per layer, both branches) and the two
# fully connected layers
CLF_CONV = [(1, 8, 64, 64), (8, 16, 32, 32), (16, 32, 16, 16),
            (1, 8, 64, 256), (8, 16, 32, 128), (16, 32, 16, 64)]
CLF_MACS = sum(h * w_ * co * ci * 9 for ci, co, h, w_ in CLF_CONV) + 10240 * 16 + 16 * 2
CLF_PATCH_BYTES = (4096 + 16384) * 4


def classifier_bench(args, H, torch, dev, pl):
    """Classifier inference: (1) hd_score_candidates on the last gulp's
    candidates (patches extracted and scored on the GPU, scores to host);
    (2) throughput of hd_classifier_score_device on 4096 device-resident
    patch pairs.  Device times from the classifier's own CUDA events."""
    peaks, peak_kind = _peaks()
    out = {}
    with H.Classifier(seed=1, gpu_id=dev.index) as clf:
        n = len(pl.candidates()) if pl is not None else 0
        if n:
            for _ in range(2):
                pl.scores(clf)
            dev_ms, wall = 0.0, 0.0
            for _ in range(args.steps):
                t0 = time.perf_counter()
                pl.scores(clf)
                wall += time.perf_counter() - t0
                dev_ms += clf.last_score_ms()
            out["gulp"] = {"api": "hd_score_candidates", "candidates": n,
                           "network_ms": round(dev_ms / args.steps, 4),
                           "call_ms_host_clock": round(wall * 1e3 / args.steps, 4)}
        nb = 4096
        g = torch.Generator(device=dev).manual_seed(5)
        dm = torch.randn((nb, 64, 64), generator=g, device=dev, dtype=torch.float32)
        ft = torch.randn((nb, 64, 256), generator=g, device=dev, dtype=torch.float32)
        torch.cuda.synchronize(dev)
        for _ in range(2):
            clf.score_device(dm.data_ptr(), ft.data_ptr(), nb)
        ms = 0.0
        for _ in range(args.steps):
            clf.score_device(dm.data_ptr(), ft.data_ptr(), nb)
            ms += clf.last_score_ms()
        ms /= args.steps
        flops = 2.0 * CLF_MACS * nb
        tflops = flops / (ms / 1e3) / 1e12
        gbs = CLF_PATCH_BYTES * nb / (ms / 1e3) / 1e9
        out["throughput"] = {
            "api": "hd_classifier_score_device", "candidates": nb,
            "ms": round(ms, 4), "candidates_per_s": round(nb / (ms / 1e3), 1),
            "flop_per_candidate": int(2 * CLF_MACS),
            "tensor": {"achieved_tflops": round(tflops, 3), "peak": peaks["bf16_tflops"],
                       "frac": round(tflops / peaks["bf16_tflops"], 5),
                       "peak_kind": f"of {peak_kind}"},
            "patch_read": {"achieved_gbs": round(gbs, 2), "peak": peaks["hbm_gbs"],
                           "frac": round(gbs / peaks["hbm_gbs"], 5),
                           "bytes_per_candidate": CLF_PATCH_BYTES},
            "note": "untrained weights (the work does not depend on their values); one "
                    "persistent fused kernel (k_clf_infer, one CTA per SM): mma.sync BF16 "
                    "convolutions with FP32 accumulation, FC layers in the same kernel"}
    out["training_gemm"] = training_gemm_bench(args, H, torch, dev, peaks, peak_kind)
    return out


def training_gemm_bench(args, H, torch, dev, peaks, peak_kind):
    """The training GEMM kernel (hd_bf16_gemm_tc: tcgen05.mma, TMEM
    accumulators, TMA-staged operands) on an im2col-shaped product: M =
    131072 patch pixels, N = 128 output channels (the kernel's widest tile),
    K = 1152 (3 x 3 taps x 128 input channels), FP32 out.  With N <= 128 the
    arithmetic intensity stays below the B200's ridge point, so the bound is
    HBM (A read once); both fractions are reported."""
    import ctypes as C
    M, N, K = 131072, 128, 1152
    g = torch.Generator(device=dev).manual_seed(9)
    A = torch.randn((M, K), generator=g, device=dev).to(torch.bfloat16)
    B = torch.randn((N, K), generator=g, device=dev).to(torch.bfloat16)
    Cm = torch.empty((M, N), device=dev, dtype=torch.float32)
    L = H.lib()

    def run():
        err = L.hd_bf16_gemm_tc(M, N, K, A.data_ptr(), K, 1, B.data_ptr(), 1, K,
                                C.cast(Cm.data_ptr(), C.POINTER(C.c_float)), N, 1, 0, 1)
        assert err == H.HD_NO_ERROR, H.error_string(err)

    for _ in range(3):
        run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = max(args.steps, 5)
    torch.cuda.synchronize(dev)
    e0.record()
    for _ in range(n):
        run()
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / n
    flops = 2.0 * M * N * K
    nbytes = 2 * M * K + 2 * N * K + 4 * M * N
    tf = flops / (ms / 1e3) / 1e12
    gbs = nbytes / (ms / 1e3) / 1e9
    return {"api": "hd_bf16_gemm_tc", "m": M, "n": N, "k": K, "ms": round(ms, 4),
            "tensor": {"achieved_tflops": round(tf, 2), "peak": peaks["bf16_tflops"],
                       "frac": round(tf / peaks["bf16_tflops"], 4), "peak_kind": f"of {peak_kind}"},
            "hbm": {"bytes": nbytes, "achieved_gbs": round(gbs, 1), "peak": peaks["hbm_gbs"],
                    "frac": round(gbs / peaks["hbm_gbs"], 4), "peak_kind": f"of {peak_kind}"},
            "bound": "hbm" if flops / nbytes < peaks["bf16_tflops"] * 1e3 / peaks["hbm_gbs"]
            else "tensor"}


def uneven_bench(args, H, torch, dev, barrier, dist, world):
    """Beams of different shapes (channel counts 128/512/2048/4096, 64/128 us,
    gulp lengths uniform in [2^14, nsamps_max], DM ranges 0-500/2000/5000 as
    fit) from device memory: the plain per-beam loop (one pipeline per
    configuration, hd_execute_device beam by beam) against one
    hd_execute_beam_set call.  Data: Gaussian noise (128, 16) with the
    survey beam's RFI (5 % of channels at +40 sd, zero-DM bursts of 1-50
    samples at +8 sd), generated on the GPU; injected-pulse recall is covered
    by the parity tests."""
    from heimdall_multibeam_b200 import synth
    ws = synth.uneven_shapes(args.uneven_beams, nsamps_range=(1 << 14, args.uneven_nsamps_max))
    g = torch.Generator(device=dev).manual_seed(2027)
    data = []
    for b, w in enumerate(ws):
        x = torch.randn((w.nsamps, w.nchans), generator=g, device=dev) * 16.0 + 128.0
        bad = torch.randperm(w.nchans, generator=g, device=dev)[: max(1, w.nchans // 20)]
        x[:, bad] += 640.0
        frac = w.nsamps * w.dt / ((1 << 18) * 64e-6)
        for _ in range(max(1, int(round(10 * frac)))):
            t0 = int(torch.randint(0, w.nsamps - 50, (1,), generator=g, device=dev))
            wd = int(torch.randint(1, 51, (1,), generator=g, device=dev))
            x[t0:t0 + wd, :] += 128.0
        data.append(x.round_().clamp_(0, 255).to(torch.uint8))
        del x
    torch.cuda.synchronize(dev)
    params = []
    for b, w in enumerate(ws):
        p = params_for(H, w)
        p.gpu_id = dev.index
        p.beam = b
        params.append(p)
    ptrs = [d.data_ptr() for d in data]
    ns = [w.nsamps for w in ws]
    beam_s = sum(w.nsamps * w.dt for w in ws)
    steps = max(1, args.uneven_steps)
    # plain per-beam loop
    pls = {}
    for w, p in zip(ws, params):
        key = (w.nchans, w.dt, w.dm_max)
        if key not in pls:
            pls[key] = H.Pipeline(p, cleaning=True)

    def plain():
        for w, ptr in zip(ws, ptrs):
            pls[(w.nchans, w.dt, w.dm_max)].execute_device(ptr, w.nsamps)

    plain()
    ms_plain = _timed(torch, dev, barrier, steps, plain)
    for pl in pls.values():
        pl.close()
    pls.clear()
    # one call for all beams
    with H.BeamSet(params, workers=args.uneven_workers, cleaning=True) as bs:
        def batched():
            err, _, _ = bs.execute(ptrs, nsamps=ns, on_device=True)
            assert err in (H.HD_NO_ERROR, H.HD_TOO_MANY_EVENTS, H.HD_TOO_FEW_NSAMPS), err
        batched()
        ms_set = _timed(torch, dev, barrier, steps, batched)
        nconf = bs.nconfigs
        ncand = sum(len(bs.candidates(b)) for b in range(len(ws)))
    ms_plain, ms_set = max_over_ranks(torch, dist, [ms_plain, ms_set], dev)
    return {"workload": f"uneven_{len(ws)}x_c128-4096_n16384-{args.uneven_nsamps_max}",
            "nbeams": len(ws), "configurations": nconf,
            "input_gib": round(sum(w.nchans * w.nsamps for w in ws) / 2**30, 3),
            "beam_seconds": round(beam_s, 3), "steps": steps,
            "beam_set": {"value": round(whole_job_value(world, beam_s, ms_set), 3), "unit": UNIT,
                         "ms_per_step": round(ms_set, 3), "workers": args.uneven_workers,
                         "api": "hd_execute_beam_set"},
            "plain": {"value": round(whole_job_value(world, beam_s, ms_plain), 3), "unit": UNIT,
                      "ms_per_step": round(ms_plain, 3),
                      "form": "one pipeline per configuration, hd_execute_device per beam"},
            "set_over_plain": round(ms_plain / ms_set, 3), "candidates": ncand,
            "data": "GPU-generated noise + RFI (no injections)"}


def survey_plain(args, H, torch, dev, barrier, dist, world):
    """The plain single-beam survey gulp (1024 ch, 2^18 samples, RFI cleaning)
    through hd_execute_device (value) and hd_execute from pinned memory (e2e)."""
    wk = workload("survey")
    w = wk.w
    nsamps = wk.nsamps
    p = params_for(H, w)
    p.gpu_id = dev.index
    pl = H.Pipeline(p, cleaning=True)
    d_fb = torch.from_numpy(wk.fbs[0]).to(dev)
    h_fb = torch.from_numpy(wk.fbs[0]).pin_memory()
    for _ in range(args.warmup):
        pl.execute_device(d_fb.data_ptr(), nsamps)
    stage = {k: 0.0 for k in pl.timing()}
    ms = _timed(torch, dev, barrier, args.steps,
                lambda: pl.execute_device(d_fb.data_ptr(), nsamps), stage, pl.timing)
    cands = pl.candidates()
    pl.execute_ptr(h_fb.data_ptr(), nsamps)
    ms_e2e = _timed(torch, dev, barrier, args.steps,
                    lambda: pl.execute_ptr(h_fb.data_ptr(), nsamps))
    pl.close()
    ms, ms_e2e = max_over_ranks(torch, dist, [ms, ms_e2e], dev)
    hit, nstrong = recall(cands, wk.pulses[0], w.dt)
    return {"workload": w.name, "value": round(whole_job_value(world, wk.beam_s, ms), 3),
            "unit": UNIT,
            "ms_per_step": round(ms, 3),
            "e2e": round(whole_job_value(world, wk.beam_s, ms_e2e), 3),
            "e2e_ms_per_step": round(ms_e2e, 3),
            "stage_ms": {k: round(v / args.steps, 4) for k, v in stage.items()},
            "recall": {"snr_ge_8_found": hit, "snr_ge_8_injected": nstrong}}


class _QuietStdout:
    """Sends file descriptor 1 to /dev/null (the reference prints a line per
    gulp), so that the JSON line stays the only output."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        fd = os.open(os.devnull, os.O_WRONLY)
        os.dup2(fd, 1)
        os.close(fd)

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)


def _ref_run(fb, w, threads, dm_max=None):
    """Seconds the reference pipeline takes on one filterbank (its own timer
    around hd_execute) and the number of DM trials searched."""
    import oracle
    dm_max = w.dm_max if dm_max is None else dm_max
    kw = dict(dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min, dm_max=dm_max,
              boxcar_max=w.boxcar_max, clean=int(w.clean))
    with _QuietStdout():
        err, proc, lines, secs = oracle.ref_execute(fb, nthreads=threads, **kw)
    d = len(oracle.dm_list(w.dm_min, dm_max, w.dt, 40.0, w.f0, w.df, w.nchans, 1.25))
    return secs, d


# ---- the reference on whole beams in parallel worker processes ---------------
# The reference deploys one heimdall process per beam; on the host cores the
# CPU reference runs the same way: P spawned worker processes, each running
# whole beams through the reference pipeline with T = cores / P threads (its
# stage code and its dedisperser).  The beams are read from one .npy file
# mapped by every worker.
_REF_W = None


def _ref_worker_init(path, wdict, threads):
    global _REF_W
    import dataclasses  # noqa: F401
    import oracle
    from heimdall_multibeam_b200 import synth
    oracle.ref_set_dedisp_threads(threads)
    _REF_W = (np.load(path, mmap_mode="r"), synth.Workload(**wdict), threads)


def _ref_worker_beam(u):
    fbs, w, threads = _REF_W
    secs, _ = _ref_run(np.ascontiguousarray(fbs[u]), w, threads)
    return secs


class RefPool:
    """Worker processes that search whole beams of one gulp with the
    reference pipeline.  gulp() returns the wall seconds of one gulp."""

    def __init__(self, wk, procs=None):
        import dataclasses
        import multiprocessing as mp
        import tempfile
        cores = os.cpu_count() or 1
        self.units = wk.units
        self.procs = max(1, min(procs or min(wk.units, cores), cores))
        self.threads = max(1, cores // self.procs)
        self.cores = self.procs * self.threads
        self.tmp = tempfile.TemporaryDirectory()
        path = os.path.join(self.tmp.name, "gulp.npy")
        np.save(path, np.stack(wk.fbs))
        ctx = mp.get_context("spawn")
        self.pool = ctx.Pool(self.procs, initializer=_ref_worker_init,
                             initargs=(path, dataclasses.asdict(wk.w), self.threads))

    def warm(self):
        """Each worker searches one beam (loads the library, touches its
        memory); untimed."""
        self.pool.map(_ref_worker_beam, [u % self.units for u in range(self.procs)],
                      chunksize=1)

    def gulp(self):
        t0 = time.perf_counter()
        self.pool.map(_ref_worker_beam, range(self.units), chunksize=1)
        return time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()
        self.tmp.cleanup()


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _ref_survey_gulp(args, wk, threads):
    """(seconds per gulp, description) of the reference on the single-beam
    survey gulp: two DM-range subsets, extrapolated linearly in the DM count
    (fixed cleaning cost + per-DM cost)."""
    import oracle
    w = wk.w
    d_full = len(oracle.dm_list(w.dm_min, w.dm_max, w.dt, 40.0, w.f0, w.df, w.nchans, 1.25))
    s1, d1 = _ref_run(wk.fbs[0], w, threads, args.ref_dm1)
    s2, d2 = _ref_run(wk.fbs[0], w, threads, args.ref_dm2)
    per_dm = max((s2 - s1) / max(d2 - d1, 1), 0.0)
    fixed = max(s1 - per_dm * d1, 0.0)
    t_full = fixed + per_dm * d_full
    return t_full, (f"reference pipeline (Thrust OpenMP build), {threads} threads, on DM "
                    f"0-{args.ref_dm1} ({d1} trials, {s1:.1f} s) and 0-{args.ref_dm2} ({d2} "
                    f"trials, {s2:.1f} s); gulp time extrapolated to {d_full} trials = "
                    f"{t_full:.1f} s")


def _ref_sample_text(pool, t_gulp, wk):
    return (f"reference pipeline (Pipeline/*.cu on Thrust's OpenMP backend + CPU "
            f"brute-force dedisperser), the whole {wk.units}-beam gulp: {pool.procs} worker "
            f"processes x {pool.threads} threads, one hd_execute per beam as the reference "
            f"runs them; {t_gulp:.2f} s per gulp")


def _one_thread_beam(wk):
    """Seconds of one beam of the gulp with one thread (reference timer)."""
    import oracle
    oracle.ref_set_dedisp_threads(1)
    try:
        return _ref_run(wk.fbs[0], wk.w, 1)[0]
    finally:
        oracle.ref_set_dedisp_threads(0)


def cpu_baseline(args, wk):
    """The reference on the host cores, one whole gulp (about 10 s of CPU
    time on the multibeam gulp), rank 0 at N = 1."""
    import oracle
    if not oracle.ref_available():
        return {"unavailable": "reference build oracle/_ref not present"}
    if wk.units == 1:
        threads = os.cpu_count() or 1
        t_gulp, sample = _ref_survey_gulp(args, wk, threads)
        return {"value": round(wk.beam_s / t_gulp, 4), "unit": UNIT, "cores": threads,
                "kind": "reference", "sample": sample, "seconds_per_gulp": round(t_gulp, 2)}
    pool = RefPool(wk, args.ref_procs)
    try:
        pool.warm()
        t_gulp = pool.gulp()
    finally:
        pool.close()
    return {"value": round(wk.beam_s / t_gulp, 4), "unit": UNIT, "cores": pool.cores,
            "kind": "reference", "sample": _ref_sample_text(pool, t_gulp, wk),
            "seconds_per_gulp": round(t_gulp, 3), "cpu_model": _cpu_model()}


def run_reference(args):
    rank = _env_int("RANK", 0)
    if rank != 0:
        return
    import oracle
    wk = workload(args.workload, args.nsamps, args.nbeams)
    w = wk.w
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing"}))
        return
    D = len(oracle.dm_list(w.dm_min, w.dm_max, w.dt, 40.0, w.f0, w.df, w.nchans, 1.25))
    config = config_for(wk, D, args.gpus)
    t_wall0 = time.time()
    if wk.units == 1:
        threads = os.cpu_count() or 1
        cores = threads
        for _ in range(args.warmup):
            _ref_run(wk.fbs[0], w, threads, args.ref_dm1)
        runs = [_ref_survey_gulp(args, wk, threads) for _ in range(args.steps)]
        times = [t for t, _ in runs]
        sample = runs[-1][1]
    else:
        pool = RefPool(wk, args.ref_procs)
        try:
            # warm-up steps: every worker searches one beam (untimed)
            for _ in range(args.warmup):
                pool.warm()
            # timed steps: the whole gulp each
            times = [pool.gulp() for _ in range(args.steps)]
        finally:
            pool.close()
        cores = pool.cores
        sample = _ref_sample_text(pool, float(np.median(times)), wk)
    t_gulp = float(np.mean(times))
    value = wk.beam_s / t_gulp
    one = _one_thread_beam(wk)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t_gulp * 1e3, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": cores,
                         "kind": "reference", "sample": sample,
                         "cpu_model": _cpu_model(),
                         "one_thread_seconds_per_beam": round(one, 3),
                         "one_thread_value": round(wk.beam_s / wk.units / one, 4)},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "step_seconds": [round(t, 3) for t in times],
        "wall_s": round(time.time() - t_wall0, 1)}), flush=True)


def stream_file_bench(args, H, torch):
    """The sigproc file gulp loop's steady state.  "survey": one file of the
    survey beam's shape (1024 ch, 64 us, DM 0-2000, boxcars to 4096,
    cleaning on; gulps of 2^18 new spectra) through hd_search_sigproc_file.
    "multibeam": 36 one-beam files of the multibeam gulp's shape (320 ch,
    655.36 us, DM 0-2000, boxcars to 512, cleaning off; gulps of 2^15 new
    spectra per file) through hd_search_sigproc_files, one batched search
    per gulp.  Reported: the time between consecutive gulps' callbacks
    against the device-resident search of one full gulp, and the start-up
    before the first gulp.  The files are written to a temporary directory
    and read once before timing (page cache)."""
    import ctypes as C
    import tempfile
    from heimdall_multibeam_b200 import synth
    multi = args.stream_workload == "multibeam"
    w = synth.SEARCH_C2 if multi else synth.SEARCH_C1
    nfiles = w.nbeams if multi else 1
    G = 1 << 15 if multi else 1 << 18
    nblocks = max(3, args.stream_blocks)
    rng = np.random.default_rng(5)
    data = rng.integers(100, 156, size=(nblocks * G + 1000, w.nchans), dtype=np.uint8)
    out = {"workload": f"sigproc_files_{nfiles}x_c{w.nchans}_{nblocks}x{G}",
           "api": "hd_search_sigproc_files" if multi else "hd_search_sigproc_file"}
    with tempfile.TemporaryDirectory(dir=args.stream_dir) as tmp:
        paths = []
        for u in range(nfiles):
            path = os.path.join(tmp, f"beam{u:02d}.fil")
            synth.write_sigproc(path, data, nchans=w.nchans, nbits=8, tsamp=w.dt, fch1=w.f0,
                                foff=w.df, tstart=60000.5, nifs=1, ibeam=u + 1,
                                source_name="stream")
            with open(path, "rb") as f:
                while f.read(1 << 26):
                    pass
            paths.append(path)
        kw = dict(dm_min=w.dm_min, dm_max=w.dm_max, boxcar_max=w.boxcar_max, output_dir=None)
        q = H.default_params(**kw)
        q.override_beam = True
        params = H.params_from_sigproc(paths[0], q)
        with H.Pipeline(params, cleaning=not multi) as pl:
            M = pl.max_overlap()
            stamps = []
            fn = H.GULP_CALLBACK(lambda user, cands, n, first: stamps.append(time.perf_counter()))
            tot, ng = C.c_size_t(0), C.c_size_t(0)
            arr = (C.c_char_p * nfiles)(*[p.encode() for p in paths])
            for rep in range(2):  # the first pass tunes and allocates
                stamps.clear()
                t0 = time.perf_counter()
                err = H.lib().hd_search_sigproc_files(pl._p, arr, nfiles, G, fn, None,
                                                      C.byref(tot), C.byref(ng))
                t1 = time.perf_counter()
                assert err in (H.HD_NO_ERROR, H.HD_TOO_MANY_EVENTS), err
            gaps = [1e3 * (b - a) for a, b in zip(stamps, stamps[1:])]
            d = torch.from_numpy(data[:G + M]).cuda()
            torch.cuda.synchronize()
            ts = []
            for _ in range(4):
                err, _, _ = pl.execute_beams([d.data_ptr()] * nfiles, nsamps=G + M,
                                             on_device=True, raise_on_error=False)
                ts.append(pl.timing()["total"])
    steady = float(np.median(gaps))
    out.update({"files": nfiles, "gulps": ng.value, "ms_between_gulps": round(steady, 2),
                "ms_between_gulps_all": [round(g, 2) for g in gaps],
                "device_search_ms": round(min(ts[1:]), 2),
                "startup_ms": round(1e3 * (stamps[0] - t0), 1),
                "beam_s_per_s_steady": round(nfiles * G * w.dt / (steady * 1e-3), 1),
                "beam_s_per_s_whole_call": round(nfiles * tot.value * w.dt / (t1 - t0), 1)})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="multibeam", choices=["multibeam", "survey"])
    ap.add_argument("--nsamps", type=int, default=None,
                    help="samples per beam (smaller gulps are for profiling)")
    ap.add_argument("--nbeams", type=int, default=None,
                    help="beams of the multibeam gulp (fewer are for profiling)")
    ap.add_argument("--batched-only", action="store_true",
                    help="time only the batched form (profiling)")
    ap.add_argument("--uneven-beams", type=int, default=256,
                    help="beams of the uneven-beam section (0 skips it)")
    ap.add_argument("--uneven-nsamps-max", type=int, default=1 << 17,
                    help="longest gulp of the uneven-beam section")
    ap.add_argument("--uneven-workers", type=int, default=4)
    ap.add_argument("--uneven-steps", type=int, default=2)
    ap.add_argument("--no-classifier", action="store_true",
                    help="skip the classifier inference measurement")
    ap.add_argument("--only-classifier", action="store_true",
                    help="only the classifier throughput (profiling); prints its object")
    ap.add_argument("--no-survey", action="store_true",
                    help="skip the secondary single-beam survey gulp")
    ap.add_argument("--ref-procs", type=int, default=None,
                    help="worker processes of the reference on the multibeam gulp "
                         "(default: one per core, at most one per beam)")
    ap.add_argument("--ref-dm1", type=float, default=20.0)
    ap.add_argument("--ref-dm2", type=float, default=60.0)
    ap.add_argument("--only-stream-file", action="store_true",
                    help="only the sigproc file gulp loop (writes a temporary file)")
    ap.add_argument("--stream-blocks", type=int, default=7)
    ap.add_argument("--stream-workload", default="survey", choices=["survey", "multibeam"])
    ap.add_argument("--stream-dir", default=None,
                    help="directory for the temporary file (default: the system's)")
    args = ap.parse_args()
    if args.only_stream_file:
        import torch
        import heimdall_multibeam_b200 as H
        torch.cuda.set_device(0)
        print(json.dumps({"stream_file": stream_file_bench(args, H, torch)}), flush=True)
        return
    if args.only_classifier:
        import torch
        import heimdall_multibeam_b200 as H
        torch.cuda.set_device(0)
        print(json.dumps({"classifier": classifier_bench(args, H, torch,
                                                         torch.device("cuda", 0), None)}),
              flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
