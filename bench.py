#!/usr/bin/env python
"""Benchmark of the per-gulp single-pulse search (Heimdall's hd_execute).

Workload: one gulp of the plain single-beam search at survey size with RFI --
1024 channels uint8, 1520 MHz top, -0.390625 MHz channels, 64 us, 2^18
samples (16.78 beam-seconds), DM 0-2000 (tol 1.25, 40 us), boxcars 2^0..2^12,
threshold 6, clean_filterbank_rfi on; seeded synthetic data (noise N(128,16^2),
20 injected dispersed pulses, narrow-band and zero-DM RFI).

Metric: beam-seconds searched per second.
  value  -- K gulps through hd_execute_device with the filterbank resident in
            HBM; CUDA events around the K calls (each call ends synchronised).
  e2e    -- the same K gulps through hd_execute (the drop-in C entry point)
            from pinned host memory: host->device copy of the gulp inside the
            timed region, candidate rows read back every step.
The input (256 MiB) is larger than L2 (126 MB), so no L2 flush is needed.

`--impl reference` times the reference's own stage code (Pipeline/*.cu rebuilt
on Thrust's OpenMP backend, oracle/_ref) with all host threads on a bounded
sample of the same gulp (a DM-range subset) and scales by the DM count.

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


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
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
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
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
        except Exception:
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


def workload(nsamps=None):
    from heimdall_multibeam_b200 import synth
    w = synth.SEARCH_C1
    b = synth.make_c1(nsamps=nsamps)
    if nsamps:
        import dataclasses
        w = dataclasses.replace(w, name=f"plain_c1024_n{nsamps}_rfi", nsamps=nsamps)
    return w, b


def params_for(H, w):
    return H.default_params(nchans=w.nchans, dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min,
                            dm_max=w.dm_max, boxcar_max=w.boxcar_max, output_dir=None)


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

    w, b = workload(args.nsamps)
    nsamps, nchans = b.data.shape
    beam_s = nsamps * w.dt
    p = params_for(H, w)
    p.gpu_id = dev.index
    pl = H.Pipeline(p, cleaning=True)

    d_fb = torch.from_numpy(b.data).to(dev)
    h_fb = torch.from_numpy(b.data).pin_memory()
    torch.cuda.synchronize(dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # ---- device-resident input --------------------------------------------
    for _ in range(args.warmup):
        err, proc = pl.execute_device(d_fb.data_ptr(), nsamps)
        assert err == 0, H.error_string(err)
    cands = pl.candidates()
    l0 = H.launch_count()
    stage = {k: 0.0 for k in pl.timing()}
    clk = ClockSampler(dev.index)
    clk.start()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        err, proc = pl.execute_device(d_fb.data_ptr(), nsamps)
        t = pl.timing()
        for k in stage:
            stage[k] += t[k]
    e1.record()
    barrier()
    clocks = clk.stop()
    launches = H.launch_count() - l0
    ms = e0.elapsed_time(e1) / args.steps

    # ---- end to end through hd_execute from pinned host memory --------------
    for _ in range(max(1, args.warmup // 2)):
        pl.execute_ptr(h_fb.data_ptr(), nsamps)
    barrier()
    e0.record()
    ncand = 0
    stage_e2e = {k: 0.0 for k in stage}
    for _ in range(args.steps):
        err, proc = pl.execute_ptr(h_fb.data_ptr(), nsamps)
        ncand = len(pl.candidates())
        t = pl.timing()
        for k in stage_e2e:
            stage_e2e[k] += t[k]
    e1.record()
    barrier()
    ms_e2e = e0.elapsed_time(e1) / args.steps

    tmax = torch.tensor([ms, ms_e2e], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    ms, ms_e2e = float(tmax[0]), float(tmax[1])
    value = world * beam_s / (ms / 1e3)
    e2e = world * beam_s / (ms_e2e / 1e3)

    if rank == 0:
        peaks, peak_kind = _peaks()
        # dominant kernel: brute-force dedispersion
        plan = H.DedispPlan(nchans, w.dt, w.f0, w.df)
        plan.generate_dm_list(w.dm_min, w.dm_max, 40.0, 1.25)
        D = len(plan.dm_list)
        nout = nsamps - plan.max_delay
        t_dd = stage["dedisperse"] / args.steps  # ms, events on the pipeline stream
        bytes_dd = nchans * nsamps + D * nout * 4
        adds = D * nout * nchans
        achieved = bytes_dd / (t_dd / 1e3) / 1e9
        sm_mhz = clocks.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
        int_peak = 148 * 128 * sm_mhz * 1e6 / 1e12  # Tadd/s, INT32 lanes x clock
        int_ach = adds / (t_dd / 1e3) / 1e12
        traffic = None
        try:
            # DRAM bytes per k_dedisp launch from the committed ncu summary
            with open(os.path.join(ROOT, "profiles", "k_dedisp_c1024_n131072.md")) as f:
                for ln in f:
                    if ln.startswith("traffic_bytes_per_launch_full_size:"):
                        traffic = int(ln.split(":")[1])
            if nsamps != 262144:
                traffic = None
        except Exception:
            pass
        hit, nstrong = recall(cands, b.pulses, w.dt)
        rec = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic",
            "config": {"workload": w.name, "nchans": nchans, "nsamps": nsamps, "nbeams": 1,
                       "dt_s": w.dt, "dm_range": [w.dm_min, w.dm_max], "dm_trials": D,
                       "boxcar_max": w.boxcar_max, "clean_filterbank_rfi": True,
                       "beam_seconds_per_gulp": round(beam_s, 4),
                       "l2": "input 256 MiB > L2, no flush", "parallelism": f"replicas{world}"},
            "e2e": {"value": round(e2e, 3), "unit": UNIT, "ms_per_step": round(ms_e2e, 3),
                    "h2d_bytes_per_step": int(nsamps * nchans),
                    "d2h_bytes_per_step": int(ncand * 64 + 128),
                    "stage_ms": {k: round(v / args.steps, 4) for k, v in stage_e2e.items()},
                    "host_buffer": "pinned (torch pin_memory)"},
            "stage_ms": {k: round(v / args.steps, 4) for k, v in stage.items()},
            "roofline": {"kernel": "k_dedisp", "bound": "hbm", "achieved": round(achieved, 2),
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic,
                         "peak_kind": f"of {peak_kind}",
                         "int_add": {"achieved_tadds": round(int_ach, 3),
                                     "peak_tadds": round(int_peak, 3),
                                     "frac": round(int_ach / int_peak, 4),
                                     "basis": "148 SMs x 128 INT32 lanes x median SM clock"},
                         "binding": "int_add"},
            "recall": {"snr_ge_8_found": hit, "snr_ge_8_injected": nstrong},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if not args.no_cpu_baseline:
            rec["cpu_baseline"] = cpu_baseline(args, b, w, beam_s)
        print(json.dumps(rec), flush=True)
    pl.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def _ref_sample(b, w, dm_max, threads):
    import oracle
    kw = dict(dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min, dm_max=dm_max,
              boxcar_max=w.boxcar_max, clean=1)
    err, proc, lines, secs = oracle.ref_execute(b.data, nthreads=threads, **kw)
    d = len(oracle.dm_list(w.dm_min, dm_max, w.dt, 40.0, w.f0, w.df, w.nchans, 1.25))
    return secs, d


def cpu_baseline(args, b, w, beam_s):
    """The reference's stage code (Thrust OpenMP build) on two DM-range
    samples of the same gulp; gulp time extrapolated linearly in the DM count
    (fixed cleaning cost + per-DM cost)."""
    import oracle
    threads = os.cpu_count() or 1
    if not oracle.ref_available():
        return {"unavailable": "reference build oracle/_ref not present"}
    d_full = len(oracle.dm_list(w.dm_min, w.dm_max, w.dt, 40.0, w.f0, w.df, w.nchans, 1.25))
    s1, d1 = _ref_sample(b, w, args.ref_dm1, threads)
    s2, d2 = _ref_sample(b, w, args.ref_dm2, threads)
    per_dm = max((s2 - s1) / max(d2 - d1, 1), 0.0)
    fixed = max(s1 - per_dm * d1, 0.0)
    t_full = fixed + per_dm * d_full
    return {"value": round(beam_s / t_full, 4), "unit": UNIT, "cores": threads,
            "kind": "reference",
            "sample": f"reference pipeline on DM 0-{args.ref_dm1} ({d1} trials, {s1:.1f} s) and "
                      f"0-{args.ref_dm2} ({d2} trials, {s2:.1f} s); gulp time extrapolated to "
                      f"{d_full} trials = {t_full:.1f} s",
            "seconds_per_gulp": round(t_full, 2)}


def run_reference(args):
    rank = _env_int("RANK", 0)
    if rank != 0:
        return
    import oracle
    w, b = workload(args.nsamps)
    nsamps = b.data.shape[0]
    beam_s = nsamps * w.dt
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing"}))
        return
    threads = os.cpu_count() or 1
    d_full = len(oracle.dm_list(w.dm_min, w.dm_max, w.dt, 40.0, w.f0, w.df, w.nchans, 1.25))
    for _ in range(args.warmup):
        _ref_sample(b, w, args.ref_dm1, threads)
    times = []
    t0 = time.time()
    for _ in range(args.steps):
        s1, d1 = _ref_sample(b, w, args.ref_dm1, threads)
        times.append((s1, d1))
    wall = time.time() - t0
    s1 = float(np.median([t for t, _ in times]))
    s2, d2 = _ref_sample(b, w, args.ref_dm2, threads)
    per_dm = max((s2 - s1) / max(d2 - d1, 1), 0.0)
    fixed = max(s1 - per_dm * d1, 0.0)
    t_full = fixed + per_dm * d_full
    value = beam_s / t_full
    sample = (f"reference pipeline (Thrust OpenMP build) with {threads} threads on DM 0-"
              f"{args.ref_dm1} ({d1} trials) per step and 0-{args.ref_dm2} ({d2} trials) once; "
              f"gulp time extrapolated to {d_full} trials = {t_full:.1f} s")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t_full * 1e3, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": w.name, "nchans": w.nchans, "nsamps": nsamps, "dm_trials": d_full},
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "wall_s": round(wall, 1)}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nsamps", type=int, default=None,
                    help="gulp length (default 2^18); smaller gulps are for profiling")
    ap.add_argument("--ref-dm1", type=float, default=20.0)
    ap.add_argument("--ref-dm2", type=float, default=60.0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
