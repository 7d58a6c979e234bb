"""Classifier training and evaluation at survey size.

Seeded survey-shaped gulps (1024 channels, 64 us, 2^18 samples, DM 0-2000,
boxcars to 4096) are generated on the GPU (synth.make_training_gulps_device)
and searched by the pipeline itself (hd_execute_beams on device memory,
cleaning off so that the RFI reaches the candidate list).  Each candidate is
labelled against the injections: a pulse if it recovers an injected pulse
(synth.match_pulse: |samp - t0| <= max(2^filter, FWHM/dt) + 2 and DM within
max(5 %, 2 trial steps)), RFI if it lies within 2048 samples of an RFI event,
noise otherwise.  The network is trained on the GPU (hd_classifier_train)
on every pulse candidate and seeded fractions of the RFI and noise
candidates (about as many as the pulse ones); held-out gulps, scored
through hd_score_candidates (patches extracted and scored on the GPU after
the merge), measure the recall of
injected S/N >= 8 pulses in the plain and the classified candidate lists and
the fraction of RFI candidates the score keeps.  The score threshold is the
largest that keeps 99.5 % of the plain recall on a validation set.

    python -m heimdall_multibeam_b200.training --out heimdall_multibeam_b200/classifier_survey

writes <out>.npy (the 175666 FP32 parameters) and <out>.json (threshold,
data, training and held-out results)."""
from __future__ import annotations

import argparse
import json
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import synth

THRESHOLDS = (0.002, 0.005, 0.01, 0.02, 0.05, 0.1, 0.2, 0.3, 0.5)


def params_for(H, w, gpu_id: int = 0):
    p = H.default_params(nchans=w.nchans, dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min,
                         dm_max=w.dm_max, boxcar_max=w.boxcar_max, output_dir=None)
    p.gpu_id = gpu_id
    return p


def label(cands, pulses, events, dt):
    """(label 1/0, matched pulse index or -1, RFI flag) per candidate."""
    lab, pid, rfi = [], [], []
    for c in cands:
        m = synth.match_pulse(c, pulses, dt)
        t = int(c["samp_idx"])
        in_rfi = any(e.t0 - 2048 <= t <= e.t0 + e.length + 2048 for e in events)
        lab.append(1 if m >= 0 else 0)
        pid.append(m)
        rfi.append(1 if (m < 0 and in_rfi) else 0)
    return lab, pid, rfi


def collect(H, torch, seeds: Sequence[int], w=None, chunk: int = 8, classifier=None,
            patches: bool = True, n_pulses: int = 40, n_rfi: int = 20, keep_rfi: float = 1.0,
            keep_noise: float = 1.0, seed: int = 0) -> Dict:
    """Searches the seeded gulps chunk by chunk.  Returns labels, matched
    pulse, RFI flag, S/N and gulp of every candidate, the injected pulses of
    every gulp, the classifier's scores (classifier given) and, with
    patches=True, the patches and labels of the kept candidates: every pulse
    candidate, and RFI and noise candidates with probabilities keep_rfi and
    keep_noise (seeded)."""
    w = w or synth.SEARCH_C1
    seeds = list(seeds)
    rng = np.random.default_rng(seed)
    out: Dict[str, List] = {k: [] for k in ("label", "pulse_id", "rfi", "snr", "gulp", "score",
                                             "dm", "ft", "kept_label", "kept_rfi")}
    pulses_all: List = []
    with H.Pipeline(params_for(H, w), cleaning=False) as pl:
        for i0 in range(0, len(seeds), chunk):
            part = seeds[i0:i0 + chunk]
            data, pulses, events = synth.make_training_gulps_device(torch, part, w, n_pulses,
                                                                    n_rfi)
            torch.cuda.synchronize()
            err, _, _ = pl.execute_beams([data[u].data_ptr() for u in range(len(part))],
                                         nsamps=w.nsamps, on_device=True)
            if err not in (H.HD_NO_ERROR, H.HD_TOO_MANY_EVENTS):
                raise H.HdError(err, "hd_execute_beams")
            if classifier is not None:
                out["score"].append(pl.scores(classifier))
            labs, rfis = [], []
            for u in range(len(part)):
                cu = pl.candidates(u)
                lab, pid, rfi = label(cu, pulses[u], events[u], w.dt)
                labs += lab
                rfis += rfi
                out["pulse_id"] += pid
                out["snr"] += [float(x) for x in cu["snr"]]
                out["gulp"] += [len(pulses_all)] * len(cu)
                pulses_all.append(pulses[u])
            out["label"] += labs
            out["rfi"] += rfis
            if patches and labs:
                la, ra = np.array(labs), np.array(rfis)
                u01 = rng.random(len(la))
                keep = (la == 1) | ((ra == 1) & (u01 < keep_rfi)) | \
                       ((la == 0) & (ra == 0) & (u01 < keep_noise))
                dm, ft = pl.patches()
                out["dm"].append(dm[keep])
                out["ft"].append(ft[keep])
                out["kept_label"].append(la[keep].astype(np.int32))
                out["kept_rfi"].append(ra[keep].astype(np.int32))
                del dm, ft
            del data
    d = {"label": np.array(out["label"], np.int32), "pulse_id": np.array(out["pulse_id"]),
         "rfi": np.array(out["rfi"], np.int32), "snr": np.array(out["snr"]),
         "gulp": np.array(out["gulp"]), "pulses_all": pulses_all}
    if out["score"]:
        d["score"] = np.concatenate(out["score"])
    if out["dm"]:
        d["dm"] = np.concatenate(out["dm"])
        d["ft"] = np.concatenate(out["ft"])
        d["kept_label"] = np.concatenate(out["kept_label"])
        d["kept_rfi"] = np.concatenate(out["kept_rfi"])
    return d


def recall_and_reduction(d: Dict, scores: np.ndarray, thresh: float,
                         snr_min: float = 8.0) -> Dict:
    """Recall of injected pulses with S/N >= snr_min in the plain list and in
    the list cut at score >= thresh; fractions of RFI and of all non-pulse
    candidates the cut keeps."""
    found0 = found1 = total = 0
    for g, pulses in enumerate(d["pulses_all"]):
        sel = d["gulp"] == g
        for k, pu in enumerate(pulses):
            if pu.snr < snr_min:
                continue
            total += 1
            hit = sel & (d["pulse_id"] == k)
            found0 += bool(hit.any())
            found1 += bool((hit & (scores >= thresh)).any())
    other = d["label"] == 0
    rfi = d["rfi"] == 1
    return {"threshold": thresh, "pulses": total,
            "recall_plain": found0 / max(total, 1), "recall_classified": found1 / max(total, 1),
            "rfi_candidates": int(rfi.sum()),
            "rfi_kept": float((scores[rfi] >= thresh).mean()) if rfi.any() else 0.0,
            "non_pulse_kept": float((scores[other] >= thresh).mean()) if other.any() else 0.0}


def main(argv: Optional[Sequence[str]] = None) -> None:
    import torch
    import heimdall_multibeam_b200 as H

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default="heimdall_multibeam_b200/classifier_survey")
    ap.add_argument("--train-gulps", type=int, default=1000)
    ap.add_argument("--keep-rfi", type=float, default=0.25,
                    help="fraction of RFI candidates kept for training")
    ap.add_argument("--keep-noise", type=float, default=0.25,
                    help="fraction of noise candidates kept for training")
    ap.add_argument("--val-gulps", type=int, default=64)
    ap.add_argument("--test-gulps", type=int, default=128)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=128)
    ap.add_argument("--lr", type=float, default=3e-4)
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args(argv)
    torch.cuda.set_device(0)
    w = synth.SEARCH_C1
    t0 = time.time()
    tr = collect(H, torch, range(0, args.train_gulps), w, keep_rfi=args.keep_rfi,
                 keep_noise=args.keep_noise, seed=args.seed)
    t_collect = time.time() - t0
    n_pos = int((tr["label"] == 1).sum())
    n_rfi = int((tr["rfi"] == 1).sum())
    n_noise = int(((tr["label"] == 0) & (tr["rfi"] == 0)).sum())
    kept = tr["kept_label"]
    t1 = time.time()
    with H.Classifier(seed=args.seed) as clf:
        losses = clf.train(tr["dm"], tr["ft"], kept, epochs=args.epochs, batch=args.batch,
                           lr=args.lr, seed=args.seed)
        t_train = time.time() - t1
        params = clf.params()
        kept_counts = {"pulse": int((kept == 1).sum()), "rfi": int(tr["kept_rfi"].sum()),
                       "noise": int(((kept == 0) & (tr["kept_rfi"] == 0)).sum())}
        del tr
        va = collect(H, torch, range(100000, 100000 + args.val_gulps), w, classifier=clf,
                     patches=False)
        te = collect(H, torch, range(200000, 200000 + args.test_gulps), w, classifier=clf,
                     patches=False)
    val = [recall_and_reduction(va, va["score"], th) for th in THRESHOLDS]
    ok = [v for v in val if v["recall_classified"] >= 0.995 * v["recall_plain"]]
    thresh = max(v["threshold"] for v in ok) if ok else min(THRESHOLDS)
    test = recall_and_reduction(te, te["score"], thresh)
    meta = {
        "workload": w.name, "cleaning": False,
        "generator": "synth.make_training_gulps_device (40 pulses, 20 RFI events per gulp)",
        "train": {"gulps": args.train_gulps,
                  "candidates_found": {"pulse": n_pos, "rfi": n_rfi, "noise": n_noise},
                  "candidates_used": kept_counts, "used": int(sum(kept_counts.values())),
                  "keep_rfi": args.keep_rfi, "keep_noise": args.keep_noise,
                  "epochs": args.epochs, "batch": args.batch, "lr": args.lr,
                  "epoch_loss": [round(float(x), 5) for x in losses],
                  "seconds_collect": round(t_collect, 1), "seconds_train": round(t_train, 1)},
        "threshold": thresh,
        "validation": {"gulps": args.val_gulps, "by_threshold": val},
        "test": dict(test, gulps=args.test_gulps),
    }
    np.save(args.out + ".npy", params.astype(np.float32))
    with open(args.out + ".json", "w") as f:
        json.dump(meta, f, indent=1)
    print(json.dumps({"threshold": thresh, "test": meta["test"], "train": meta["train"]}),
          flush=True)


if __name__ == "__main__":
    main()
