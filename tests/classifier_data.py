"""Builds labelled candidate sets for the classifier tests: seeded training
gulps (synth.make_training_beam) searched by the pipeline itself (cleaning
off, so RFI reaches the candidate list), patches from hd_extract_patches,
label 1 for candidates that recover an injected pulse."""
import numpy as np

import heimdall_multibeam_b200 as H
from heimdall_multibeam_b200 import synth


def build(seeds, batch: int = 16, w=synth.TRAIN):
    """Returns dict(dm, ft, label, pulse_id, rfi, snr, gulp) over all
    candidates of the gulps, and per gulp the injected pulses."""
    p = H.default_params(nchans=w.nchans, dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min,
                         dm_max=w.dm_max, boxcar_max=w.boxcar_max, output_dir=None)
    dms, fts, labels, pid, rfi, snr, gulp = [], [], [], [], [], [], []
    pulses_all = []
    seeds = list(seeds)
    with H.Pipeline(p, cleaning=False) as pl:
        for i0 in range(0, len(seeds), batch):
            chunk = seeds[i0:i0 + batch]
            made = [synth.make_training_beam(s, w) for s in chunk]
            err, _, st = pl.execute_beams([b.data for b, _ in made])
            assert err in (H.HD_NO_ERROR, H.HD_TOO_MANY_EVENTS)
            dm, ft = pl.patches()
            rows = pl.candidates()
            k = 0
            for u, (b, ev) in enumerate(made):
                cu = pl.candidates(u)
                g = len(pulses_all)
                pulses_all.append(b.pulses)
                for c in cu:
                    m = synth.match_pulse(c, b.pulses, w.dt)
                    t = int(c["samp_idx"])
                    in_rfi = any(e.t0 - 2048 <= t <= e.t0 + e.length + 2048 for e in ev)
                    labels.append(1 if m >= 0 else 0)
                    pid.append(m)
                    rfi.append(1 if (m < 0 and in_rfi) else 0)
                    snr.append(float(c["snr"]))
                    gulp.append(g)
                dms.append(dm[k:k + len(cu)])
                fts.append(ft[k:k + len(cu)])
                k += len(cu)
            assert k == len(rows)
    return dict(dm=np.concatenate(dms), ft=np.concatenate(fts), label=np.array(labels, np.int32),
                pulse_id=np.array(pid), rfi=np.array(rfi, np.int32), snr=np.array(snr),
                gulp=np.array(gulp)), pulses_all


def recall_and_reduction(d, pulses_all, scores, thresh=0.5, snr_min=8.0):
    """(plain recall, classified recall, non-pulse kept fraction, RFI kept
    fraction) at S/N >= snr_min for the injected pulses."""
    found0 = found1 = total = 0
    for g, pulses in enumerate(pulses_all):
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
    kept_other = (scores[other] >= thresh).mean() if other.any() else 0.0
    kept_rfi = (scores[rfi] >= thresh).mean() if rfi.any() else 0.0
    return found0 / max(total, 1), found1 / max(total, 1), kept_other, kept_rfi, total
