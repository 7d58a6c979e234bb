"""Synthetic per-beam .cand lists for the coincidence tests: clusters of
candidates shared by several beams (time within a few boxcar widths, S/N
ratios around the 0.4 cut, filters within and beyond the filter cut), exact
boundary cases, and unrelated candidates."""
import numpy as np

UTC = "2025-01-02-03:04:05"


def lines_by_beam(nbeams: int = 5, seed: int = 3):
    rng = np.random.default_rng(seed)
    beams = [[] for _ in range(nbeams)]
    for e in range(12):
        t = int(rng.integers(40000, 200000))
        f = int(rng.integers(0, 9))
        snr0 = float(rng.uniform(6, 40))
        dm = int(rng.integers(0, 1500))
        for b in rng.choice(nbeams, size=int(rng.integers(1, nbeams + 1)), replace=False):
            ff = max(0, f + int(rng.integers(-5, 6)))
            tt = t + int(rng.integers(-4, 5)) * (1 << max(f, ff))
            s = snr0 * float(rng.uniform(0.3, 2.5))
            beams[b].append((s, tt, ff, max(0, dm + int(rng.integers(-20, 21)))))
    # exact boundaries between beams 0 and 1: |dt| == 3 * 2^2, S/N 7 vs 3 (ratio 0.4)
    beams[0].append((7.0, 50000, 2, 100))
    beams[1].append((3.0, 50012, 2, 100))
    beams[1].append((3.0, 50013, 2, 100))   # one sample too far for beam 0's entry
    for b in range(nbeams):
        for _ in range(3):
            beams[b].append((float(rng.uniform(6, 9)), int(rng.integers(100, 250000)),
                             int(rng.integers(0, 12)), int(rng.integers(0, 1500))))
    out = []
    for b, lst in enumerate(beams):
        ls = []
        for s, t, f, dm in lst:
            ls.append("%g\t%d\t%g\t%d\t%d\t%g\t%d\t%d\t%d\t%d\t" % (
                np.float32(s), t, np.float32(t * 6.4e-5), f, dm, np.float32(dm * 1.3),
                int(rng.integers(1, 50)), t - 3, t + 3, b + 1))
        out.append(ls)
    return out


def write_files(tmp_path, beam_lines):
    files = []
    for b, ls in enumerate(beam_lines):
        p = tmp_path / ("%s_%02d.cand" % (UTC, b + 1))
        p.write_text("".join(x + "\n" for x in ls))
        files.append(str(p))
    return files


def format_all(rows, co):
    """_all.cand lines from parsed rows and (nbeams, primary, max_snr)."""
    return ["%g\t%d\t%g\t%d\t%d\t%g\t%d\t%d\t%d\t%d\t\t%d\t%g\t%d" % (
        r["snr"], r["samp_idx"], r["time"], r["filter"], r["dm_trial"], r["dm"], r["members"],
        r["begin"], r["end"], c[0], c[1], c[2], r["beam"]) for r, c in zip(rows, co)]
