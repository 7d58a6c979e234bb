"""A seeded sweep of random small configurations through the C-ABI against
the oracle (every giant bit for bit, labels, the .cand lines): channel
counts that are not powers of two, ragged lengths, 1-3 beams per
filterbank (STF), boxcar_max 1-1024, cleaning on and off, channel zaps,
thresholds, and configurations whose search is skipped (max_delay +
boxcar_max beyond a beam)."""
import dataclasses
import os
import sys

import numpy as np
import pytest

import oracle
from heimdall_multibeam_b200 import synth

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from test_gpu_parity import _compare  # noqa: E402

pytestmark = pytest.mark.gpu


@dataclasses.dataclass
class Shape:
    nchans: int
    dt: float
    f0: float
    df: float
    dm_min: float
    dm_max: float
    boxcar_max: int


def _config(seed):
    rng = np.random.default_rng(5000 + seed)
    nchans = int(rng.choice([32, 48, 100, 128, 200, 256, 320]))
    dt = float(rng.choice([64e-6, 128e-6, 327.68e-6]))
    f0 = float(rng.uniform(400.0, 1600.0))
    df = -float(rng.uniform(50.0, 300.0)) / nchans
    boxcar_max = int(2 ** rng.integers(0, 11))
    nbeams = int(rng.integers(1, 4))
    dm_max = float(rng.choice([30.0, 80.0, 200.0, 500.0]))
    table = oracle.delay_table(nchans, dt, f0, df)
    # keep the oracle's dedispersion work to a few seconds
    while True:
        dms = oracle.dm_list(0.0, dm_max, dt, 40.0, f0, df, nchans, 1.25)
        md = int(oracle.delays(dms[-1:], table).max())
        per_beam = md + boxcar_max + int(rng.integers(1500, 12000))
        if len(dms) * nchans * per_beam * nbeams < 2.5e9 or dm_max <= 30.0:
            break
        dm_max /= 2
    if seed % 5 == 4:
        per_beam = md + boxcar_max // 2 + 10  # search skipped: delay + boxcars exceed a beam
    shape = Shape(nchans, dt, f0, df, 0.0, dm_max, boxcar_max)
    clean = bool(rng.integers(0, 2))
    zaps = [(int(a), int(a) + int(rng.integers(1, 6)))
            for a in rng.integers(0, nchans - 6, int(rng.integers(0, 3)))]
    thresh = float(rng.choice([6.0, 6.0, 5.0, 7.5]))
    beams = []
    for b in range(nbeams):
        g = np.random.default_rng(seed * 10 + b)
        hi = max(per_beam - md - boxcar_max, boxcar_max + 2)
        pulses = [synth.Pulse(float(g.uniform(boxcar_max + 1, hi)), float(g.uniform(0, dm_max)),
                              float(g.uniform(0.5, 5.0)) * dt * 4, float(g.uniform(10, 40)))
                  for _ in range(2)]
        beams.append(synth.make_beam(per_beam, nchans, dt, f0, df, pulses, seed=seed, beam=b,
                                     n_bursts=int(clean) * 2).data)
    return shape, np.concatenate(beams), nbeams, clean, zaps, thresh


@pytest.mark.parametrize("seed", range(14))
def test_random_configuration(hdb, oracle_lib, seed):
    shape, fb, nbeams, clean, zaps, thresh = _config(seed)
    _compare(fb, nbeams, shape, clean, zaps=zaps, detect_thresh=thresh)
