"""The narrow-band RFI restatement (oracle/oracle.c: or_measure_bandpass,
or_narrow_band) against the reference's own code for it (no GPU):
Pipeline/measure_bandpass.cu from the reference build, and
zap_narrow_rfi_functor compiled from Pipeline/clean_filterbank_rfi.cu
(oracle/ref/narrow_driver.cpp), bit for bit."""
import numpy as np
import pytest

import oracle
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.skipif(not oracle.ref_available(),
                                reason="the reference build (make -C oracle ref) is missing")


def narrowband_beam(nsamps, nchans, seed, dt=64e-6):
    """Noise with a sloped bandpass, persistent narrowband channels and
    short narrowband bursts."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((nsamps, nchans)).astype(np.float32) * 12.0
    x += (100.0 + 40.0 * np.sin(np.linspace(0, 3, nchans)))[None, :].astype(np.float32)
    bad = rng.choice(nchans, size=max(1, nchans // 25), replace=False)
    x[:, bad] += 90.0
    for _ in range(20):
        c0 = int(rng.integers(0, nchans - 4))
        t0 = int(rng.integers(0, nsamps - 200))
        x[t0:t0 + int(rng.integers(5, 200)), c0:c0 + int(rng.integers(1, 4))] += 120.0
    np.rint(x, out=x)
    np.clip(x, 0, 255, out=x)
    return x.astype(np.uint8)


@pytest.mark.parametrize("nsamps,nchans", [(4000, 64), (20000, 256), (7777, 120)])
def test_measure_bandpass_matches_reference(oracle_lib, nsamps, nchans):
    fb = narrowband_beam(nsamps, nchans, nchans)
    bp, rms = oracle.measure_bandpass(fb)
    rbp, rrms = oracle.measure_bandpass(fb, ref=True)
    np.testing.assert_array_equal(bp, rbp)
    assert rms == rrms and rms > 0


@pytest.mark.parametrize("nsamps,nchans,dt", [(40000, 64, 64e-6), (70000, 256, 64e-6),
                                              (9000, 120, 655.36e-6)])
def test_narrow_band_matches_reference(oracle_lib, nsamps, nchans, dt):
    """Several bandpass stretches of baseline_length / dt spectra each (the
    last one short), zapped in index order."""
    fb = narrowband_beam(nsamps, nchans, nchans + 1, dt)
    mine = oracle.narrow_band(fb, dt)
    ref = oracle.narrow_band(fb, dt, ref=True)
    np.testing.assert_array_equal(mine, ref)
    changed = (mine != fb).mean()
    assert 0.0 < changed < 0.2
