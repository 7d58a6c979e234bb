"""S/N of the float chain against the same chain held in double (no GPU).

The product's S/N values are bit-identical to the float chain of the oracle
(the GPU parity tests), which restates the reference's float arithmetic
(Pipeline/remove_baseline.cu, get_rms.cu, matched_filter.cu).  This states
how far that float chain lies from the same chain with every value in double
(oracle/snr64.c), giant by giant.  The error grows with the boxcar width: the
float baseline is subtracted from raw dedispersed sums near 2^15 (256
channels of 8-bit samples), so its rounding (about 2e-3 there) is smooth in
time and adds up coherently over a wide boxcar; the prefix sum itself
contributes well under 1e-6.  Measured maxima: 1.5e-4 over every giant of the
256-channel gulp (2.1e-5 over its candidates); 5.7e-4 over the giants of
unscrunched widths and 3.4e-3 over the time-scrunched width of the
1024-channel gulp.
"""
import numpy as np
import pytest

import oracle
from heimdall_multibeam_b200 import synth

# bounds of the relative S/N error |snr32 - snr64| / snr64 that the tests hold
# (the measured values are about half of these)
CAND_MAX = 1e-4     # merged candidates (the reported rows)
GIANT_MAX = 3e-4    # every giant before merging, widest boxcars included
GIANT_MEDIAN = 3e-5


def _kw(w, **extra):
    d = dict(dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min, dm_max=w.dm_max,
             boxcar_max=w.boxcar_max)
    d.update(extra)
    return d


def _rel_errors(fb, nbeams, kw, key):
    r = oracle.execute(fb, nbeams=nbeams, **kw)
    assert r["error"] == 0
    g = r[key]
    s64 = oracle.giant_snr_fp64(fb, g["dm_inds"], g["filter_inds"], g["inds"], nbeams=nbeams,
                                **kw)
    s32 = g["peaks"].astype(np.float64)
    return np.abs(s32 - s64) / np.abs(s64), g


@pytest.mark.parametrize("clean", [0, 1])
def test_snr_against_fp64_single_beam(oracle_lib, clean):
    w = synth.SEARCH_C0
    fb = synth.make_c0().data
    kw = _kw(w, clean=clean)
    rel_g, g = _rel_errors(fb, 1, kw, "giants")
    assert len(rel_g) >= 50
    assert len(set(g["filter_inds"].tolist())) == 11  # every boxcar width 2^0..2^10
    assert rel_g.max() < GIANT_MAX, rel_g.max()
    assert np.median(rel_g) < GIANT_MEDIAN
    rel_c, _ = _rel_errors(fb, 1, kw, "groups")
    assert len(rel_c) >= 3
    assert rel_c.max() < CAND_MAX, rel_c.max()


def test_snr_against_fp64_multibeam(oracle_lib):
    """Four beams concatenated in time: per-beam baseline and RMS."""
    w = synth.Workload("mb_small", 64, 655.36e-6, 851.0, -0.390625, 8192, 4, 0.0, 600.0, 256,
                       False, "")
    beams = synth.make_multibeam(w, seed=7, snr_lo=15, snr_hi=30)
    fb = synth.stf(beams)
    kw = _kw(w, clean=1, baseline_length=1.0)
    rel_g, _ = _rel_errors(fb, w.nbeams, kw, "giants")
    assert len(rel_g) >= 10
    assert rel_g.max() < GIANT_MAX, rel_g.max()
    rel_c, _ = _rel_errors(fb, w.nbeams, kw, "groups")
    assert rel_c.max() < CAND_MAX, rel_c.max()


def test_snr_against_fp64_survey_channels(oracle_lib):
    """1024 channels with RFI and cleaning (the survey beam's shape, 2^16
    spectra): raw sums near 2^17, boxcars to 4096.  The widest boxcar is the
    one time-scrunched width (min_tscrunch_width 4096); its block RMS window
    also holds the values the previous width left behind, and its error is
    about ten times the others'."""
    w = synth.SEARCH_C1
    fb = synth.make_c1(nsamps=1 << 16).data
    kw = _kw(w, clean=1)
    rel_g, g = _rel_errors(fb, 1, kw, "giants")
    assert len(rel_g) >= 1000
    scr = g["filter_inds"] == 12
    assert scr.sum() >= 100 and (~scr).sum() >= 1000
    assert rel_g[~scr].max() < 2e-3, rel_g[~scr].max()
    assert rel_g[scr].max() < 2e-2, rel_g[scr].max()
    assert np.median(rel_g) < 2e-4
    rel_c, _ = _rel_errors(fb, 1, kw, "groups")
    assert len(rel_c) >= 5
    assert rel_c.max() < 2e-2, rel_c.max()


def test_fp64_chain_places_every_giant(oracle_lib):
    """A giant index that the chain cannot hold is an error, not a value."""
    w = synth.SEARCH_C0
    fb = synth.make_c0().data
    with pytest.raises(RuntimeError):
        oracle.giant_snr_fp64(fb, [5], [3], [10 ** 9], **_kw(w))
