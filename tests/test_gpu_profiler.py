"""The candidate profiler on the GPU (hd_profile_candidates) against the
oracle's restatement of Applications/candidate_profiler.C (which
tests/test_oracle_profiler.py pins to the reference application itself):
DM-time plot, DM-0 series, freq-time plot, the first maximum, SNR vs DM and
SNR vs time, for a batch of candidates (several widths, DMs and window
sizes, windows at the filterbank's edges), in both filtering modes, from
host and from device memory.  Finite values are bit-exact; NaN and inf
(rows without deviation, as the reference divides by zero) sit at the same
places."""
import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu


def _same(a, b, what):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    assert a.shape == b.shape, what
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b), err_msg=what)
    m = ~np.isnan(a)
    np.testing.assert_array_equal(a[m].view(np.uint32), b[m].view(np.uint32), err_msg=what)


def _requests(b, dms, nsamps):
    reqs = []
    for k, p in enumerate(b.pulses):
        dm_idx = int(np.argmin(np.abs(dms - p.dm)))
        reqs.append((int(p.t0), (2, 4, 7)[k % 3], dm_idx))
    reqs.append((40, 0, 3))                       # window clipped at the start
    reqs.append((nsamps - 30, 5, len(dms) - 2))   # runs past the end, last trials
    return reqs


@pytest.mark.parametrize("do_filter", [False, True])
@pytest.mark.parametrize("on_device", [False, True])
def test_profiler_equals_oracle(hdb, oracle_lib, do_filter, on_device):
    w = synth.SEARCH_C0
    b = synth.make_c0()
    fb = b.data
    dms = oracle.dm_list(0.0, 1000.0, w.dt, 40.0, w.f0, w.df, w.nchans, 1.25)
    reqs = _requests(b, dms, fb.shape[0])
    out_n, out_d, fs = 64, 24, 16
    if on_device:
        import torch
        d = torch.from_numpy(fb).cuda()
        torch.cuda.synchronize()
        got = H.profile_candidates(d.data_ptr(), w.dt, w.f0, w.df, dms, reqs, out_n, out_d, fs,
                                   do_filter, nsamps=fb.shape[0], nchans=fb.shape[1],
                                   on_device=True)
    else:
        got = H.profile_candidates(fb, w.dt, w.f0, w.df, dms, reqs, out_n, out_d, fs, do_filter)
    for (samp, filt, dm_idx), g in zip(reqs, got):
        r = oracle.profile(fb, w.dt, w.f0, w.df, dms, samp, filt, dm_idx, out_n, out_d, fs,
                           do_filter)
        what = f"samp {samp} filter {filt} trial {dm_idx}"
        assert g["n_dm"] == r["n_dm"] and g["max_idx"] == r["max_idx"], what
        assert g["snr_dm_first"] == r["snr_dm_first"], what
        for k in ("dm_time", "dm0_time", "freq_time", "snr_dm", "snr_time"):
            _same(g[k], r[k], f"{k} {what}")


def test_profiler_wide_window_and_survey_band(hdb, oracle_lib):
    """1024 channels, a 128-sample plot of 64 trials with fscrunch 32, a
    long boxcar (2^9) and a freq-time window wider than the plot's span."""
    w = synth.SEARCH_C1
    b = synth.make_c1(nsamps=1 << 16, npulses=4)
    fb = b.data
    dms = oracle.dm_list(0.0, 600.0, w.dt, 40.0, w.f0, w.df, w.nchans, 1.25)
    p = b.pulses[0]
    reqs = [(int(p.t0), 9, int(np.argmin(np.abs(dms - min(p.dm, 590.0)))))]
    got = H.profile_candidates(fb, w.dt, w.f0, w.df, dms, reqs, 128, 64, 32, False)
    r = oracle.profile(fb, w.dt, w.f0, w.df, dms, *reqs[0], 128, 64, 32, False)
    for k in ("dm_time", "dm0_time", "freq_time", "snr_dm", "snr_time"):
        _same(got[0][k], r[k], k)
    assert got[0]["max_idx"] == r["max_idx"]
