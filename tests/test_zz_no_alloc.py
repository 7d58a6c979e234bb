"""The allocation-free cleaning entry point (hd_clean_filterbank_rfi_noalloc).

It exists for callers that cannot allocate device memory while they run (a
real-time loop in which an allocation would synchronise the device, or a fixed
device-memory budget).  These tests drive it through the C interface on
caller-owned device buffers and check every result against the allocating
entry point hd_clean_filterbank_rfi: the cleaned bytes and the RFI mask are
integer data and must match exactly.  Cases: two calls in a row; a large call
followed by smaller ones (what a call leaves in the shared scratch array must
not reach the next); 4 and 64 beams per filterbank on a caller's stream; the
largest accepted gulp; and the requests the fixed array cannot serve.  The
file is collected after the other tests and passes both on its own in a fresh
process and after the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

import heimdall_multibeam_b200 as H
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu
DT = synth.SEARCH_C1.dt


def _filterbank(seed, nsamps=1 << 15, nchans=64, n_bursts=6):
    w = synth.SEARCH_C1
    return synth.make_beam(nsamps, nchans, w.dt, w.f0, w.df * (w.nchans // nchans),
                           [synth.Pulse(nsamps / 8.0, 0.0, 0.5e-3, 40.0)], seed=seed,
                           n_bursts=n_bursts, rfi_chan_frac=0.05).data


def _allocating(fb, nbeams=1, boxcar_max=64):
    with H.Pipeline(H.default_params(nchans=fb.shape[1], output_dir=None)) as pl:
        return pl.clean_filterbank_rfi(fb, DT, boxcar_max=boxcar_max, nbeams=nbeams)


def _noalloc(torch, fbs, nbeams=1, stream=None, boxcar_max=64):
    """Calls in a row on caller-owned device buffers; returns (out, mask,
    status) per call after the stream has finished."""
    dev = torch.device("cuda", 0)
    d_in = [torch.from_numpy(fb).to(dev) for fb in fbs]
    d_out = [torch.full_like(t, 7) for t in d_in]
    d_mask = [torch.full((fb.shape[0],), -1, dtype=torch.int32, device=dev) for fb in fbs]
    d_status = torch.full((len(fbs),), 0xABCD, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    s = None if stream is None else C.c_void_p(stream.cuda_stream)
    for i, fb in enumerate(fbs):
        nsamps, nchans = fb.shape
        err = H.lib().hd_clean_filterbank_rfi_noalloc(
            d_in[i].data_ptr(), nsamps, nchans, 8, d_out[i].data_ptr(), d_mask[i].data_ptr(),
            DT, 2.0, 5.0, boxcar_max, nbeams, s, d_status.data_ptr() + 4 * i)
        assert err == H.HD_NO_ERROR, H.error_string(err)
    if stream is not None:
        stream.synchronize()
    torch.cuda.synchronize()
    st = d_status.cpu().numpy()
    return [(d_out[i].cpu().numpy(), d_mask[i].cpu().numpy(), int(st[i]))
            for i in range(len(fbs))]


def _check(got, fbs, nbeams=1):
    for i, (fb, (out, mask, status)) in enumerate(zip(fbs, got)):
        ref_out, ref_mask = _allocating(fb, nbeams)
        assert status == 0, f"call {i}"
        np.testing.assert_array_equal(mask, ref_mask, err_msg=f"call {i}")
        np.testing.assert_array_equal(out, ref_out, err_msg=f"call {i}")


def test_noalloc_matches_allocating_entry_point(hdb):
    import torch
    fbs = [_filterbank(3), _filterbank(4)]
    got = _noalloc(torch, fbs)
    assert all(m.sum() > 0 for _, m, _ in got)
    _check(got, fbs)


def test_noalloc_large_then_small_calls(hdb):
    """A long gulp, two short ones and the long one again: each result equals
    the allocating call's, whatever the previous call left in the array."""
    import torch
    fbs = [_filterbank(10, 1 << 18, n_bursts=20), _filterbank(11, 1 << 14),
           _filterbank(12, 5000), _filterbank(10, 1 << 18, n_bursts=20)]
    _check(_noalloc(torch, fbs), fbs)


@pytest.mark.parametrize("nbeams,nsamps", [(4, 1 << 16), (64, 1 << 17)])
def test_noalloc_multibeam_on_caller_stream(hdb, nbeams, nsamps):
    """Filterbanks of 4 and 64 time-concatenated beams (per-beam baselines and
    RMS), queued on a caller-created, non-default stream."""
    import torch
    fbs = [_filterbank(20 + nbeams, nsamps, n_bursts=12)]
    stream = torch.cuda.Stream()
    _check(_noalloc(torch, fbs, nbeams=nbeams, stream=stream), fbs, nbeams=nbeams)


def test_noalloc_largest_accepted_gulp(hdb):
    import torch
    fbs = [_filterbank(30, H.HD_NOALLOC_MAX_NSAMPS, nchans=32, n_bursts=30)]
    _check(_noalloc(torch, fbs), fbs)


def test_noalloc_rejects_requests_beyond_the_array(hdb):
    """Beyond the fixed scratch size the call returns an error before touching
    any buffer (the pointers here are never dereferenced)."""
    L = H.lib()
    bogus = C.c_void_p(16)
    for nsamps, nbeams, bmax in [(H.HD_NOALLOC_MAX_NSAMPS + 1, 1, 64),
                                 (1 << 16, H.HD_NOALLOC_MAX_BEAMS + 1, 64),
                                 (1 << 16, 1, 256)]:
        err = L.hd_clean_filterbank_rfi_noalloc(bogus, nsamps, 64, 8, bogus, bogus, DT, 2.0,
                                                5.0, bmax, nbeams, None, None)
        assert err == H.HD_INVALID_STRIDE, (nsamps, nbeams, bmax)
