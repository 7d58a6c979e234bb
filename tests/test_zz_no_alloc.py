"""The allocation-free cleaning entry point (hd_clean_filterbank_rfi_noalloc).

It exists for callers that cannot allocate device memory while they run (a
real-time loop in which an allocation would synchronise the device, or a fixed
device-memory budget).  This test drives it through the C interface on
caller-owned device buffers, twice in a row on different filterbanks, and
checks both results against the allocating entry point hd_clean_filterbank_rfi:
the cleaned bytes and the RFI mask are integer data and must match exactly.
It lives in its own file, collected after the other tests, and passes both on
its own in a fresh process and after the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

import heimdall_multibeam_b200 as H
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu


def _filterbank(seed):
    w = synth.SEARCH_C1
    return synth.make_beam(1 << 15, 64, w.dt, w.f0, w.df * 16,
                           [synth.Pulse(4000.0, 0.0, 0.5e-3, 40.0)], seed=seed, n_bursts=6,
                           rfi_chan_frac=0.05).data


def test_noalloc_matches_allocating_entry_point(hdb):
    import torch
    L = H.lib()
    dt = synth.SEARCH_C1.dt
    fbs = [_filterbank(3), _filterbank(4)]
    nsamps, nchans = fbs[0].shape

    # reference results from the allocating entry point (host buffers)
    expected = []
    with H.Pipeline(H.default_params(nchans=nchans, output_dir=None)) as pl:
        for fb in fbs:
            expected.append(pl.clean_filterbank_rfi(fb, dt))
    assert all(m.sum() > 0 for _, m in expected)

    # two allocation-free calls in a row on caller-owned device buffers
    dev = torch.device("cuda", 0)
    d_in = [torch.from_numpy(fb).to(dev) for fb in fbs]
    d_out = [torch.zeros_like(t) for t in d_in]
    d_mask = [torch.full((nsamps,), -1, dtype=torch.int32, device=dev) for _ in fbs]
    torch.cuda.synchronize()
    for i in range(2):
        err = L.hd_clean_filterbank_rfi_noalloc(
            d_in[i].data_ptr(), nsamps, nchans, 8, d_out[i].data_ptr(), d_mask[i].data_ptr(),
            dt, 2.0, 5.0, 64, 1, None)
        assert err == H.HD_NO_ERROR, H.error_string(err)
    torch.cuda.synchronize()
    for i, (ref_out, ref_mask) in enumerate(expected):
        np.testing.assert_array_equal(d_mask[i].cpu().numpy(), ref_mask, err_msg=f"call {i}")
        np.testing.assert_array_equal(d_out[i].cpu().numpy(), ref_out, err_msg=f"call {i}")


def test_noalloc_rejects_oversized_requests(hdb):
    """Beyond the fixed scratch size the call returns an error before touching
    any buffer (the pointers here are never dereferenced)."""
    L = H.lib()
    bogus = C.c_void_p(16)
    err = L.hd_clean_filterbank_rfi_noalloc(bogus, H.HD_NOALLOC_MAX_NSAMPS + 1, 64, 8, bogus,
                                            bogus, 64e-6, 2.0, 5.0, 64, 1, None)
    assert err == H.HD_INVALID_STRIDE
