"""Packed and 16-bit input on the GPU (nbits = 1, 2, 4, 16).

* dedisp_execute on packed samples equals the oracle's dedispersion of the
  same values as bytes (1, 2, 4 bits), and for 16-bit samples spanning the
  whole range, a numpy brute force of the reference's definition: the
  integer sum of the delayed samples, converted once to float.
* hd_execute on packed samples writes the same candidates as the oracle's
  run of the same values as bytes (the search only sees sample values).
* Requests the search does not serve are refused: cleaning, which the
  reference runs on bytes here, with packed input; 16-bit input with
  adaptive dt; a channel count whose packed spectrum is not whole words.
"""
import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu


def _beam(nbits, nsamps=1 << 14, nchans=64, seed=0):
    w = synth.SEARCH_C0
    b = synth.make_beam(nsamps, nchans, w.dt, w.f0, w.df * 4,
                        [synth.Pulse(3000.0, 150.0, 1e-3, 40.0),
                         synth.Pulse(9000.0, 60.0, 2e-3, 30.0)], seed=seed + nbits)
    kw = dict(dt=w.dt, f0=w.f0, df=w.df * 4, dm_min=0.0, dm_max=300.0, boxcar_max=256)
    return b.data, kw


def _numpy_dedisperse(v, dms, table):
    """out[d][t] = float(sum_c v[t + delay(d, c)][c]) in int64."""
    nsamps, nchans = v.shape
    delays = oracle.delays(dms, table).astype(np.int64).reshape(len(dms), nchans)
    md = int(delays.max())
    nout = nsamps - md
    out = np.zeros((len(dms), nout), np.int64)
    vi = v.astype(np.int64)
    for d in range(len(dms)):
        for c in range(nchans):
            out[d] += vi[delays[d, c]:delays[d, c] + nout, c]
    return out.astype(np.float32)


@pytest.mark.parametrize("nbits", [1, 2, 4])
def test_dedisp_packed_equals_oracle(hdb, oracle_lib, nbits):
    data, kw = _beam(nbits)
    v = (data >> (8 - nbits)).astype(np.uint8)
    plan = H.DedispPlan(v.shape[1], kw["dt"], kw["f0"], kw["df"])
    plan.generate_dm_list(0.0, 300.0, 40.0, 1.25)
    got = plan.execute(synth.pack_filterbank(v, nbits), nbits=nbits)
    table = oracle.delay_table(v.shape[1], kw["dt"], kw["f0"], kw["df"])
    np.testing.assert_array_equal(got, oracle.dedisperse(v, plan.dm_list, table))


def test_dedisp_16bit_full_range_equals_numpy(hdb, oracle_lib):
    rng = np.random.default_rng(16)
    nchans = 64
    v = rng.integers(0, 1 << 16, size=(6000, nchans)).astype(np.uint16)
    v[:50] = 65535  # the largest sums
    w = synth.SEARCH_C0
    plan = H.DedispPlan(nchans, w.dt, w.f0, w.df * 4)
    plan.generate_dm_list(0.0, 120.0, 40.0, 1.25)
    got = plan.execute(synth.pack_filterbank(v, 16), nbits=16)
    table = oracle.delay_table(nchans, w.dt, w.f0, w.df * 4)
    np.testing.assert_array_equal(got, _numpy_dedisperse(v, plan.dm_list, table))


@pytest.mark.parametrize("nbits", [1, 2, 4, 16])
def test_search_packed_equals_oracle(hdb, oracle_lib, nbits):
    data, kw = _beam(nbits)
    v = data if nbits == 16 else (data >> (8 - nbits))
    v8 = v.astype(np.uint8)
    r = oracle.execute(v8, clean=0, **kw)
    want = oracle.cand_lines(r["groups"], v8.shape[0], 1, 0, r["nsamps_processed"],
                             kw["boxcar_max"], kw["dt"])
    packed = synth.pack_filterbank(v.astype(np.uint16 if nbits == 16 else np.uint8), nbits)
    with H.Pipeline(H.default_params(nchans=v.shape[1], output_dir=None, **kw),
                    cleaning=False) as pl:
        err, proc = pl.execute(packed, nbits=nbits)
        assert err == H.HD_NO_ERROR and proc == r["nsamps_processed"]
        assert H.cand_lines(pl.candidates()) == want
    if nbits >= 4:
        assert len(want) >= 1


def test_unsupported_requests_refused(hdb):
    data, kw = _beam(2)
    packed = synth.pack_filterbank((data >> 6).astype(np.uint8), 2)
    with H.Pipeline(H.default_params(nchans=64, output_dir=None, **kw), cleaning=True) as pl:
        err, _ = pl.execute(packed, nbits=2, raise_on_error=False)
        assert err == H.HD_INVALID_NBITS
    with H.Pipeline(H.default_params(nchans=64, output_dir=None, **kw), cleaning=False) as pl:
        err, _ = pl.execute(packed, nbits=3, raise_on_error=False)
        assert err == H.HD_INVALID_NBITS
    # 1-bit samples of 48 channels: 6 bytes per spectrum, not whole words
    with H.Pipeline(H.default_params(nchans=48, output_dir=None, **kw), cleaning=False) as pl:
        err, _ = pl.execute(np.zeros((1 << 14, 6), np.uint8), nbits=1, raise_on_error=False)
        assert err == H.HD_INVALID_STRIDE
    p = H.default_params(nchans=64, output_dir=None, use_scrunching=True, **kw)
    with H.Pipeline(p, cleaning=False) as pl:
        err, _ = pl.execute(synth.pack_filterbank(data.astype(np.uint16), 16), nbits=16,
                            raise_on_error=False)
        assert err == H.HD_INVALID_NBITS
