"""The product's S/N against the same search chain held in double precision.

hd_get_giants gives every giant of the gulp (S/N, sample index, filter and DM
trial); the oracle's double-precision chain (oracle/snr64.c) evaluates the S/N
of the same giants with every value in double.  The product's values equal
the float chain of the reference bit for bit; this states how far that float
arithmetic lies from double precision on the product's own output.  The bounds
match tests/test_oracle_fp64.py.
"""
import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("clean", [False, True])
def test_product_snr_against_fp64(hdb, oracle_lib, clean):
    w = synth.SEARCH_C0
    fb = synth.make_c0().data
    kw = dict(dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min, dm_max=w.dm_max,
              boxcar_max=w.boxcar_max)
    with H.Pipeline(H.default_params(nchans=w.nchans, output_dir=None, **kw),
                    cleaning=clean) as pl:
        err, _ = pl.execute(fb)
        assert err == H.HD_NO_ERROR
        g = pl.giants()
        cands = pl.candidates()
    assert len(g["peaks"]) >= 50 and len(cands) >= 3
    s64 = oracle.giant_snr_fp64(fb, g["dm_inds"], g["filter_inds"], g["inds"],
                                clean=int(clean), **kw)
    rel = np.abs(g["peaks"].astype(np.float64) - s64) / np.abs(s64)
    assert rel.max() < 3e-4, rel.max()
    assert np.median(rel) < 3e-5
    # the reported rows: single beam, so a row's giant index is its sample index
    c64 = oracle.giant_snr_fp64(fb, cands["dm_trial"], cands["filter"], cands["samp_idx"],
                                clean=int(clean), **kw)
    crel = np.abs(cands["snr"].astype(np.float64) - c64) / np.abs(c64)
    assert crel.max() < 1e-4, crel.max()
