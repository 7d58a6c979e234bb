"""Adaptive time resolution (use_scrunching, dedisp_enable_adaptive_dt) on
the GPU against the oracle.

Each trial has a scrunch factor s (the restated rule of include/dedisp.h)
and is dedispersed at sampling time s dt from the byte-mean scrunched input;
the search then runs at that resolution (pipeline.cu:489-775: scrunched
series, strides and delays, boxcars from width s, indices rescaled by s x
tscrunch).  The oracle's scrunched chain equals the reference pipeline's own
scrunched path (tests/test_oracle.py); here the product equals the oracle:
scrunch factors, dedispersed sums, giants, labels and .cand lines, for one
beam, a 4-beam STF gulp, and a batch of independent filterbanks."""
import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu


def _kw(w, **extra):
    d = dict(dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min, dm_max=w.dm_max,
             boxcar_max=w.boxcar_max)
    d.update(extra)
    return d


def test_scrunch_factors_and_dedispersion(hdb, oracle_lib):
    w = synth.SEARCH_C0
    fb = synth.make_c0().data
    plan = H.DedispPlan(w.nchans, w.dt, w.f0, w.df)
    plan.generate_dm_list(w.dm_min, w.dm_max, 40.0, 1.25)
    plan.enable_adaptive_dt(40.0, 1.15)
    dms = plan.dm_list
    want_f = oracle.scrunch_factors(dms, w.dt, 40.0, w.f0, w.df, w.nchans, 1.15)
    np.testing.assert_array_equal(plan.dt_factors, want_f)
    assert int(want_f.max()) >= 32
    got = plan.execute(fb)
    table = oracle.delay_table(w.nchans, w.dt, w.f0, w.df)
    want = oracle.dedisperse_scrunched(fb, dms, table, want_f)
    for d in range(len(dms)):
        np.testing.assert_array_equal(got[d, :len(want[d])], want[d], err_msg=f"trial {d}")
    # the factors follow a new DM list; disabling gives the native resolution
    plan.set_dm_list(dms[::2])
    np.testing.assert_array_equal(
        plan.dt_factors, oracle.scrunch_factors(dms[::2], w.dt, 40.0, w.f0, w.df, w.nchans, 1.15))
    plan.disable_adaptive_dt()
    assert set(plan.dt_factors.tolist()) == {1}


def _compare(fb, nbeams, w, clean, **extra):
    kw = _kw(w, **extra)
    r = oracle.execute(fb, nbeams=nbeams, clean=int(clean), use_scrunching=1, **kw)
    assert int(r["scrunch"].max()) >= 2
    p = H.default_params(nchans=w.nchans, output_dir=None, use_scrunching=True, **kw)
    with H.Pipeline(p, cleaning=clean) as pl:
        err, proc = pl.execute(fb, nbeams=nbeams, raise_on_error=False)
        cands, g = pl.candidates(), pl.giants()
    assert err == r["error"] and proc == r["nsamps_processed"]
    og = r["giants"]
    assert len(g["peaks"]) == len(og["peaks"]) > 0
    for k in ("inds", "begins", "ends", "filter_inds", "dm_inds"):
        np.testing.assert_array_equal(g[k], og[k], err_msg=k)
    np.testing.assert_array_equal(g["peaks"].view(np.uint32), og["peaks"].view(np.uint32))
    np.testing.assert_array_equal(g["labels"], r["labels"])
    want = oracle.cand_lines(r["groups"], fb.shape[0], nbeams, 0, r["nsamps_processed"],
                             w.boxcar_max, w.dt)
    assert H.cand_lines(cands) == want
    assert len(want) >= 1


@pytest.mark.parametrize("clean", [False, True])
def test_adaptive_dt_single_beam(hdb, oracle_lib, clean):
    _compare(synth.make_c0().data, 1, synth.SEARCH_C0, clean)


def test_adaptive_dt_headline_beam_and_stf(hdb, oracle_lib):
    w = synth.SEARCH_C2
    _compare(synth.make_multibeam(w, seed=2026)[3].data, 1, w, False)
    ws = synth.Workload("mb_small", 64, 655.36e-6, 851.0, -0.390625, 8192, 4, 0.0, 600.0, 256,
                        False, "")
    fb = synth.stf(synth.make_multibeam(ws, seed=7, snr_lo=15, snr_hi=30))
    _compare(fb, 4, ws, True, baseline_length=1.0)


def test_adaptive_dt_batched_equals_separate(hdb, oracle_lib):
    """Several filterbanks in one batched call with adaptive dt (series laid
    out by scrunch factor, giants gathered back filterbank by filterbank)
    equal separate calls and the oracle."""
    w = synth.SEARCH_C0
    beams = [synth.make_beam(1 << 15, 128, w.dt, w.f0, w.df * 2,
                             [synth.Pulse(4000.0 + 3000.0 * u, 150.0 + 200.0 * u, 1e-3, 25.0),
                              synth.Pulse(12000.0, 600.0, 4e-3, 30.0)], seed=60 + u, beam=u).data
             for u in range(3)]
    kw = _kw(w, df=w.df * 2, dm_max=800.0, boxcar_max=512)
    p = H.default_params(nchans=128, output_dir=None, use_scrunching=True, **kw)
    with H.Pipeline(p, cleaning=True) as pl:
        err, proc, st = pl.execute_beams(beams)
        got = [H.cand_lines(pl.candidates(u)) for u in range(3)]
    total = 0
    for u, fb in enumerate(beams):
        r = oracle.execute(fb, clean=1, use_scrunching=1, **kw)
        assert st[u] == r["error"]
        want = oracle.cand_lines(r["groups"], fb.shape[0], 1, 0, r["nsamps_processed"], 512,
                                 w.dt, beam=u)
        assert got[u] == want, u
        total += len(want)
    assert total >= 3
