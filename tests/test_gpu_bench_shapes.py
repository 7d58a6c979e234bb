"""Parity at the shapes the benchmark measures.

* The headline multibeam gulp exactly as `bench.py` draws it (36 beams x 320
  channels x 2^15 samples at 655.36 us, 851 MHz top, DM 0-2000 = 234 trials,
  boxcars to 512, seed 2026), through the batched call: every beam's giants
  (peak bits, index, begin, end, width, DM trial), cluster labels and .cand
  lines equal the oracle's run of that beam, from host input and from device
  input in both of the benchmark's forms (host-sized, and the CUDA graph
  replay of a shape seen before).
* Beams shaped like the uneven-beam workload, where the dedispersion runs
  long staged rows and many drains: a 4096-channel beam of 2^16 samples, a
  2048-channel beam at DM 4800-5000 (delays near 59 000 samples) and a
  512-channel beam at DM 0-5000 over 2^17 samples, with RFI and cleaning, in
  one beam-set call.  Dedispersed sums and candidate lines equal the
  oracle's.  DM windows keep the oracle's CPU time to seconds.
"""
import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu
SNR_RTOL = 1e-4


def _okw(w, **extra):
    d = dict(dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min, dm_max=w.dm_max,
             boxcar_max=w.boxcar_max)
    d.update(extra)
    return d


def test_headline_gulp_every_beam_equals_oracle(hdb, oracle_lib):
    w = synth.SEARCH_C2
    beams = synth.make_multibeam(w, seed=2026)
    assert len(beams) == 36
    p = H.default_params(nchans=w.nchans, output_dir=None, **_okw(w))
    torch = pytest.importorskip("torch")
    with H.Pipeline(p, cleaning=w.clean) as pl:
        err, proc, st = pl.execute_beams([b.data for b in beams])
        assert err == H.HD_NO_ERROR
        g = pl.giants()
        cands = [pl.candidates(u) for u in range(len(beams))]
        # the benchmark's own call: the 36 filterbanks resident on the device,
        # the first gulp host-sized, the second a CUDA graph replay; both
        # equal the host-input call (which the oracle checks below)
        d = torch.from_numpy(np.stack([b.data for b in beams])).cuda()
        fb_bytes = w.nsamps * w.nchans
        ptrs = [d.data_ptr() + u * fb_bytes for u in range(len(beams))]
        for _ in range(2):
            err_d, proc_d, st_d = pl.execute_beams(ptrs, nsamps=w.nsamps, on_device=True)
            assert (err_d, proc_d, st_d) == (err, proc, st)
            g_d = pl.giants()
            for k in g:
                np.testing.assert_array_equal(g_d[k].view(np.uint8), g[k].view(np.uint8),
                                              err_msg=k)
            for u in range(len(beams)):
                assert H.cand_lines(pl.candidates(u)) == H.cand_lines(cands[u]), u
                np.testing.assert_array_equal(pl.candidates(u)["snr"].view(np.uint32),
                                              cands[u]["snr"].view(np.uint32))
        assert pl.graph_replays() == 1
    off = 0
    total = 0
    for u, b in enumerate(beams):
        r = oracle.execute(b.data, clean=int(w.clean), **_okw(w))
        assert r["dm_count"] == 234
        assert st[u] == r["error"] == H.HD_NO_ERROR
        assert proc == r["nsamps_processed"]
        og = r["giants"]
        n = len(og["peaks"])
        for k in ("inds", "begins", "ends", "filter_inds", "dm_inds"):
            np.testing.assert_array_equal(g[k][off:off + n], og[k], err_msg=f"{k} beam {u}")
        np.testing.assert_allclose(g["peaks"][off:off + n], og["peaks"], rtol=SNR_RTOL)
        np.testing.assert_array_equal(g["peaks"][off:off + n].view(np.uint32),
                                      og["peaks"].view(np.uint32))
        np.testing.assert_array_equal(g["labels"][off:off + n], r["labels"] + off)
        want = oracle.cand_lines(r["groups"], w.nsamps, 1, 0, r["nsamps_processed"],
                                 w.boxcar_max, w.dt, beam=u)
        assert H.cand_lines(cands[u]) == want, u
        off += n
        total += len(want)
    assert off == len(g["peaks"])
    assert total >= 36


UNEVEN = [
    # channels, dt, samples, DM window
    (4096, 64e-6, 1 << 16, 400.0, 500.0),
    (2048, 128e-6, 1 << 17, 4800.0, 5000.0),
    (512, 64e-6, 1 << 17, 0.0, 5000.0),
]


def _uneven():
    ws = [synth.Workload(f"uneven_c{c}_n{n}", c, dt, synth.UNEVEN_F_TOP, -synth.UNEVEN_BW / c,
                         n, 1, lo, hi, synth.UNEVEN_BOXCAR_MAX, True, "")
          for c, dt, n, lo, hi in UNEVEN]
    beams = [synth.make_uneven_beam(w, seed=77, beam=w.nchans) for w in ws]
    return ws, beams


def test_uneven_shapes_dedispersion_equals_oracle(hdb, oracle_lib):
    ws, beams = _uneven()
    for w, b in zip(ws, beams):
        plan = H.DedispPlan(w.nchans, w.dt, w.f0, w.df)
        plan.generate_dm_list(w.dm_min, w.dm_max, 40.0, 1.25)
        table = oracle.delay_table(w.nchans, w.dt, w.f0, w.df)
        np.testing.assert_array_equal(
            plan.dm_list, oracle.dm_list(w.dm_min, w.dm_max, w.dt, 40.0, w.f0, w.df, w.nchans,
                                         1.25))
        got = plan.execute(b.data)
        want = oracle.dedisperse(b.data, plan.dm_list, table)
        assert got.shape == want.shape and got.shape[1] > 0
        np.testing.assert_array_equal(got, want, err_msg=w.name)


def test_uneven_shapes_beam_set_equals_oracle(hdb, oracle_lib):
    ws, beams = _uneven()
    params = []
    for b, w in enumerate(ws):
        p = H.default_params(nchans=w.nchans, output_dir=None, **_okw(w))
        p.beam = b
        params.append(p)
    with H.BeamSet(params, workers=3, cleaning=True) as bs:
        err, st, proc = bs.execute([b.data for b in beams])
        lines = [H.cand_lines(bs.candidates(b)) for b in range(len(ws))]
    total = 0
    for b, (w, beam) in enumerate(zip(ws, beams)):
        r = oracle.execute(beam.data, clean=1, **_okw(w))
        assert st[b] == r["error"] == H.HD_NO_ERROR, (b, st[b], r["error"])
        assert proc[b] == r["nsamps_processed"]
        want = oracle.cand_lines(r["groups"], w.nsamps, 1, 0, r["nsamps_processed"],
                                 w.boxcar_max, w.dt, beam=b)
        assert lines[b] == want, w.name
        total += len(want)
    assert total >= 10
