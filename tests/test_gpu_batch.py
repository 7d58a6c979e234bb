"""Batched search of independent filterbanks (hd_execute_beams) against the
plain per-filterbank form (hd_execute) and the oracle.

The batched call must give, for every filterbank, exactly what a separate
hd_execute of that filterbank gives: the same candidate rows (bit-exact,
SNRs included), the same giants and labels, the same status and .cand file.
"""
import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu

# 8 beams x 128 channels, 2^14 samples each (a scaled-down multibeam gulp)
W = synth.Workload("mb8_c128_n16384", 128, 655.36e-6, 851.0, -0.3125, 1 << 14, 8, 0.0, 1000.0,
                   256, False, "")


def _kw(w, **extra):
    d = dict(nchans=w.nchans, dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min, dm_max=w.dm_max,
             boxcar_max=w.boxcar_max, output_dir=None)
    d.update(extra)
    return d


def _beams(seed=31, strong_beam=None):
    beams = [b.data for b in synth.make_multibeam(W, seed=seed, pulses_per_beam=3, snr_lo=10,
                                                  snr_hi=30)]
    # the same pulse at the same time and DM in beams 0 and 1: giants that
    # would cluster if the beams were not kept apart
    twin = [synth.Pulse(5000.0, 300.0, 5e-3, 25.0)]
    for u in (0, 1):
        beams[u] = synth.make_beam(W.nsamps, W.nchans, W.dt, W.f0, W.df, twin, seed=seed + 100,
                                   beam=u).data
    if strong_beam is not None:
        rng = np.random.default_rng(seed)
        many = [synth.Pulse(float(t), float(rng.uniform(50, 900)), 2e-3, 30.0)
                for t in np.linspace(600, W.nsamps - 1500, 40)]
        beams[strong_beam] = synth.make_beam(W.nsamps, W.nchans, W.dt, W.f0, W.df, many,
                                             seed=seed + 7, beam=strong_beam).data
    return beams


def _separate(beams, clean, nbeams=1, **kw):
    out = []
    for u, fb in enumerate(beams):
        p = H.default_params(beam=u * nbeams, **kw)
        with H.Pipeline(p, cleaning=clean) as pl:
            err, proc = pl.execute(fb, nbeams=nbeams, raise_on_error=False)
            out.append((err, proc, pl.candidates(), pl.giants()))
    return out


def _check(batch_pl, err, statuses, sep):
    assert err == (H.HD_TOO_MANY_EVENTS if any(s[0] == H.HD_TOO_MANY_EVENTS for s in sep)
                   else H.HD_NO_ERROR)
    g = batch_pl.giants()
    off = 0
    for u, (e_u, _, c_u, g_u) in enumerate(sep):
        assert statuses[u] == e_u, u
        got = batch_pl.candidates(u)
        if e_u == H.HD_TOO_MANY_EVENTS:
            assert len(got) == 0
            continue
        assert H.cand_lines(got) == H.cand_lines(c_u), u
        np.testing.assert_array_equal(got["snr"].view(np.uint32), c_u["snr"].view(np.uint32))
        n = len(g_u["peaks"])
        for k in ("inds", "begins", "ends", "filter_inds", "dm_inds"):
            np.testing.assert_array_equal(g[k][off:off + n], g_u[k], err_msg=f"{k} beam {u}")
        np.testing.assert_array_equal(g["peaks"][off:off + n].view(np.uint32),
                                      g_u["peaks"].view(np.uint32))
        np.testing.assert_array_equal(g["labels"][off:off + n], g_u["labels"] + off)
        off += n
    all_c = batch_pl.candidates()
    assert H.cand_lines(all_c) == sum((H.cand_lines(batch_pl.candidates(u))
                                       for u in range(len(sep))), [])


@pytest.mark.parametrize("clean", [False, True])
def test_batch_equals_separate(hdb, clean):
    beams = _beams()
    kw = _kw(W)
    sep = _separate(beams, clean, **kw)
    assert sum(len(c) for _, _, c, _ in sep) >= 10
    assert len(sep[0][2]) >= 1 and len(sep[1][2]) >= 1
    with H.Pipeline(H.default_params(**kw), cleaning=clean) as pl:
        err, proc, st = pl.execute_beams(beams)
        assert proc == sep[0][1]
        _check(pl, err, st, sep)
        # twin pulse: one candidate per beam, beam numbers 1 and 2
        assert pl.candidates(0)["beam"].tolist() == [1] * len(pl.candidates(0))
        assert pl.candidates(1)["beam"].tolist() == [2] * len(pl.candidates(1))


def test_batch_beam0_matches_oracle(hdb, oracle_lib):
    beams = _beams()
    kw = _kw(W)
    with H.Pipeline(H.default_params(**kw), cleaning=True) as pl:
        pl.execute_beams(beams[:3])
        for u in range(3):
            okw = {k: v for k, v in kw.items() if k not in ("nchans", "output_dir")}
            r = oracle.execute(beams[u], nbeams=1, clean=1, **okw)
            want = oracle.cand_lines(r["groups"], W.nsamps, 1, 0, r["nsamps_processed"],
                                     W.boxcar_max, W.dt, beam=u)
            assert H.cand_lines(pl.candidates(u)) == want


def test_batch_rate_bailout_per_beam(hdb):
    """Only the beam over the giant rate bails out; the others are unchanged."""
    beams = _beams(strong_beam=5)
    kw = _kw(W)
    counts = [len(g["peaks"]) for _, _, _, g in _separate(beams, False, **kw)]
    lo = sorted(counts)[-2]
    hi = counts[5]
    assert hi > lo, counts
    mins = W.nsamps * W.dt / 60.0
    rate = 0.5 * (lo + hi) / mins
    kw = _kw(W, max_giant_rate=rate)
    sep = _separate(beams, False, **kw)
    assert [s[0] for s in sep].count(H.HD_TOO_MANY_EVENTS) == 1
    with H.Pipeline(H.default_params(**kw), cleaning=False) as pl:
        err, _, st = pl.execute_beams(beams)
        assert st[5] == H.HD_TOO_MANY_EVENTS
        for u in range(len(beams)):
            if u == 5:
                continue
            assert H.cand_lines(pl.candidates(u)) == H.cand_lines(sep[u][2])
        assert err == H.HD_TOO_MANY_EVENTS


def test_batch_stf_units_and_device_pointers(hdb):
    """Filterbanks that each hold 2 time-concatenated beams, passed as device
    pointers, with explicit beam numbers."""
    torch = pytest.importorskip("torch")
    mb = synth.make_multibeam(W, seed=41, pulses_per_beam=2, snr_lo=12, snr_hi=30)
    fbs = [synth.stf(mb[2 * i:2 * i + 2]) for i in range(3)]
    kw = _kw(W, baseline_length=1.0)
    sep = _separate(fbs, True, nbeams=2, **kw)
    dev = [torch.from_numpy(f).cuda() for f in fbs]
    torch.cuda.synchronize()
    with H.Pipeline(H.default_params(**kw), cleaning=True) as pl:
        err, proc, st = pl.execute_beams([d.data_ptr() for d in dev], nsamps=fbs[0].shape[0],
                                         nbeams=2, beams=[0, 2, 4], on_device=True)
        assert proc == sep[0][1]
        _check(pl, err, st, sep)


def test_batch_cand_files(hdb, tmp_path):
    beams = _beams()[:3]
    kw = _kw(W, output_dir=str(tmp_path), spectra_per_second=1)
    with H.Pipeline(H.default_params(**kw), cleaning=False) as pl:
        pl.execute_beams(beams, beams=[4, 9, 10])
        names = sorted(f.name for f in tmp_path.glob("*.cand"))
        assert names == [f"1970-01-01-00:00:00_{b:02d}.cand" for b in (5, 10, 11)]
        for u, b in enumerate((5, 10, 11)):
            text = (tmp_path / f"1970-01-01-00:00:00_{b:02d}.cand").read_text().splitlines()
            assert text == H.cand_lines(pl.candidates(u))


def test_batch_errors(hdb):
    beams = _beams()[:2]
    with H.Pipeline(H.default_params(**_kw(W)), cleaning=False) as pl:
        # shorter than the largest delay (about 880 samples): nothing is dedispersed
        err, _, _ = pl.execute_beams([beams[0][:800], beams[1][:800]], raise_on_error=False)
        assert err == H.HD_TOO_FEW_NSAMPS
        # longer than the delay but shorter than delay + widest boxcar: no search
        err, proc, st = pl.execute_beams([beams[0][:1000], beams[1][:1000]])
        assert err == H.HD_NO_ERROR and st == [0, 0] and len(pl.candidates()) == 0
        n = H.C.c_size_t(0)
        assert H.lib().hd_get_beam_candidates(pl._p, 5, None, H.C.byref(n)) != H.HD_NO_ERROR


def test_prefetched_equals_execute_beams(hdb):
    """hd_prefetch_beams / hd_execute_prefetched: gulps queued ahead (two
    slots) are searched in queue order with exactly the results that
    hd_execute_beams gives for the same filterbanks."""
    gulps = [[np.ascontiguousarray(x) for x in _beams(seed=s)[:3]] for s in (31, 57, 31)]
    kw = _kw(W)
    beams = [4, 9, 10]

    def snapshot(pl, err, proc, st):
        g = pl.giants()
        return (err, proc, st, [H.cand_lines(pl.candidates(u)) for u in range(3)],
                g["inds"].tolist(), g["peaks"].view(np.uint32).tolist(), g["labels"].tolist())

    with H.Pipeline(H.default_params(**kw), cleaning=True) as ref:
        want = [snapshot(ref, *ref.execute_beams(g, first_idx=700 * k, beams=beams))
                for k, g in enumerate(gulps)]
    assert sum(len(c) for c in want[0][3]) >= 3
    ptrs = [[x.ctypes.data for x in g] for g in gulps]
    with H.Pipeline(H.default_params(**kw), cleaning=True) as pl:
        assert pl.execute_prefetched(3)[0] == H.HD_INVALID_POINTER  # nothing queued
        assert pl.prefetch_beams(ptrs[0], W.nsamps) == H.HD_NO_ERROR
        assert pl.prefetch_beams(ptrs[1], W.nsamps) == H.HD_NO_ERROR
        assert pl.prefetch_beams(ptrs[2], W.nsamps) == H.HD_INVALID_STRIDE  # both slots busy
        got = [snapshot(pl, *pl.execute_prefetched(3, first_idx=0, beams=beams))]
        assert pl.prefetch_beams(ptrs[2], W.nsamps) == H.HD_NO_ERROR
        for k in (1, 2):
            got.append(snapshot(pl, *pl.execute_prefetched(3, first_idx=700 * k, beams=beams)))
        assert pl.execute_prefetched(3)[0] == H.HD_INVALID_POINTER
    for k in range(3):
        assert got[k] == want[k], k
