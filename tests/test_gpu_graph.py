"""The batched gulp as a CUDA graph replay (hd_execute_beams with device input,
hd_execute_prefetched).

The first gulp of a shape runs on the host-sized path; later gulps of the
shape replay one captured graph whose hit and giant totals stay on the device.
Every replayed gulp must give exactly what the host-sized path gives for the
same filterbanks (candidate rows with SNR bits, giants, labels, statuses),
including when a gulp overflows the captured capacities or needs more
clustering sweeps than were captured: those gulps are searched again on the
host-sized path.  The host-sized path itself is checked against separate
per-beam hd_execute calls and the oracle in test_gpu_batch.py.
"""
import numpy as np
import pytest

import heimdall_multibeam_b200 as H
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu

# 8 beams x 128 channels, 2^14 samples each (a scaled-down multibeam gulp)
W = synth.Workload("mb8_c128_n16384", 128, 655.36e-6, 851.0, -0.3125, 1 << 14, 8, 0.0, 1000.0,
                   256, False, "")


def _kw(**extra):
    d = dict(nchans=W.nchans, dt=W.dt, f0=W.f0, df=W.df, dm_min=W.dm_min, dm_max=W.dm_max,
             boxcar_max=W.boxcar_max, output_dir=None)
    d.update(extra)
    return d


def _gulp(seed, pulses=3, dense=False):
    beams = [b.data for b in synth.make_multibeam(W, seed=seed, pulses_per_beam=pulses,
                                                  snr_lo=10, snr_hi=30)]
    if dense:
        # many strong pulses in two beams: far more hits and giants than a
        # quiet gulp of the same shape
        rng = np.random.default_rng(seed)
        for u in (2, 6):
            many = [synth.Pulse(float(t), float(rng.uniform(50, 900)), 2e-3, 30.0)
                    for t in np.linspace(600, W.nsamps - 1500, 40)]
            beams[u] = synth.make_beam(W.nsamps, W.nchans, W.dt, W.f0, W.df, many,
                                       seed=seed + 7, beam=u).data
    return beams


def _result(pl, err, st):
    g = pl.giants()
    return (err, list(st), [H.cand_lines(pl.candidates(u)) for u in range(W.nbeams)],
            [pl.candidates(u)["snr"].view(np.uint32).tolist() for u in range(W.nbeams)],
            {k: np.asarray(v).copy() for k, v in g.items()})


def _same(a, b):
    assert a[0] == b[0]
    assert a[1] == b[1]
    assert a[2] == b[2]
    assert a[3] == b[3]
    assert set(a[4]) == set(b[4])
    for k in a[4]:
        np.testing.assert_array_equal(a[4][k].view(np.uint8), b[4][k].view(np.uint8), err_msg=k)


def _host_sized(gulps, clean):
    """Each gulp through a pipeline with the graph form off."""
    torch = pytest.importorskip("torch")
    out = []
    with H.Pipeline(H.default_params(**_kw()), cleaning=clean) as pl:
        pl.set_graphs(False)
        for beams in gulps:
            d = [torch.from_numpy(b).cuda() for b in beams]
            err, _, st = pl.execute_beams([t.data_ptr() for t in d], nsamps=W.nsamps,
                                          on_device=True, raise_on_error=False)
            torch.cuda.synchronize()
            out.append(_result(pl, err, st))
        assert pl.graph_replays() == 0
    return out


@pytest.mark.parametrize("clean", [False, True])
def test_replays_equal_host_sized(hdb, clean):
    torch = pytest.importorskip("torch")
    gulps = [_gulp(51), _gulp(52), _gulp(53), _gulp(52)]
    want = _host_sized(gulps, clean)
    assert sum(len(c) for c in want[1][2]) >= 8
    # one set of device buffers refilled per gulp: one capture, then replays
    bufs = [torch.empty((W.nsamps, W.nchans), dtype=torch.uint8, device="cuda")
            for _ in range(W.nbeams)]
    with H.Pipeline(H.default_params(**_kw()), cleaning=clean) as pl:
        for k, beams in enumerate(gulps):
            for t, b in zip(bufs, beams):
                t.copy_(torch.from_numpy(b))
            err, _, st = pl.execute_beams([t.data_ptr() for t in bufs], nsamps=W.nsamps,
                                          on_device=True, raise_on_error=False)
            _same(_result(pl, err, st), want[k])
        assert pl.graph_replays() == len(gulps) - 1
        # other input buffers: a second capture, the same results
        other = [torch.from_numpy(b).cuda() for b in gulps[2]]
        err, _, st = pl.execute_beams([t.data_ptr() for t in other], nsamps=W.nsamps,
                                      on_device=True, raise_on_error=False)
        _same(_result(pl, err, st), want[2])
        assert pl.graph_replays() == len(gulps)


def test_overflow_and_extra_sweeps_fall_back(hdb, monkeypatch):
    """Capacities far below a dense gulp's totals and a single sweep pair: the
    replay's overflow (or unfinished clustering) sends the gulp back to the
    host-sized path, the capacities grow, and the next replay serves it."""
    torch = pytest.importorskip("torch")
    monkeypatch.setenv("HDB_GRAPH_CAPS", "64,16,1")
    quiet, dense = _gulp(61, pulses=1), _gulp(62, dense=True)
    gulps = [quiet] + [dense] * 6
    want = _host_sized(gulps[:2], False)
    assert sum(len(c) for c in want[1][2]) > 16
    d = [torch.from_numpy(b).cuda() for b in quiet], [torch.from_numpy(b).cuda() for b in dense]
    with H.Pipeline(H.default_params(**_kw()), cleaning=False) as pl:
        for k in range(len(gulps)):
            err, _, st = pl.execute_beams([t.data_ptr() for t in d[min(k, 1)]],
                                          nsamps=W.nsamps, on_device=True, raise_on_error=False)
            _same(_result(pl, err, st), want[min(k, 1)])
        # the first dense gulp overflows (no replay serves it); once the
        # capacities and the sweep pairs have grown, replays serve the rest
        assert 2 <= pl.graph_replays() <= 5


def test_prefetched_gulps_replay(hdb):
    """The streaming form: gulps copied ahead into rotating slots, each
    searched in place; every gulp equals the host-sized search."""
    torch = pytest.importorskip("torch")
    gulps = [_gulp(71 + k) for k in range(6)]
    want = _host_sized(gulps, False)
    host = [[torch.from_numpy(b).pin_memory() for b in beams] for beams in gulps]
    with H.Pipeline(H.default_params(**_kw()), cleaning=False) as pl:
        assert pl.prefetch_beams([t.data_ptr() for t in host[0]], W.nsamps) == H.HD_NO_ERROR
        for k in range(len(gulps)):
            if k + 1 < len(gulps):
                assert pl.prefetch_beams([t.data_ptr() for t in host[k + 1]],
                                         W.nsamps) == H.HD_NO_ERROR
            err, _, st = pl.execute_prefetched(W.nbeams)
            _same(_result(pl, err, st), want[k])
        assert pl.graph_replays() >= 2


def test_graphs_off_for_adaptive_dt(hdb):
    """Adaptive dt stays on the host-sized path (no replay)."""
    torch = pytest.importorskip("torch")
    beams = _gulp(81)
    d = [torch.from_numpy(b).cuda() for b in beams]
    with H.Pipeline(H.default_params(**_kw(use_scrunching=True)), cleaning=False) as pl:
        for _ in range(3):
            pl.execute_beams([t.data_ptr() for t in d], nsamps=W.nsamps, on_device=True,
                             raise_on_error=False)
        assert pl.graph_replays() == 0
