"""Beams of different shapes in one call (hd_execute_beam_set): every beam's
candidates, status and processed count equal a separate hd_execute of that
beam with its own parameters.  Shapes follow the uneven-beam workload
(channel counts, gulp lengths, sampling times and DM ranges that differ from
beam to beam; RFI and cleaning as the survey-size beam) at sizes a test can
generate on the host."""
import dataclasses

import numpy as np
import pytest

import heimdall_multibeam_b200 as H
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FIELDS = ("snr", "samp_idx", "time", "filter", "dm_trial", "dm", "members", "begin", "end", "beam")


def _params(w, beam):
    p = H.default_params(nchans=w.nchans, dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min,
                         dm_max=w.dm_max, boxcar_max=w.boxcar_max, output_dir=None)
    p.beam = beam
    return p


def _beams():
    ws = synth.uneven_shapes(8, seed=31, nchans=(128, 256, 512, 1024),
                             nsamps_range=(1 << 14, 1 << 15), dm_maxes=(300.0, 500.0, 1000.0),
                             boxcar_max=1024)
    # a twin of beam 0 (same shape and length: one batched run of two) and a
    # beam too short for its DM range (HD_TOO_FEW_NSAMPS)
    ws.append(dataclasses.replace(ws[0], name="twin"))
    ws.append(dataclasses.replace(ws[3], name="short", nsamps=4096, dm_max=1200.0))
    beams = [synth.make_uneven_beam(w, seed=31, beam=b) for b, w in enumerate(ws)]
    return ws, beams


def _check(bs, ws, beams, st, proc, cleaning=True):
    assert len(set(w.nchans for w in ws)) >= 4
    assert len(set(w.nsamps for w in ws)) >= 8
    nc_total = 0
    for b, (w, beam) in enumerate(zip(ws, beams)):
        with H.Pipeline(_params(w, 10 + b), cleaning=cleaning) as pl:
            err, processed = pl.execute(beam.data, raise_on_error=False)
            ref = pl.candidates()
        assert st[b] == err, (b, st[b], err)
        assert proc[b] == processed, (b, proc[b], processed)
        got = bs.candidates(b)
        assert len(got) == len(ref), (b, len(got), len(ref))
        for f in FIELDS:
            np.testing.assert_array_equal(got[f], ref[f], err_msg=f"beam {b} field {f}")
        nc_total += len(ref)
    return nc_total


def test_beam_set_matches_separate_pipelines(hdb):
    ws, beams = _beams()
    params = [_params(w, 10 + b) for b, w in enumerate(ws)]
    with H.BeamSet(params, workers=3, cleaning=True) as bs:
        assert bs.nconfigs == len(ws) - 1  # the twin shares beam 0's configuration
        err, st, proc = bs.execute([b.data for b in beams])
        assert st[-1] == H.HD_TOO_FEW_NSAMPS
        # the status of the lowest-numbered beam that did not succeed
        assert err == next(x for x in st if x != H.HD_NO_ERROR)
        n = _check(bs, ws, beams, st, proc)
        assert n > 10
        # a second call reuses the workers' pipelines and gives the same lists
        first = [bs.candidates(b) for b in range(len(ws))]
        bs.execute([b.data for b in beams])
        for b in range(len(ws)):
            for f in FIELDS:
                np.testing.assert_array_equal(bs.candidates(b)[f], first[b][f])


def test_beam_set_device_inputs_and_cleaning_off(hdb):
    ws, beams = _beams()
    ws, beams = ws[:-1], beams[:-1]
    params = [_params(w, 10 + b) for b, w in enumerate(ws)]
    dev = [torch.from_numpy(b.data).cuda() for b in beams]
    torch.cuda.synchronize()
    with H.BeamSet(params, workers=4, cleaning=False) as bs:
        err, st, proc = bs.execute([d.data_ptr() for d in dev], nsamps=[w.nsamps for w in ws],
                                   on_device=True)
        assert err in (H.HD_NO_ERROR, H.HD_TOO_MANY_EVENTS)
        _check(bs, ws, beams, st, proc, cleaning=False)


def test_beam_set_one_worker_equals_many(hdb):
    ws, beams = _beams()
    params = [_params(w, 10 + b) for b, w in enumerate(ws)]
    out = []
    for workers in (1, 5):
        with H.BeamSet(params, workers=workers) as bs:
            bs.execute([b.data for b in beams])
            out.append([bs.candidates(b) for b in range(len(ws))])
    for b in range(len(ws)):
        for f in FIELDS:
            np.testing.assert_array_equal(out[0][b][f], out[1][b][f])


def test_beam_set_concurrent_workers_repeat(hdb):
    """Many workers launching the same kernels with different shared-memory
    sizes at once (every configuration differs): repeated calls never fail
    and always give the same lists."""
    ws, beams = _beams()
    ws, beams = ws[:-1], beams[:-1]
    params = [_params(w, 10 + b) for b, w in enumerate(ws)]
    dev = [torch.from_numpy(b.data).cuda() for b in beams]
    torch.cuda.synchronize()
    with H.BeamSet(params, workers=len(ws), cleaning=True) as bs:
        first = None
        for _ in range(6):
            err, st, _ = bs.execute([d.data_ptr() for d in dev], nsamps=[w.nsamps for w in ws],
                                    on_device=True)
            assert err in (H.HD_NO_ERROR, H.HD_TOO_MANY_EVENTS), st
            lists = [H.cand_lines(bs.candidates(b)) for b in range(len(ws))]
            if first is None:
                first = lists
            assert lists == first
