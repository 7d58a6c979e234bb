"""Error paths on the GPU, made without faulting it.

* A bounded wait that runs out: with HDB_TEST_WITHHOLD_STAGE=1 the
  dedispersion kernel's producer issues no copy for its last channel stage,
  so the consumers' wait on that stage (a short limit in this mode) gives up
  and records it in the plan's error word.  The producer waits only for the
  copies it did issue, so no copy is in flight when a block exits.  The gulp
  returns HD_INTERNAL_GPU_ERROR and the next gulp on the same pipeline, with
  the switch cleared, equals the oracle.
* An allocation that fails: a batch whose first device buffer cannot fit on
  any GPU returns HD_MEM_ALLOC_FAILED before any input is read, and the
  pipeline searches the next gulp normally (the failure is not left in the
  runtime's error state for later launch checks to report).
"""
import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu


def _small():
    w = synth.SEARCH_C0
    pulses = [synth.Pulse(3000.0, 150.0, 1e-3, 30.0), synth.Pulse(9000.0, 60.0, 2e-3, 25.0)]
    b = synth.make_beam(1 << 14, 64, w.dt, w.f0, w.df * 4, pulses, seed=41)
    kw = dict(dt=w.dt, f0=w.f0, df=w.df * 4, dm_min=0.0, dm_max=300.0, boxcar_max=256)
    return b.data, kw


def _oracle_lines(fb, kw):
    r = oracle.execute(fb, clean=1, **kw)
    return oracle.cand_lines(r["groups"], fb.shape[0], 1, 0, r["nsamps_processed"],
                             kw["boxcar_max"], kw["dt"])


def test_dedisp_wait_gives_up_and_pipeline_recovers(hdb, oracle_lib, monkeypatch):
    fb, kw = _small()
    want = _oracle_lines(fb, kw)
    assert len(want) >= 2
    monkeypatch.setenv("HDB_DEDISP_TILE", "16x512")
    with H.Pipeline(H.default_params(nchans=fb.shape[1], output_dir=None, **kw)) as pl:
        monkeypatch.setenv("HDB_TEST_WITHHOLD_STAGE", "1")
        err, _ = pl.execute(fb, raise_on_error=False)
        assert err == H.HD_INTERNAL_GPU_ERROR
        monkeypatch.delenv("HDB_TEST_WITHHOLD_STAGE")
        err, _ = pl.execute(fb, raise_on_error=False)
        assert err == H.HD_NO_ERROR
        assert H.cand_lines(pl.candidates()) == want
    # the dedisp_* interface reports the same failure and recovers too
    plan = H.DedispPlan(fb.shape[1], kw["dt"], kw["f0"], kw["df"])
    plan.generate_dm_list(0.0, 300.0, 40.0, 1.25)
    monkeypatch.setenv("HDB_TEST_WITHHOLD_STAGE", "1")
    with pytest.raises(RuntimeError, match="Internal GPU error"):
        plan.execute(fb)
    monkeypatch.delenv("HDB_TEST_WITHHOLD_STAGE")
    table = oracle.delay_table(fb.shape[1], kw["dt"], kw["f0"], kw["df"])
    np.testing.assert_array_equal(plan.execute(fb), oracle.dedisperse(fb, plan.dm_list, table))


def test_allocation_failure_reported_and_pipeline_recovers(hdb, oracle_lib):
    import torch
    fb, kw = _small()
    want = _oracle_lines(fb, kw)
    d = torch.from_numpy(fb).cuda()
    torch.cuda.synchronize()
    with H.Pipeline(H.default_params(nchans=fb.shape[1], output_dir=None, **kw)) as pl:
        # 500 filterbanks of 2^24 spectra x 64 channels: the first device
        # buffer (512 GiB of input) cannot be allocated on any GPU, and the call
        # returns before it reads the inputs (all the same, too short buffer)
        err, _, _ = pl.execute_beams([d.data_ptr()] * 500, nsamps=1 << 24, on_device=True,
                                     raise_on_error=False)
        assert err == H.HD_MEM_ALLOC_FAILED
        err, _ = pl.execute_device(d.data_ptr(), fb.shape[0])
        assert err == H.HD_NO_ERROR
        assert H.cand_lines(pl.candidates()) == want
