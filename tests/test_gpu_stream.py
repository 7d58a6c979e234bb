"""The gulp loop over a sigproc file (hd_search_sigproc_file,
Applications/heimdall.C:153-292): the overlap carried on the device and the
blocks read while the GPU searches give, gulp by gulp, the candidates of an
hd_execute of the gulp the loop's plan predicts (oracle.gulp_plan) and the
CPU oracle's .cand lines for it; the short last block is not searched."""
import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu

NCH, DT, F0, DF = 256, 64e-6, 1500.0, -1.5625
GULP = 16384


def _file(tmp_path):
    nsamps = 3 * GULP + 6000
    rng = np.random.default_rng(77)
    pulses = [synth.Pulse(float(t), float(dm), 1e-3, 25.0)
              for t, dm in zip(rng.uniform(2000, nsamps - 4000, 9), rng.uniform(20, 280, 9))]
    b = synth.make_beam(nsamps, NCH, DT, F0, DF, pulses, seed=78)
    path = str(tmp_path / "stream.fil")
    synth.write_sigproc(path, b.data, nchans=NCH, nbits=8, tsamp=DT, fch1=F0, foff=DF,
                        tstart=60000.5, nifs=1, source_name="stream_test")
    return path, b.data


def test_sigproc_gulp_loop(hdb, oracle_lib, tmp_path):
    path, data = _file(tmp_path)
    kw = dict(dm_min=0.0, dm_max=300.0, boxcar_max=256)
    params = H.params_from_sigproc(path, H.default_params(output_dir=None, **kw))
    assert params.nchans == NCH and params.nbeams == 1
    with H.Pipeline(params, cleaning=False) as pl:
        overlap = pl.max_overlap()
        err, total, gulps = pl.search_sigproc_file(path, GULP)
    assert err == H.HD_NO_ERROR
    plan = oracle.gulp_plan(data.shape[0], GULP, overlap)
    assert len(gulps) == len(plan) == 3
    assert total == sum(n - overlap for _, n, _ in plan)
    found = 0
    with H.Pipeline(params, cleaning=False) as ref:
        for (start, n, first), (first_got, got) in zip(plan, gulps):
            assert first_got == first
            g = data[start:start + n]
            ref.execute(g, first_idx=first)
            want = ref.candidates()
            assert H.cand_lines(got) == H.cand_lines(want)
            r = oracle.execute(g, first_idx=first, clean=0, dt=DT, f0=F0, df=DF, **kw)
            lines = oracle.cand_lines(r["groups"], n, 1, first, r["nsamps_processed"], 256, DT)
            assert H.cand_lines(got) == lines
            found += len(got)
    assert found >= 9
