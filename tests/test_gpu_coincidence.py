"""hd_coincide (cross-beam coincidence on the GPU) and the _all.cand writer
against the reference's own coincidencer (Applications/Candidates.C,
oracle/_ref/coinc_ref, run where the reference was built) and against the
oracle's restatement: on synthetic per-beam lists, and on the .cand files
the batched pipeline writes for beams that share pulses."""
import os
import sys

import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import coinc_data as D  # noqa: E402

pytestmark = pytest.mark.gpu


def _check(tmp_path, bl, sep_time, sep_filter):
    rows = [H.parse_cand_lines(ls) for ls in bl]
    allrows = np.concatenate(rows)
    co = H.coincide(allrows, len(bl), sep_time, sep_filter)
    want = oracle.coincide(rows, sep_time, sep_filter)
    got = []
    o = 0
    for r in rows:
        got.append([(int(c["nbeams"]), int(c["primary_beam"]), np.float32(c["max_snr"]))
                    for c in co[o:o + len(r)]])
        o += len(r)
    assert got == [[(a, b, np.float32(c)) for a, b, c in w] for w in want]
    out = str(tmp_path / "gpu_all.cand")
    H.write_coincident_candidates(out, allrows, co)
    lines = open(out).read().splitlines()
    if oracle.ref_coinc_available():
        files = D.write_files(tmp_path, bl)
        assert lines == oracle.ref_coincide(files, len(bl), sep_time, sep_filter)
    return co


@pytest.mark.parametrize("seed,sep_time,sep_filter", [(3, 3, 4), (5, 1, 1), (6, 6, 8)])
def test_coincide_synthetic(hdb, tmp_path, seed, sep_time, sep_filter):
    _check(tmp_path, D.lines_by_beam(5, seed), sep_time, sep_filter)


def test_coincide_pipeline_beams(hdb, tmp_path):
    """Six beams searched in one batch, pulses shared by several beams at
    different S/N; the .cand files the pipeline writes go through both
    coincidencers."""
    w = synth.SEARCH_C2
    rng = np.random.default_rng(11)
    shared = [synth.Pulse(float(t), float(dm), 5e-3, 0.0)
              for t, dm in zip(rng.uniform(3000, 25000, 5), rng.uniform(100, 1800, 5))]
    beams = []
    for b in range(6):
        ps = [synth.Pulse(p.t0, p.dm, p.fwhm_s, float(rng.uniform(8, 40)))
              for p in shared if rng.random() < 0.7]
        beams.append(synth.make_beam(w.nsamps, w.nchans, w.dt, w.f0, w.df, ps, seed=12,
                                     beam=b).data)
    out_dir = tmp_path / "cands"
    out_dir.mkdir()
    p = H.default_params(nchans=w.nchans, dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min,
                         dm_max=w.dm_max, boxcar_max=w.boxcar_max, output_dir=str(out_dir))
    p.utc_start = 1700000000
    p.spectra_per_second = 1525
    with H.Pipeline(p, cleaning=False) as pl:
        err, _, _ = pl.execute_beams(beams)
        assert err == H.HD_NO_ERROR
    files = sorted(str(out_dir / f) for f in os.listdir(out_dir))
    assert len(files) == 6
    bl = [open(f).read().splitlines() for f in files]
    co = _check(tmp_path, bl, 3, 4)
    assert int(co["nbeams"].max()) >= 3
