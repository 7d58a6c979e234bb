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


def test_sigproc_gulp_loop_two_beams(hdb, tmp_path):
    """A file of 2 beams (nbeams = 2 in the header): each block of GULP
    spectra holds beam 0's GULP / 2 spectra and then beam 1's.  Every gulp is
    the STF concatenation of each beam's overlap carry and its part of the
    block, and its candidates equal an hd_execute of that gulp (cleaning on,
    so the per-beam cleaning of the loop's gulps is covered too)."""
    half = GULP // 2
    nfull, tail = 3, 3000
    per_beam = nfull * half + tail
    rng = np.random.default_rng(91)
    streams = []
    for b in range(2):
        pulses = [synth.Pulse(float(t), float(dm), 1e-3, 25.0)
                  for t, dm in zip(rng.uniform(2000, per_beam - 3000, 5), rng.uniform(20, 280, 5))]
        streams.append(synth.make_beam(per_beam, NCH, DT, F0, DF, pulses, seed=92 + b).data)
    rows = []
    for k in range(nfull):
        rows += [streams[0][k * half:(k + 1) * half], streams[1][k * half:(k + 1) * half]]
    rows.append(streams[0][nfull * half:])  # a short last block: not searched
    data = np.concatenate(rows)
    path = str(tmp_path / "two_beams.fil")
    synth.write_sigproc(path, data, nchans=NCH, nbits=8, tsamp=DT, fch1=F0, foff=DF,
                        tstart=60000.5, nifs=1, nbeams=2, ibeam=1, source_name="two_beams")
    kw = dict(dm_min=0.0, dm_max=300.0, boxcar_max=256)
    params = H.params_from_sigproc(path, H.default_params(output_dir=None, **kw))
    with H.Pipeline(params, cleaning=True) as pl:
        overlap = pl.max_overlap()  # per beam
        err, total, gulps = pl.search_sigproc_file(path, GULP)
    assert err == H.HD_NO_ERROR
    plan = oracle.gulp_plan(per_beam, half, overlap)
    assert len(gulps) == len(plan) == nfull
    assert total == sum(n - overlap for _, n, _ in plan)
    found = 0
    with H.Pipeline(params, cleaning=True) as ref:
        for (start, n, first), (first_got, got) in zip(plan, gulps):
            assert first_got == first
            g = np.concatenate([s[start:start + n] for s in streams])
            ref.execute(g, nbeams=2, first_idx=first)
            assert H.cand_lines(got) == H.cand_lines(ref.candidates())
            found += len(got)
    assert found >= 5


def test_sigproc_files_lockstep(hdb, tmp_path):
    """hd_search_sigproc_files over three single-beam files: every gulp is one
    hd_execute_beams call over the three files' gulps, and its candidates are,
    file by file, those of hd_search_sigproc_file on that file alone (with
    the file's beam number).  The shortest file ends the loop; files of
    another channel count are refused."""
    rng = np.random.default_rng(101)
    paths, lengths = [], [3 * GULP + 5000, 3 * GULP + 9000, 2 * GULP + 7000]
    for u, nsamps in enumerate(lengths):
        pulses = [synth.Pulse(float(t), float(dm), 1e-3, 25.0)
                  for t, dm in zip(rng.uniform(2000, nsamps - 4000, 6), rng.uniform(20, 280, 6))]
        b = synth.make_beam(nsamps, NCH, DT, F0, DF, pulses, seed=110 + u)
        path = str(tmp_path / f"beam{u}.fil")
        synth.write_sigproc(path, b.data, nchans=NCH, nbits=8, tsamp=DT, fch1=F0, foff=DF,
                            tstart=60000.5, nifs=1, ibeam=u + 1, source_name="lockstep")
        paths.append(path)
    kw = dict(dm_min=0.0, dm_max=300.0, boxcar_max=256, output_dir=None)

    def params(beam):
        q = H.default_params(**kw)
        q.override_beam = True
        q.beam = beam
        return H.params_from_sigproc(paths[0], q)

    singles = []
    for u, path in enumerate(paths):
        with H.Pipeline(params(u), cleaning=True) as pl:
            err, total, gulps = pl.search_sigproc_file(path, GULP)
            assert err == H.HD_NO_ERROR
            singles.append((total, gulps))
    with H.Pipeline(params(0), cleaning=True) as pl:
        err, total, gulps = pl.search_sigproc_files(paths, GULP)
    assert err == H.HD_NO_ERROR
    ng = min(len(g) for _, g in singles)
    assert ng == 2 and len(gulps) == ng
    assert total == singles[2][0]  # the shortest file's two gulps
    found = 0
    for k in range(ng):
        first, got = gulps[k]
        want = []
        for _, g_u in singles:
            assert g_u[k][0] == first
            want += H.cand_lines(g_u[k][1])
        assert H.cand_lines(got) == want
        found += len(got)
    assert found >= 6
    # files that do not share the search's shape are refused
    other = str(tmp_path / "other.fil")
    synth.write_sigproc(other, np.zeros((GULP, NCH // 2), np.uint8), nchans=NCH // 2, nbits=8,
                        tsamp=DT, fch1=F0, foff=DF, tstart=60000.5, nifs=1)
    with H.Pipeline(params(0), cleaning=True) as pl:
        err, _, gulps = pl.search_sigproc_files([paths[0], other], GULP)
    assert err == H.HD_INVALID_STRIDE and gulps == []


@pytest.mark.parametrize("nbits", [2, 4])
def test_sigproc_gulp_loop_packed_file(hdb, tmp_path, nbits):
    """A packed sigproc file (the reference's writer order) searched by the
    gulp loop gives, gulp by gulp, the candidates of the 8-bit file of the
    same sample values."""
    _, data = _file(tmp_path)
    v = (data >> (8 - nbits)).astype(np.uint8)
    hdr = dict(nchans=NCH, tsamp=DT, fch1=F0, foff=DF, tstart=60000.5, nifs=1,
               source_name="stream_test")
    packed_path, bytes_path = str(tmp_path / "packed.fil"), str(tmp_path / "bytes.fil")
    synth.write_sigproc(packed_path, synth.pack_filterbank(v, nbits), nbits=nbits, **hdr)
    synth.write_sigproc(bytes_path, v, nbits=8, **hdr)
    kw = dict(dm_min=0.0, dm_max=300.0, boxcar_max=256)
    out = []
    for path in (packed_path, bytes_path):
        params = H.params_from_sigproc(path, H.default_params(output_dir=None, **kw))
        with H.Pipeline(params, cleaning=False) as pl:
            err, total, gulps = pl.search_sigproc_file(path, GULP)
        assert err == H.HD_NO_ERROR
        out.append((total, [(first, H.cand_lines(c)) for first, c in gulps]))
    assert out[0] == out[1]
    assert len(out[0][1]) == 3 and sum(len(c) for _, c in out[0][1]) >= 3
