"""Sigproc input (no GPU): hd_read_sigproc_header, hd_mjd_to_utc and
hd_params_from_sigproc against the reference's own reader and conversion
(Formats/hd/header.h:133-198, Formats/hd/DataSource.h:49-82, compiled from
the reference's headers into oracle/_ref/sigproc_dump), and the gulp plan of
the streaming loop (Applications/heimdall.C:153-292)."""
import os

import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

FULL = dict(telescope_id=7, machine_id=3, data_type=1, source_name="FRB_TEST_0001",
            rawdatafile="beam_04.fil", az_start=123.25, za_start=17.5, src_raj=123456.78,
            src_dej=-452310.5, tstart=60123.4567891234, tsamp=6.4e-05, fch1=1520.0,
            foff=-0.390625, nchans=1024, nbits=8, nifs=1, nbeams=13, ibeam=4, barycentric=0,
            pulsarcentric=0, refdm=123.4)

need_ref = pytest.mark.skipif(not oracle.ref_sigproc_available(),
                              reason="oracle/_ref/sigproc_dump is built from the reference "
                                     "(make -C oracle ref)")


def _write(tmp_path, name, nsamps=100, **fields):
    f = dict(FULL)
    f.update(fields)
    nc = f["nchans"]
    data = (np.arange(nsamps * nc) % 251).astype(np.uint8).reshape(nsamps, nc)
    path = str(tmp_path / name)
    size = synth.write_sigproc(path, data, **f)
    return path, size, data


def test_header_fields(hdb, tmp_path):
    path, size, _ = _write(tmp_path, "a.fil", nsamples=100, signed=1)
    h = H.read_sigproc_header(path)
    assert h["size"] == size
    for k, v in FULL.items():
        assert h[k] == v, k
    assert h["nsamples"] == 100 and h["signed_data"] == 1 and h["unknown_keys"] == 0


@need_ref
@pytest.mark.parametrize("case", ["full", "no_nsamples", "unknown_key", "reordered", "minimal"])
def test_header_matches_reference_reader(hdb, tmp_path, case):
    if case == "full":
        path, _, _ = _write(tmp_path, "f.fil", nsamples=100, signed=0, period=0.7,
                            nbins=5, npuls=2)
    elif case == "no_nsamples":
        # nsamples from the file size, header included (the reference's rule)
        path, _, _ = _write(tmp_path, "n.fil", nsamps=333, nchans=64)
    elif case == "unknown_key":
        path = str(tmp_path / "u.fil")
        synth.write_sigproc(path, np.zeros((10, 64), np.uint8), nchans=64, nbits=8,
                            tsamp=1e-3, fch1=1400.0, foff=-1.0, mystery=0, tstart=55000.5)
    elif case == "reordered":
        path = str(tmp_path / "r.fil")
        synth.write_sigproc(path, np.zeros((10, 32), np.uint8),
                            order=["foff", "source_name", "nbits", "tstart", "nchans"],
                            source_name="X", nbits=8, tstart=59000.25, nchans=32, foff=-2.0,
                            fch1=1300.0, tsamp=2e-4)
    else:
        path = str(tmp_path / "m.fil")
        synth.write_sigproc(path, np.zeros((7, 16), np.uint8), nchans=16, nbits=8)
    ref = oracle.ref_sigproc_dump(path)
    assert ref["ok"]
    got = H.read_sigproc_header(path)
    for k in ("source_name", "rawdatafile", "az_start", "za_start", "src_raj", "src_dej",
              "tstart", "tsamp", "period", "fch1", "foff", "refdm", "nchans", "telescope_id",
              "machine_id", "data_type", "ibeam", "nbeams", "nbits", "barycentric",
              "pulsarcentric", "nbins", "nsamples", "nifs", "npuls", "size"):
        assert got[k] == ref[k], (k, got[k], ref[k])
    if case == "unknown_key":
        assert got["unknown_keys"] == 1


@need_ref
def test_mjd_to_utc_matches_reference(hdb, tmp_path):
    path, _, _ = _write(tmp_path, "t.fil")
    rng = np.random.default_rng(5)
    mjds = [40587.0, 40587.5, 51544.0, 51544.99999, 54000.123456, 55197.0, 60000.0,
            60123.4567891234, 60676.999999] + list(rng.uniform(45000, 70000, 40))
    ref = oracle.ref_sigproc_dump(path, mjds)["utc"]
    got = [H.lib().hd_mjd_to_utc(m) for m in mjds]
    assert got == ref


def test_params_from_header(hdb, tmp_path):
    path, _, _ = _write(tmp_path, "p.fil")
    p = H.params_from_sigproc(path)
    assert p.nchans == 1024 and p.nbeams == 13 and p.beam == 3
    assert p.dt == np.float32(6.4e-05) and p.f0 == 1520.0 and p.df == np.float32(-0.390625)
    assert p.spectra_per_second == int(1.0 / np.float32(6.4e-05))  # 15625
    assert p.utc_start == H.lib().hd_mjd_to_utc(FULL["tstart"])
    q = H.default_params()
    q.override_beam = True
    q.beam = 9
    assert H.params_from_sigproc(path, q).beam == 9


def test_bad_headers(hdb, tmp_path):
    bad = tmp_path / "bad.fil"
    bad.write_bytes(b"\x05\x00\x00\x00HELLO" + b"\x00" * 64)
    with pytest.raises(H.HdError):
        H.read_sigproc_header(str(bad))
    path, size, _ = _write(tmp_path, "trunc.fil")
    with open(path, "rb") as f:
        head = f.read(size // 2)
    trunc = tmp_path / "trunc2.fil"
    trunc.write_bytes(head)
    with pytest.raises(H.HdError):
        H.read_sigproc_header(str(trunc))
    with pytest.raises(H.HdError):
        H.read_sigproc_header(str(tmp_path / "missing.fil"))


def test_gulp_plan():
    # one beam, gulps of 1000 spectra, overlap 300, 3750 spectra in the file
    plan = oracle.gulp_plan(3750, 1000, 300)
    assert plan == [(0, 1000, 0), (700, 1300, 700), (1700, 1300, 1700)]
    # every searched spectrum is searched once: gulp k covers [first_idx, first_idx + n - 300)
    cover = [(s, s + n - 300) for s, n, _ in plan]
    assert all(a[1] == b[0] for a, b in zip(cover, cover[1:]))
    assert oracle.gulp_plan(999, 1000, 300) == []
    assert oracle.gulp_plan(2000, 1000, 300) == [(0, 1000, 0), (700, 1300, 700)]
