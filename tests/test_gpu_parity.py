"""GPU parity: the CUDA product (through its C-ABI) against the oracle.

Integer work (dedispersed sums, zapped filterbank, masks, giant indices,
widths, DM indices, labels, counts) must be bit-exact.  Float SNRs are
compared bit-exactly too: every float expression of the chain is evaluated in
the reference's order on both sides (the 1e-4 relative bound of the
specification is asserted as well, for the record)."""
import os

import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
SNR_RTOL = 1e-4


def _params(w, **kw):
    d = dict(nchans=w.nchans, dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min, dm_max=w.dm_max,
             boxcar_max=w.boxcar_max)
    d.update(kw)
    return d


def _run_gpu(fb, nbeams=1, clean=True, zaps=(), **kw):
    p = H.default_params(output_dir=None, **kw)
    with H.Pipeline(p, cleaning=clean, channel_zaps=zaps) as pl:
        err, proc = pl.execute(fb, nbeams=nbeams, raise_on_error=False)
        return err, proc, pl.candidates(), pl.giants()


def _compare(fb, nbeams, w, clean, zaps=(), **kw):
    pk = _params(w, **kw)
    okw = dict(pk)
    okw.pop("nchans")
    r = oracle.execute(fb, nbeams=nbeams, clean=int(clean), channel_zaps=list(zaps), **okw)
    err, proc, cands, g = _run_gpu(fb, nbeams=nbeams, clean=clean, zaps=zaps, **pk)
    assert err == r["error"]
    assert proc == r["nsamps_processed"]
    if err == H.HD_TOO_MANY_EVENTS:
        # the reference stops searching at the bail-out; only the (empty)
        # candidate list is defined
        assert len(cands) == 0
        return cands
    og = r["giants"]
    assert len(g["peaks"]) == len(og["peaks"])
    for k in ("inds", "begins", "ends", "filter_inds", "dm_inds"):
        np.testing.assert_array_equal(g[k], og[k], err_msg=k)
    np.testing.assert_allclose(g["peaks"], og["peaks"], rtol=SNR_RTOL)
    np.testing.assert_array_equal(g["peaks"].view(np.uint32), og["peaks"].view(np.uint32))
    np.testing.assert_array_equal(g["labels"], r["labels"])
    lines = oracle.cand_lines(r["groups"], fb.shape[0], nbeams, 0, r["nsamps_processed"],
                              w.boxcar_max, w.dt)
    assert H.cand_lines(cands) == lines
    return cands


def test_dedisp_bit_exact(hdb, oracle_lib):
    rng = np.random.default_rng(5)
    nchans, nsamps = 128, 20000
    fb = rng.integers(0, 256, size=(nsamps, nchans), dtype=np.uint8)
    plan = H.DedispPlan(nchans, 64e-6, 1500.0, -1.5625)
    plan.generate_dm_list(0.0, 300.0, 40.0, 1.25)
    dms = plan.dm_list
    table = oracle.delay_table(nchans, 64e-6, 1500.0, -1.5625)
    np.testing.assert_array_equal(
        dms, oracle.dm_list(0.0, 300.0, 64e-6, 40.0, 1500.0, -1.5625, nchans, 1.25))
    out = plan.execute(fb)
    ref = oracle.dedisperse(fb, dms, table)
    assert out.shape == ref.shape
    np.testing.assert_array_equal(out, ref)
    km = np.ones(nchans, np.int32)
    km[[3, 17, 64, 65, 127]] = 0
    plan.set_killmask(km)
    np.testing.assert_array_equal(plan.execute(fb), oracle.dedisperse(fb, dms, table, km))


def test_dedisp_odd_sizes(hdb, oracle_lib):
    """Ragged sizes: channel count not a multiple of the staging chunk, DM
    count not a multiple of the DM block, output length not a multiple of the
    time block."""
    rng = np.random.default_rng(9)
    nchans, nsamps = 36, 7001
    fb = rng.integers(0, 256, size=(nsamps, nchans), dtype=np.uint8)
    plan = H.DedispPlan(nchans, 128e-6, 1400.0, -4.0)
    dms = np.array([0.0, 3.0, 77.7, 150.0, 151.0, 299.0, 300.0], np.float32)
    plan.set_dm_list(dms)
    table = oracle.delay_table(nchans, 128e-6, 1400.0, -4.0)
    np.testing.assert_array_equal(plan.execute(fb), oracle.dedisperse(fb, dms, table))


@pytest.mark.parametrize("nchans,dt,dm_max,nsamps,rows", [
    (128, 128e-6, 2000.0, 26000, 2),   # 6.5 KB staged rows: 2 rows per stage
    (128, 64e-6, 2000.0, 50000, 1),    # 13 KB rows: 1 row per stage
    (512, 128e-6, 5000.0, 62000, 4),   # 5 KB rows: 4 rows per stage
])
def test_dedisp_long_delay_spans(hdb, oracle_lib, nchans, dt, dm_max, nsamps, rows):
    """Few channels over a wide DM range (a 400 MHz band below 1520 MHz):
    the delay span of a 16-trial DM block is thousands of samples, so the
    staged channel rows are long and the kernel stages fewer rows per
    stage (`rows`, from the rows' length); the sums stay bit-exact."""
    rng = np.random.default_rng(nchans + nsamps)
    fb = rng.integers(0, 256, size=(nsamps, nchans), dtype=np.uint8)
    df = -400.0 / nchans
    plan = H.DedispPlan(nchans, dt, 1520.0, df)
    plan.generate_dm_list(0.0, dm_max, 40.0, 1.25)
    dms = plan.dm_list
    table = oracle.delay_table(nchans, dt, 1520.0, df)
    dl = oracle.delays(dms, table).astype(np.int64)
    span = max(int((dl[b:b + 16].max(0) - dl[b:b + 16].min(0)).max()) for b in range(0, len(dms), 16))
    rowb = (span + 16 + 512 + 8 + 15) // 16 * 16
    smem = [128 + 3 * 16 * ch * 4 + 3 * ch * rowb for ch in (8, 4, 2, 1)]
    want = next(ch for cap in (72 << 10, 110 << 10, 200 << 10)
                for ch, sm in zip((8, 4, 2, 1), smem) if sm <= cap)
    assert want == rows
    out = plan.execute(fb)
    np.testing.assert_array_equal(out, oracle.dedisperse(fb, dms, table))


TILES = ["8x1024", "8x640", "8x768", "8x1152", "8x1280", "16x512", "16x384", "16x640",
         "16x768", "32x256", "32x384"]


@pytest.mark.parametrize("tile", TILES)
def test_dedisp_every_tile(hdb, oracle_lib, tile, monkeypatch):
    """Every dedispersion tile the autotuner may pick (DM trials x output
    samples per CTA, forced through HDB_DEDISP_TILE; lanes owning 1, 3 or 5
    consecutive output words) gives the oracle's sums, for short rows and for
    long ones (128 channels over DM 0-2000)."""
    monkeypatch.setenv("HDB_DEDISP_TILE", tile)
    db, tb = (int(x) for x in tile.split("x"))
    for nchans, dt, f0, df, dm_max, nsamps in [(256, 64e-6, 1500.0, -1.5625, 1000.0, 30000),
                                               (128, 64e-6, 1520.0, -3.125, 2000.0, 50000)]:
        rng = np.random.default_rng(nchans)
        fb = rng.integers(0, 256, size=(nsamps, nchans), dtype=np.uint8)
        plan = H.DedispPlan(nchans, dt, f0, df)
        plan.generate_dm_list(0.0, dm_max, 40.0, 1.25)
        table = oracle.delay_table(nchans, dt, f0, df)
        np.testing.assert_array_equal(plan.execute(fb), oracle.dedisperse(fb, plan.dm_list, table))
    # the pipeline reports the tile it used
    w = synth.SEARCH_C0
    b = synth.make_c0()
    with H.Pipeline(H.default_params(nchans=w.nchans, dt=w.dt, f0=w.f0, df=w.df, dm_max=w.dm_max,
                                     boxcar_max=w.boxcar_max, output_dir=None),
                    cleaning=False) as pl:
        pl.execute(b.data)
        assert pl.dedisp_tile()[:2] == (db, tb)


def test_dedisp_autotuner_keeps_results(hdb, monkeypatch):
    """The autotuned tile is one of the candidates and the gulp's candidates
    equal those of the default tile."""
    w = synth.SEARCH_C0
    b = synth.make_c0()
    kw = dict(nchans=w.nchans, dt=w.dt, f0=w.f0, df=w.df, dm_max=w.dm_max,
              boxcar_max=w.boxcar_max, output_dir=None)
    out = {}
    for mode in ("tuned", "default"):
        if mode == "default":
            monkeypatch.setenv("HDB_DEDISP_TUNE", "0")
        with H.Pipeline(H.default_params(**kw), cleaning=False) as pl:
            pl.execute(b.data)
            out[mode] = (pl.candidates(), pl.dedisp_tile())
    assert out["default"][1][:2] == (16, 512)
    assert "%dx%d" % out["tuned"][1][:2] in TILES
    np.testing.assert_array_equal(out["tuned"][0], out["default"][0])


def test_clean_bit_exact(hdb, oracle_lib):
    w = synth.SEARCH_C1
    b = synth.make_beam(1 << 15, 64, w.dt, w.f0, w.df * 16,
                        [synth.Pulse(4000.0, 0.0, 0.5e-3, 40.0)], seed=3, n_bursts=6,
                        rfi_chan_frac=0.05)
    ref_out, ref_mask = oracle.clean_filterbank(b.data, w.dt)
    assert ref_mask.sum() > 0
    with H.Pipeline(H.default_params(nchans=64, output_dir=None)) as pl:
        out, mask = pl.clean_filterbank_rfi(b.data, w.dt)
    np.testing.assert_array_equal(mask, ref_mask)
    np.testing.assert_array_equal(out, ref_out)


@pytest.mark.parametrize("clean", [False, True])
def test_execute_c0(hdb, oracle_lib, clean):
    b = synth.make_c0()
    cands = _compare(b.data, 1, synth.SEARCH_C0, clean)
    assert len(cands) >= 3


@pytest.mark.parametrize("bmax", [1, 2, 4, 8])
def test_execute_small_boxcar(hdb, oracle_lib, bmax):
    """Boxcar offsets below 4 or not a multiple of 4 take the scalar
    threshold and block-RMS kernels; 8 is the smallest vector case."""
    b = synth.make_c0()
    cands = _compare(b.data, 1, synth.SEARCH_C0, False, boxcar_max=bmax)
    assert len(cands) >= 1


def test_execute_multibeam(hdb, oracle_lib):
    w = synth.Workload("mb_small", 64, 655.36e-6, 851.0, -0.390625, 8192, 4, 0.0, 600.0, 256,
                       False, "")
    beams = synth.make_multibeam(w, seed=7, snr_lo=15, snr_hi=30)
    _compare(synth.stf(beams), w.nbeams, w, True, baseline_length=1.0)


def test_execute_zaps_and_rate(hdb, oracle_lib):
    w = synth.SEARCH_C1
    df = w.df * 8
    pulses = [synth.Pulse(3000.0, 120.0, 1e-3, 25.0), synth.Pulse(9000.0, 400.0, 4e-3, 15.0)]
    b = synth.make_beam(1 << 15, 128, w.dt, w.f0, df, pulses, seed=11, n_bursts=3)
    kw = dict(df=df, dm_max=500.0, boxcar_max=256)
    wl = synth.Workload("z", 128, w.dt, w.f0, df, 1 << 15, 1, 0.0, 500.0, 256, True, "")
    cands = _compare(b.data, 1, wl, True, zaps=((10, 20), (100, 128)), **kw)
    assert len(cands) >= 2
    _compare(b.data, 1, wl, True, zaps=((10, 20), (100, 128)), max_giant_rate=1.0, **kw)


def test_too_few_samples(hdb):
    b = synth.make_c0()
    err, proc, c, g = _run_gpu(b.data[:20000], **_params(synth.SEARCH_C0))
    assert err == H.HD_TOO_FEW_NSAMPS and len(c) == 0


@pytest.mark.parametrize("clean", [False, True])
def test_channel_count_not_whole_words(hdb, clean):
    """8-bit spectra of 130 channels are not whole 32-bit words: rejected
    before any work, and the pipeline still searches a valid gulp after."""
    fb = np.zeros((8192, 130), np.uint8)
    p = H.default_params(nchans=130, dt=655.36e-6, f0=851.0, df=-0.3125, dm_max=300.0,
                         boxcar_max=64, output_dir=None)
    with H.Pipeline(p, cleaning=clean) as pl:
        err, _ = pl.execute(fb, raise_on_error=False)
        assert err == H.HD_INVALID_STRIDE
        err, _, _ = pl.execute_beams([fb, fb], raise_on_error=False)
        assert err == H.HD_INVALID_STRIDE
        assert len(pl.candidates()) == 0
    w = synth.SEARCH_C0
    b = synth.make_c0()
    err, _, c, _ = _run_gpu(b.data, clean=clean, **_params(w))
    assert err == H.HD_NO_ERROR and len(c) >= 3


def test_cand_file_written(hdb, tmp_path):
    b = synth.make_c0()
    p = H.default_params(output_dir=str(tmp_path), spectra_per_second=15625,
                         **_params(synth.SEARCH_C0))
    with H.Pipeline(p, cleaning=True) as pl:
        pl.execute(b.data)
        c = pl.candidates()
    files = list(tmp_path.glob("*.cand"))
    assert len(files) == 1 and files[0].name == "1970-01-01-00:00:00_01.cand"
    assert files[0].read_text().splitlines() == H.cand_lines(c)


@pytest.mark.slow
def test_execute_c1_full(hdb, oracle_lib):
    """Full survey-size gulp with RFI: 1024 channels, 2^18 samples, DM 0-2000,
    boxcars to 4096 (the widest boxcar is time-scrunched)."""
    b = synth.make_c1()
    cands = _compare(b.data, 1, synth.SEARCH_C1, True)
    assert len(cands) >= 20


def test_raw_candidates_match_rows(hdb):
    """hd_get_raw_candidates gives the rows of hd_get_candidates as the
    reference's RawCandidates arrays."""
    import ctypes as C
    w = synth.SEARCH_C0
    b = synth.make_c0()
    with H.Pipeline(H.default_params(output_dir=None, **_params(w)), cleaning=False) as pl:
        pl.execute(b.data)
        rows = pl.candidates()
        n = len(rows)
        assert n >= 3
        arrs = {"peaks": np.zeros(n, np.float32)}
        for k in ("inds", "begins", "ends", "filter_inds", "dm_inds", "members"):
            arrs[k] = np.zeros(n, np.uint64)
        raw = H.RawCandidates(arrs["peaks"].ctypes.data_as(C.POINTER(C.c_float)),
                              *(arrs[k].ctypes.data_as(C.POINTER(C.c_size_t))
                                for k in ("inds", "begins", "ends", "filter_inds", "dm_inds",
                                          "members")))
        cnt = C.c_size_t(n)
        assert H.lib().hd_get_raw_candidates(pl._p, C.byref(raw), C.byref(cnt)) == 0
        assert cnt.value == n
    np.testing.assert_array_equal(arrs["peaks"], rows["snr"])
    for k, f in (("inds", "samp_idx"), ("begins", "begin"), ("ends", "end"),
                 ("filter_inds", "filter"), ("dm_inds", "dm_trial"), ("members", "members")):
        np.testing.assert_array_equal(arrs[k], rows[f])

