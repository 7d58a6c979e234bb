"""CPU tests of the checker: golden vectors, known answers, and bit-exact
agreement with the reference's own stage code rebuilt on Thrust's OpenMP
backend (oracle/_ref, built by `make -C oracle ref`)."""
import os

import numpy as np
import pytest

import oracle
from heimdall_multibeam_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))


def test_dm_list_matches_golden(oracle_lib):
    """Share/dm2000.list: the reference's default setup (1024 ch, 64 us,
    f0 1581.804688 MHz, df -0.390625 MHz, 40 us pulse, tol 1.25, DM 0-2000).
    The shipped list omits the leading DM 0; values compare at the file's
    printed precision (%g)."""
    golden = open(os.path.join(HERE, "golden", "dm2000.list")).read().split()
    dms = oracle.dm_list(0.0, 2000.0, 64e-6, 40.0, 1581.804688, -0.390625, 1024, 1.25)
    assert dms[0] == 0.0
    got = ["%g" % float(x) for x in dms[1:]]
    assert got == golden


def test_medians_known_answers(oracle_lib):
    import itertools
    vals = [1.0, 2.0, 3.0, 4.0, 5.0]
    for p in itertools.permutations(vals):
        assert oracle.median(*p) == 3.0
    for p in itertools.permutations(vals[:4]):
        assert oracle.median(*p) == 2.5
    for p in itertools.permutations(vals[:3]):
        assert oracle.median(*p) == 2.0
    # ties
    assert oracle.median(1.0, 1.0, 2.0, 2.0, 2.0) == 2.0
    assert oracle.median(7.0, 7.0, 7.0, 1.0, 9.0) == 7.0


def test_rng_restatement(oracle_lib):
    """Park-Miller minimal standard: from seed 1 the 10000th output of the
    multiplier-48271 generator is 399268537 (the published check value)."""
    import ctypes as C
    L = oracle.lib()
    s = C.c_uint32(1)
    for _ in range(10000):
        L.or_uniform_uint(C.byref(s), 0, 0)
    assert s.value == 399268537


def test_dedisperse_impulse(oracle_lib):
    """A single-sample broadband impulse dedispersed at its own DM sums all
    channels into one sample."""
    nchans, nsamps = 64, 4096
    table = oracle.delay_table(nchans, 64e-6, 1500.0, -2.0)
    dms = np.array([0.0, 50.0, 100.0], np.float32)
    dl = oracle.delays(dms, table)
    fb = np.zeros((nsamps, nchans), np.uint8)
    t0 = 100
    for c in range(nchans):
        fb[t0 + int(dl[1, c]), c] = 3
    out = oracle.dedisperse(fb, dms, table)
    assert out[1, t0] == 3 * nchans
    assert out[1].sum() == 3 * nchans


def _small_params(w, **kw):
    d = dict(dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min, dm_max=w.dm_max,
             boxcar_max=w.boxcar_max)
    d.update(kw)
    return d


needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference build (oracle/_ref) not present")


@needs_ref
@pytest.mark.parametrize("clean", [0, 1])
def test_oracle_equals_reference_c0(oracle_lib, clean):
    """Whole hd_execute chain on the 256-channel single-beam workload: the C
    restatement writes the same .cand lines as the reference's own pipeline."""
    b = synth.make_c0()
    w = synth.SEARCH_C0
    kw = _small_params(w, clean=clean)
    r = oracle.execute(b.data, **kw)
    lines = oracle.cand_lines(r["groups"], b.data.shape[0], 1, 0, r["nsamps_processed"],
                              w.boxcar_max, w.dt)
    err, proc, ref_lines, _ = oracle.ref_execute(b.data, nthreads=1, **kw)
    assert err == 0 and proc == r["nsamps_processed"]
    assert len(lines) >= 3
    assert lines == ref_lines


@needs_ref
def test_oracle_equals_reference_multibeam(oracle_lib):
    """STF multibeam semantics (per-beam baseline and RMS, shared block RMS,
    beam-window candidate filter) on 4 short beams."""
    w = synth.Workload("mb_small", 64, 655.36e-6, 851.0, -0.390625, 8192, 4, 0.0, 600.0, 256,
                       False, "")
    beams = synth.make_multibeam(w, seed=7, snr_lo=15, snr_hi=30)
    fb = synth.stf(beams)
    kw = _small_params(w, clean=1, baseline_length=1.0)
    r = oracle.execute(fb, nbeams=w.nbeams, **kw)
    lines = oracle.cand_lines(r["groups"], fb.shape[0], w.nbeams, 0, r["nsamps_processed"],
                              w.boxcar_max, w.dt)
    err, proc, ref_lines, _ = oracle.ref_execute(fb, nbeams=w.nbeams, nthreads=1, **kw)
    assert err == 0
    assert lines == ref_lines


@needs_ref
def test_oracle_equals_reference_zaps_and_rate(oracle_lib):
    """Manual channel zaps and the giant-rate bail-out."""
    w = synth.SEARCH_C1
    df = w.df * 8
    pulses = [synth.Pulse(3000.0, 120.0, 1e-3, 25.0), synth.Pulse(9000.0, 400.0, 4e-3, 15.0)]
    b = synth.make_beam(1 << 15, 128, w.dt, w.f0, df, pulses, seed=11, n_bursts=3)
    kw = _small_params(w, df=df, clean=1, dm_max=500.0, boxcar_max=256,
                       channel_zaps=[(10, 20), (100, 128)])
    r = oracle.execute(b.data, **kw)
    lines = oracle.cand_lines(r["groups"], b.data.shape[0], 1, 0, r["nsamps_processed"], 256,
                              w.dt)
    err, proc, ref_lines, _ = oracle.ref_execute(b.data, nthreads=1, **kw)
    assert err == 0 and len(lines) >= 2 and lines == ref_lines
    kw["max_giant_rate"] = 1.0
    r = oracle.execute(b.data, **kw)
    err, proc, ref_lines, _ = oracle.ref_execute(b.data, nthreads=1, **kw)
    assert r["error"] == 12 and err == 12
    assert ref_lines == []


def test_clustering_sequential_semantics(oracle_lib):
    """The fixed sequential sweep differs from connected components: giant 2
    (DM trial 150) is coincident with giants 0 (trial 0) and 1 (trial 300),
    which are not coincident with each other.  When 1 is swept, 2 still holds
    its own label, so 1 stays a root: two groups where connected components
    would give one."""
    import ctypes as C
    L = oracle.lib()
    g = oracle.OrGiants()
    n = 3
    inds = (C.c_size_t * n)(100, 100, 100)
    filt = (C.c_size_t * n)(0, 0, 0)
    dms = (C.c_size_t * n)(0, 300, 150)
    peaks = (C.c_float * n)(7.0, 8.0, 9.0)
    g.count = n
    g.inds = C.cast(inds, C.POINTER(C.c_size_t))
    g.filter_inds = C.cast(filt, C.POINTER(C.c_size_t))
    g.dm_inds = C.cast(dms, C.POINTER(C.c_size_t))
    g.peaks = C.cast(peaks, C.POINTER(C.c_float))
    labels = (C.c_size_t * n)()
    L.or_label_clusters.restype = C.c_size_t
    L.or_label_clusters.argtypes = [C.c_size_t, C.POINTER(oracle.OrGiants), C.c_size_t,
                                    C.c_size_t, C.c_size_t, C.c_size_t, C.POINTER(C.c_size_t)]
    nl = L.or_label_clusters(n, C.byref(g), 3, 3, 200, 1 << 20, labels)
    assert list(labels) == [0, 1, 0] and nl == 2


@needs_ref
def test_oracle_equals_reference_headline_beam(oracle_lib):
    """One beam of the benchmarked multibeam gulp exactly as the benchmark
    draws it (320 channels, 851 MHz top, 655.36 us, 2^15 samples, DM 0-2000,
    boxcars to 512, seed 2026): the restatement writes the reference
    pipeline's .cand lines."""
    w = synth.SEARCH_C2
    beams = synth.make_multibeam(w, seed=2026)
    for u in (0, 17):
        fb = beams[u].data
        kw = _small_params(w, clean=int(w.clean))
        r = oracle.execute(fb, **kw)
        lines = oracle.cand_lines(r["groups"], fb.shape[0], 1, 0, r["nsamps_processed"],
                                  w.boxcar_max, w.dt)
        err, proc, ref_lines, _ = oracle.ref_execute(fb, nthreads=1, **kw)
        assert err == 0 and proc == r["nsamps_processed"]
        assert len(lines) >= 1
        assert lines == ref_lines, u


@needs_ref
def test_oracle_equals_reference_survey_gulp(oracle_lib):
    """The full survey gulp (1024 channels, 2^18 samples, 64 us, boxcars to
    4096, persistent narrow-band channels and zero-DM bursts, cleaning on),
    searched over the DM 240-300 trials of its list (77 of 1482, to keep the
    single-threaded reference stage code within seconds): the same .cand
    lines as the reference."""
    w = synth.SEARCH_C1
    b = synth.make_c1()
    kw = _small_params(w, clean=1, dm_min=240.0, dm_max=300.0)
    r = oracle.execute(b.data, **kw)
    assert r["dm_count"] == 77
    lines = oracle.cand_lines(r["groups"], b.data.shape[0], 1, 0, r["nsamps_processed"],
                              w.boxcar_max, w.dt)
    err, proc, ref_lines, _ = oracle.ref_execute(b.data, nthreads=1, **kw)
    assert err == 0 and proc == r["nsamps_processed"]
    assert len(lines) >= 5
    assert lines == ref_lines


@needs_ref
@pytest.mark.parametrize("case", ["c0", "c0_clean", "headline_beam", "stf4"])
def test_oracle_equals_reference_adaptive_dt(oracle_lib, case):
    """use_scrunching = 1: the reference pipeline's own scrunched path
    (pipeline.cu:489-775 with per-trial factors > 1: scrunched series and
    strides, widths from the factor up, indices rescaled by factor x
    tscrunch) run on the CPU dedisperser with the restated adaptive-dt rule
    writes the same .cand lines as the restatement."""
    if case.startswith("c0"):
        w = synth.SEARCH_C0
        fb, nbeams = synth.make_c0().data, 1
        kw = _small_params(w, clean=int(case == "c0_clean"))
    elif case == "headline_beam":
        w = synth.SEARCH_C2
        fb, nbeams = synth.make_multibeam(w, seed=2026)[0].data, 1
        kw = _small_params(w, clean=0)
    else:
        w = synth.Workload("mb_small", 64, 655.36e-6, 851.0, -0.390625, 8192, 4, 0.0, 600.0,
                           256, False, "")
        fb = synth.stf(synth.make_multibeam(w, seed=7, snr_lo=15, snr_hi=30))
        nbeams = 4
        kw = _small_params(w, clean=1, baseline_length=1.0)
    kw["use_scrunching"] = 1
    r = oracle.execute(fb, nbeams=nbeams, **kw)
    assert int(r["scrunch"].max()) >= 2
    lines = oracle.cand_lines(r["groups"], fb.shape[0], nbeams, 0, r["nsamps_processed"],
                              w.boxcar_max, w.dt)
    err, proc, ref_lines, _ = oracle.ref_execute(fb, nbeams=nbeams, nthreads=1, **kw)
    assert err == 0 and proc == r["nsamps_processed"]
    assert len(lines) >= 3
    assert lines == ref_lines


def test_scrunch_factors_rule(oracle_lib):
    """The restated rule: factors start at 1, never decrease, only double,
    and a trial doubles exactly when the smearing at twice the previous
    sampling time is below tol times that at the previous one."""
    w = synth.SEARCH_C1
    dms = oracle.dm_list(0.0, 2000.0, w.dt, 40.0, w.f0, w.df, w.nchans, 1.25)
    sc = oracle.scrunch_factors(dms, w.dt, 40.0, w.f0, w.df, w.nchans, 1.15).astype(np.int64)
    assert sc[0] == 1 and np.all(np.diff(sc) >= 0)
    assert set(np.unique(sc[1:] // sc[:-1])) <= {1, 2}
    f = (w.f0 + (w.nchans // 2 - 0.5) * w.df) * 1e-3
    a = 8.3 * w.df / f ** 3
    for d in range(1, len(dms)):
        s = sc[d - 1]
        w1 = np.sqrt((s * w.dt * 1e6) ** 2 + 40.0 ** 2 + (a * float(dms[d])) ** 2)
        w2 = np.sqrt((2 * s * w.dt * 1e6) ** 2 + 40.0 ** 2 + (a * float(dms[d])) ** 2)
        assert sc[d] == (2 * s if w2 / w1 < 1.15 else s), d
    assert sc[-1] >= 8
