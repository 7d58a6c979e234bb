"""ctypes front end of the CPU checker (TEST INFRASTRUCTURE ONLY).

Two libraries are wrapped:

* ``_build/liboracle.so`` -- the C restatement in oracle.c of every stage of
  Heimdall's per-gulp chain;
* ``_ref/libhdref.so`` -- the reference's own ``Pipeline/*.cu`` rebuilt on
  Thrust's OpenMP backend (``make -C oracle ref``), driven through its own
  ``hd_create_pipeline`` / ``hd_execute`` (Pipeline/pipeline.cu:138-1087).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU baseline leg import
this package.  The product (heimdall_multibeam_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess
import tempfile
from typing import Dict, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libhdref.so")            # CLEANING defined
REF_NOCLEAN_PATH = os.path.join(HERE, "_ref", "libhdref_noclean.so")

_szp = C.POINTER(C.c_size_t)
_fp = C.POINTER(C.c_float)


class OrParams(C.Structure):
    _fields_ = [
        ("nchans", C.c_size_t),
        ("dt", C.c_float), ("f0", C.c_float), ("df", C.c_float),
        ("dm_min", C.c_float), ("dm_max", C.c_float), ("dm_tol", C.c_float),
        ("dm_pulse_width", C.c_float),
        ("baseline_length", C.c_float),
        ("rfi_tol", C.c_float),
        ("boxcar_max", C.c_size_t),
        ("detect_thresh", C.c_float),
        ("cand_sep_time", C.c_size_t), ("cand_sep_filter", C.c_size_t),
        ("cand_sep_dm", C.c_size_t),
        ("max_giant_rate", C.c_float),
        ("min_tscrunch_width", C.c_size_t),
        ("clean", C.c_int),
        ("num_channel_zaps", C.c_uint),
        ("channel_zaps", _szp),
        ("nthreads", C.c_int),
        ("use_scrunching", C.c_int),
        ("scrunch_tol", C.c_float),
    ]


class OrGiants(C.Structure):
    _fields_ = [("count", C.c_size_t), ("cap", C.c_size_t), ("peaks", _fp),
                ("inds", _szp), ("begins", _szp), ("ends", _szp),
                ("filter_inds", _szp), ("dm_inds", _szp), ("members", _szp)]


class OrResult(C.Structure):
    _fields_ = [("error", C.c_int), ("nsamps_processed", C.c_size_t),
                ("dm_count", C.c_size_t), ("max_delay", C.c_size_t),
                ("giants", OrGiants), ("labels", _szp), ("label_count", C.c_size_t),
                ("groups", OrGiants), ("group_dms", _fp), ("scrunch", _szp)]


DEFAULTS = dict(  # Pipeline/default_params.C:10-66
    nchans=1024, dt=64e-6, f0=1581.804688, df=-0.390625, dm_min=0.0, dm_max=1000.0,
    dm_tol=1.25, dm_pulse_width=40.0, baseline_length=2.0, rfi_tol=5.0, boxcar_max=4096,
    detect_thresh=6.0, cand_sep_time=3, cand_sep_filter=3, cand_sep_dm=200,
    max_giant_rate=0.0, min_tscrunch_width=4096, clean=0, channel_zaps=(), nthreads=0,
    beam=0, use_scrunching=0, scrunch_tol=1.15)

_lib = None
_ref = {}


def build(ref: bool = False) -> None:
    """Compiles the checker (and, with ref=True, the reference build)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref:
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.or_generate_dm_list.restype = C.c_size_t
        L.or_generate_dm_list.argtypes = [C.c_float, C.c_float, C.c_double, C.c_double,
                                          C.c_double, C.c_double, C.c_size_t, C.c_double,
                                          _fp, C.c_size_t]
        L.or_delay_table.argtypes = [C.c_size_t, C.c_float, C.c_float, C.c_float, _fp]
        L.or_max_delay.restype = C.c_size_t
        L.or_max_delay.argtypes = [_fp, C.c_size_t, _fp, C.c_size_t]
        L.or_dedisperse.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t,
                                    C.c_void_p, _fp, C.c_size_t, _fp, _fp, C.c_size_t, C.c_int]
        L.or_dedisperse_scrunched.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t,
                                              C.c_void_p, _fp, C.c_size_t, _fp, _szp, _fp,
                                              C.c_size_t, C.c_int]
        L.or_scrunch_factors.argtypes = [_fp, C.c_size_t, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_size_t, C.c_double, _szp]
        for n in ("or_median3", "or_median4", "or_median5"):
            getattr(L, n).restype = C.c_float
        L.or_median3.argtypes = [C.c_float] * 3
        L.or_median4.argtypes = [C.c_float] * 4
        L.or_median5.argtypes = [C.c_float] * 5
        L.or_hd_execute.argtypes = [C.POINTER(OrParams), C.c_void_p, C.c_size_t, C.c_size_t,
                                    C.c_size_t, C.c_size_t, C.POINTER(OrResult)]
        L.or_result_free.argtypes = [C.POINTER(OrResult)]
        L.or_clean_filterbank_rfi.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t,
                                              C.c_float, C.c_float, C.c_float, C.c_size_t,
                                              C.c_size_t, C.c_void_p, C.c_void_p]
        L.or_hash.restype = C.c_uint32
        L.or_hash.argtypes = [C.c_uint32]
        L.or_uniform_uint.restype = C.c_uint32
        L.or_uniform_uint.argtypes = [C.POINTER(C.c_uint32), C.c_uint32, C.c_uint32]
        L.or_rms_block.restype = C.c_float
        L.or_rms_block.argtypes = [_fp, C.c_size_t, C.c_size_t, C.c_size_t]
        L.or_rms_beams.argtypes = [_fp, _fp, C.c_size_t, C.c_size_t, C.c_size_t]
        L.or_remove_baseline.argtypes = [_fp, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t,
                                         C.c_size_t]
        L.or_baseline_plan.argtypes = [C.c_size_t, C.c_size_t, _szp, _szp, _szp]
        L.or_exclusive_scan.argtypes = [_fp, C.c_size_t, _fp]
        L.or_linear_stretch.argtypes = [_fp, C.c_size_t, _fp, C.c_size_t]
        L.or_set_scan_capture.argtypes = [C.c_void_p, C.c_size_t]
        L.or64_giant_snr.restype = C.c_int
        L.or64_giant_snr.argtypes = [C.POINTER(OrParams), C.c_void_p, C.c_size_t, C.c_size_t,
                                     C.c_size_t, _szp, _szp, _szp, C.POINTER(C.c_double)]
        L.or_normalise_rows.argtypes = [_fp, C.c_size_t, C.c_size_t]
        L.or_patch_dm.argtypes = [_fp, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t,
                                  C.c_size_t, C.c_size_t, _fp]
        L.or_patch_ft.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t,
                                  C.c_size_t, _fp]
        L.or_cnn_param_count.restype = C.c_size_t
        L.or_bf16.restype = C.c_float
        L.or_bf16.argtypes = [C.c_float]
        L.or_cnn_run.argtypes = [_fp, _fp, _fp, C.c_void_p, C.c_size_t, _fp, _fp, _fp]
        L.or_measure_bandpass.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, _fp, _fp]
        L.or_narrow_band.restype = C.c_int
        L.or_narrow_band.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_float, C.c_float,
                                     C.c_float]
        L.or_set_narrow_band.argtypes = [C.c_int]
        _lib = L
    return _lib


def reference_dir() -> str:
    """Where the reference tree lies: HEIMDALL_REFERENCE, else the location
    the build recipe (oracle/Makefile REF) reads by default."""
    return os.environ.get("HEIMDALL_REFERENCE", "/root/reference")


def ref_available() -> bool:
    return os.path.exists(REF_PATH) and os.path.exists(REF_NOCLEAN_PATH)


def ref_lib(clean: bool = True):
    path = REF_PATH if clean else REF_NOCLEAN_PATH
    if path not in _ref:
        if not os.path.exists(path):
            raise FileNotFoundError(
                "reference build missing: run `make -C oracle ref` where the reference "
                "sources are present")
        R = C.CDLL(path)
        R.ref_execute.restype = C.c_int
        R.ref_execute.argtypes = [C.POINTER(OrParams), C.c_void_p, C.c_size_t, C.c_size_t,
                                  C.c_size_t, C.c_size_t, C.c_char_p, _szp,
                                  C.POINTER(C.c_double), C.c_int]
        R.ref_measure_bandpass.restype = C.c_int
        R.ref_measure_bandpass.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, _fp, _fp]
        R.ref_narrow_band.restype = C.c_int
        R.ref_narrow_band.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_float, C.c_float,
                                      C.c_float]
        R.dedisp_cpu_set_threads.restype = None
        R.dedisp_cpu_set_threads.argtypes = [C.c_int]
        _ref[path] = R
    return _ref[path]


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def make_params(**kw) -> OrParams:
    d = dict(DEFAULTS)
    d.update(kw)
    p = OrParams()
    for name, _ in OrParams._fields_:
        if name in ("channel_zaps", "num_channel_zaps"):
            continue
        setattr(p, name, d[name])
    zaps = np.asarray(d.get("channel_zaps") or [], dtype=np.uintp).reshape(-1)
    p._zaps = np.ascontiguousarray(zaps, dtype=np.uint64)
    p.num_channel_zaps = len(zaps) // 2
    p.channel_zaps = p._zaps.ctypes.data_as(_szp) if len(zaps) else None
    return p


# ---------------------------------------------------------------- stages
def dm_list(dm_start, dm_end, dt, ti, f0, df, nchans, tol) -> np.ndarray:
    L = lib()
    n = L.or_generate_dm_list(dm_start, dm_end, dt, ti, f0, df, nchans, tol, None, 0)
    out = np.zeros(n, np.float32)
    L.or_generate_dm_list(dm_start, dm_end, dt, ti, f0, df, nchans, tol, _fptr(out), n)
    return out


def delay_table(nchans, dt, f0, df) -> np.ndarray:
    out = np.zeros(nchans, np.float32)
    lib().or_delay_table(nchans, dt, f0, df, _fptr(out))
    return out


def delays(dms: np.ndarray, table: np.ndarray) -> np.ndarray:
    """delay(d, c) = (size_t)(dm * table[c] + 0.5f), float arithmetic."""
    v = np.float32(dms)[:, None] * np.float32(table)[None, :] + np.float32(0.5)
    return np.where(v > 0, v, 0).astype(np.uint64)


def scrunch_factors(dms, dt, ti, f0, df, nchans, tol) -> np.ndarray:
    """Per-trial scrunch factors of adaptive dt (or_scrunch_factors)."""
    dms = np.ascontiguousarray(dms, np.float32)
    out = np.zeros(len(dms), np.uint64)
    lib().or_scrunch_factors(_fptr(dms), len(dms), dt, ti, f0, df, nchans, tol,
                             out.ctypes.data_as(_szp))
    return out


def dedisperse_scrunched(fb: np.ndarray, dms: np.ndarray, table: np.ndarray,
                         scrunch: np.ndarray, killmask: Optional[np.ndarray] = None,
                         nthreads: int = 0) -> List[np.ndarray]:
    """Dedispersion with per-trial scrunch factors: row d holds
    (nsamps - max_delay) // scrunch[d] samples."""
    fb = np.ascontiguousarray(fb, dtype=np.uint8)
    nsamps, nchans = fb.shape
    dms = np.ascontiguousarray(dms, np.float32)
    table = np.ascontiguousarray(table, np.float32)
    sc = np.ascontiguousarray(scrunch, np.uint64)
    km = np.ones(nchans, np.int32) if killmask is None else np.ascontiguousarray(killmask, np.int32)
    md = lib().or_max_delay(_fptr(dms), len(dms), _fptr(table), nchans)
    nout = nsamps - md
    out = np.zeros((len(dms), nout), np.float32)
    lib().or_dedisperse_scrunched(fb.ctypes.data, nsamps, nchans, nchans, km.ctypes.data,
                                  _fptr(dms), len(dms), _fptr(table), sc.ctypes.data_as(_szp),
                                  _fptr(out), nout, nthreads)
    return [out[d, : nout // int(sc[d])].copy() for d in range(len(dms))]


def dedisperse(fb: np.ndarray, dms: np.ndarray, table: np.ndarray,
               killmask: Optional[np.ndarray] = None, nthreads: int = 0) -> np.ndarray:
    fb = np.ascontiguousarray(fb, dtype=np.uint8)
    nsamps, nchans = fb.shape
    dms = np.ascontiguousarray(dms, np.float32)
    table = np.ascontiguousarray(table, np.float32)
    km = np.ones(nchans, np.int32) if killmask is None else np.ascontiguousarray(killmask, np.int32)
    md = lib().or_max_delay(_fptr(dms), len(dms), _fptr(table), nchans)
    nout = nsamps - md
    out = np.zeros((len(dms), nout), np.float32)
    lib().or_dedisperse(fb.ctypes.data, nsamps, nchans, nchans, km.ctypes.data, _fptr(dms),
                        len(dms), _fptr(table), _fptr(out), nout, nthreads)
    return out


def median(*v) -> float:
    L = lib()
    return {3: L.or_median3, 4: L.or_median4, 5: L.or_median5}[len(v)](*[float(x) for x in v])


def clean_filterbank(fb: np.ndarray, dt: float, baseline_length=2.0, rfi_tol=5.0,
                     nbeams: int = 1, boxcar_max: int = 64):
    fb = np.ascontiguousarray(fb, dtype=np.uint8)
    nsamps, nchans = fb.shape
    out = np.zeros_like(fb)
    mask = np.zeros(nsamps, np.int32)
    rc = lib().or_clean_filterbank_rfi(fb.ctypes.data, nsamps, 8, nchans, dt, baseline_length,
                                       rfi_tol, boxcar_max, nbeams, out.ctypes.data,
                                       mask.ctypes.data)
    if rc != 0:
        raise ValueError("resample radius not below nsamps")
    return out, mask


# ---------------------------------------------------------------- chain
def _giants_to_dict(g: OrGiants) -> Dict[str, np.ndarray]:
    n = g.count

    def arr(p, dt):
        if n == 0:
            return np.zeros(0, dt)
        return np.ctypeslib.as_array(p, shape=(n,)).astype(dt).copy()
    return dict(peaks=arr(g.peaks, np.float32), inds=arr(g.inds, np.uint64),
                begins=arr(g.begins, np.uint64), ends=arr(g.ends, np.uint64),
                filter_inds=arr(g.filter_inds, np.uint64), dm_inds=arr(g.dm_inds, np.uint64),
                members=arr(g.members, np.uint64))


def execute(fb: np.ndarray, nbeams: int = 1, first_idx: int = 0, **kw) -> dict:
    """Whole hd_execute chain on one gulp (STF layout for nbeams > 1)."""
    fb = np.ascontiguousarray(fb, dtype=np.uint8)
    nsamps, nchans = fb.shape
    p = make_params(nchans=nchans, **kw)
    res = OrResult()
    lib().or_hd_execute(C.byref(p), fb.ctypes.data, nsamps, 8, first_idx, nbeams, C.byref(res))
    out = dict(error=res.error, nsamps_processed=res.nsamps_processed, dm_count=res.dm_count,
               max_delay=res.max_delay, giants=_giants_to_dict(res.giants),
               label_count=res.label_count)
    G = res.giants.count
    out["labels"] = (np.ctypeslib.as_array(res.labels, shape=(G,)).astype(np.uint64).copy()
                     if res.labels and G else np.zeros(0, np.uint64))
    grp = _giants_to_dict(res.groups) if res.labels else _giants_to_dict(OrGiants())
    L = len(grp["peaks"])
    grp["dms"] = (np.ctypeslib.as_array(res.group_dms, shape=(L,)).astype(np.float32).copy()
                  if L else np.zeros(0, np.float32))
    out["groups"] = grp
    D = res.dm_count
    out["scrunch"] = (np.ctypeslib.as_array(res.scrunch, shape=(D,)).astype(np.uint64).copy()
                      if res.scrunch and D else np.ones(D, np.uint64))
    lib().or_result_free(C.byref(res))
    return out


def cand_lines(groups: dict, nsamps: int, nbeams: int, first_idx: int,
               nsamps_processed: int, boxcar_max: int, dt: float, beam: int = 0) -> List[str]:
    """The .cand lines Pipeline/pipeline.cu:1012-1039 writes for these groups."""
    lines = []
    nsamps_beam = np.uint32(nsamps // nbeams)
    nsamps_valid = np.uint32(nsamps_processed // nbeams)
    dtf = np.float32(dt)
    for i in range(len(groups["peaks"])):
        ind = int(groups["inds"][i])
        beam_idx = int(np.floor(np.float32(ind) / np.float32(nsamps_beam)))
        beam_start = beam_idx * int(nsamps_beam) + boxcar_max // 2
        beam_end = beam_start + int(nsamps_valid)
        if not (beam_start <= ind < beam_end):
            continue
        samp_idx = first_idx + (ind - int(nsamps_beam) * beam_idx)
        peak = np.float32(groups["peaks"][i])
        snr = 0.0 if np.isinf(peak) else float(peak)
        t = float(dtf * np.float32(samp_idx))
        lines.append("%g\t%d\t%g\t%d\t%d\t%g\t%d\t%d\t%d\t%d\t" % (
            snr, samp_idx, t, int(groups["filter_inds"][i]), int(groups["dm_inds"][i]),
            float(groups["dms"][i]), int(groups["members"][i]),
            first_idx + int(groups["begins"][i]) % int(nsamps_beam),
            first_idx + int(groups["ends"][i]) % int(nsamps_beam), beam + beam_idx + 1))
    return lines


def ref_set_dedisp_threads(n: int) -> None:
    """Threads of the CPU dedisperser the reference pipeline links
    (0: every host core), for both reference builds."""
    for clean in (True, False):
        ref_lib(clean).dedisp_cpu_set_threads(int(n))


def ref_execute(fb: np.ndarray, nbeams: int = 1, first_idx: int = 0, nthreads: int = 1,
                nbits: int = 8, nchans: Optional[int] = None, **kw):
    """Runs the reference's own pipeline (the CLEANING build when kw clean=1,
    the shipped build otherwise); returns (error, nsamps_processed, .cand
    lines, seconds).  nthreads=1 fixes the order of the reference's racy
    clustering sweep (Pipeline/label_candidate_clusters.cu:179-195).  With
    nbits != 8, fb holds one row of packed samples per spectrum and nchans
    is given."""
    if nbits == 8:
        fb = np.ascontiguousarray(fb, dtype=np.uint8)
        nsamps, nchans = fb.shape
    else:
        fb = np.ascontiguousarray(fb)
        nsamps = fb.shape[0]
    p = make_params(nchans=nchans, **kw)
    with tempfile.TemporaryDirectory() as d:
        proc = C.c_size_t(0)
        secs = C.c_double(0)
        err = ref_lib(bool(kw.get("clean", 0))).ref_execute(C.byref(p), fb.ctypes.data, nsamps, nbits, first_idx, nbeams,
                                    d.encode(), C.byref(proc), C.byref(secs), nthreads)
        lines: List[str] = []
        for f in sorted(glob.glob(os.path.join(d, "*.cand"))):
            with open(f) as fh:
                lines += [ln.rstrip("\n") for ln in fh if ln.strip()]
    return err, proc.value, lines, secs.value


# ---------------------------------------------------------------------------
# Classifier restatement (oracle/classifier.c)
# ---------------------------------------------------------------------------
def execute_with_scans(fb: np.ndarray, nbeams: int = 1, **kw):
    """execute() that also returns every DM trial's prefix sum
    ([dm_count, nc + 1] float32, nc = nsamps - max_delay)."""
    fb = np.ascontiguousarray(fb, dtype=np.uint8)
    nsamps, nchans = fb.shape
    okw = {k: v for k, v in kw.items() if k not in ("output_dir",)}
    dms = dm_list(okw.get("dm_min", 0.0), okw.get("dm_max", 1000.0), okw.get("dt", 64e-6),
                  okw.get("dm_pulse_width", 40.0), okw.get("f0", 1400.0), okw.get("df", -0.39),
                  nchans, okw.get("dm_tol", 1.25))
    table = delay_table(nchans, okw.get("dt", 64e-6), okw.get("f0", 1400.0), okw.get("df", -0.39))
    md = int(lib().or_max_delay(_fptr(dms), len(dms), _fptr(table), nchans))
    pitch = nsamps - md + 8
    scans = np.zeros((len(dms), pitch), np.float32)
    lib().or_set_scan_capture(scans.ctypes.data, pitch)
    try:
        r = execute(fb, nbeams=nbeams, **okw)
    finally:
        lib().or_set_scan_capture(None, 0)
    return r, scans[:, :nsamps - md + 1], dms, table


def giant_snr_fp64(fb: np.ndarray, dm_inds, filter_inds, inds, nbeams: int = 1,
                   **kw) -> np.ndarray:
    """S/N of the given giants (DM trial, filter index, giant sample index as
    execute() reports them in "groups"/"giants") from the same chain with
    every value held in double (snr64.c)."""
    fb = np.ascontiguousarray(fb, dtype=np.uint8)
    nsamps, nchans = fb.shape
    okw = {k: v for k, v in kw.items() if k not in ("output_dir",)}
    p = make_params(nchans=nchans, **okw)
    d = np.ascontiguousarray(dm_inds, dtype=np.uint64)
    f = np.ascontiguousarray(filter_inds, dtype=np.uint64)
    i = np.ascontiguousarray(inds, dtype=np.uint64)
    n = len(d)
    assert len(f) == n and len(i) == n
    out = np.zeros(max(n, 1), np.float64)
    err = lib().or64_giant_snr(C.byref(p), fb.ctypes.data, nsamps, nbeams, n,
                               d.ctypes.data_as(_szp), f.ctypes.data_as(_szp),
                               i.ctypes.data_as(_szp),
                               out.ctypes.data_as(C.POINTER(C.c_double)))
    if err:
        raise RuntimeError(f"or64_giant_snr failed ({err})")
    return out[:n]


def normalise_rows(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32).copy()
    lib().or_normalise_rows(_fptr(a), a.shape[-1], a.size // a.shape[-1])
    return a


def patch_dm(scans: np.ndarray, dm: int, ind: int, filt: int) -> np.ndarray:
    scans = np.ascontiguousarray(scans, dtype=np.float32)
    out = np.zeros((64, 64), np.float32)
    lib().or_patch_dm(_fptr(scans), scans.shape[1], scans.shape[1] - 1, scans.shape[0], dm, ind,
                      filt, _fptr(out))
    return out


def patch_ft(fb: np.ndarray, max_delay: int, ind: int, filt: int) -> np.ndarray:
    fb = np.ascontiguousarray(fb, dtype=np.uint8)
    out = np.zeros((64, 256), np.float32)
    lib().or_patch_ft(fb.ctypes.data, fb.shape[0], fb.shape[1], max_delay, ind, filt, _fptr(out))
    return out


def cnn_param_count() -> int:
    return int(lib().or_cnn_param_count())


def cnn_run(params: np.ndarray, dm_time: np.ndarray, freq_time: np.ndarray, labels=None):
    """(probabilities, gradients or None, loss or None) of the CPU network."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    dm_time = np.ascontiguousarray(dm_time, dtype=np.float32)
    freq_time = np.ascontiguousarray(freq_time, dtype=np.float32)
    n = dm_time.shape[0]
    probs = np.zeros(n, np.float32)
    grads = loss = None
    if labels is not None:
        labels = np.ascontiguousarray(labels, dtype=np.int32)
        grads = np.zeros_like(params)
        lossv = np.zeros(1, np.float32)
        lib().or_cnn_run(_fptr(params), _fptr(dm_time), _fptr(freq_time), labels.ctypes.data, n,
                         _fptr(probs), _fptr(grads), _fptr(lossv))
        loss = float(lossv[0])
    else:
        lib().or_cnn_run(_fptr(params), _fptr(dm_time), _fptr(freq_time), None, n, _fptr(probs),
                         None, None)
    return probs, grads, loss


# ---------------------------------------------------------------------------
# Sigproc input and the gulp loop (Applications/heimdall.C:153-292)
# ---------------------------------------------------------------------------
def ref_sigproc_dump(path: str, mjds=()) -> dict:
    """The reference's own header reader (Formats/hd/header.h:133-198) and
    mjd2utctm (Formats/hd/DataSource.h:49-82), run through
    _ref/sigproc_dump (built from the reference's headers)."""
    import json
    import subprocess
    exe = os.path.join(HERE, "_ref", "sigproc_dump")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    r = subprocess.run([exe, path] + ["%.17g" % m for m in mjds], capture_output=True,
                       text=True, check=True)
    return json.loads(r.stdout)


def ref_sigproc_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "sigproc_dump"))


def gulp_plan(nsamps_file: int, nsamps_gulp: int, overlap: int):
    """heimdall.C's loop on one beam as a list of (first spectrum of the file
    in the gulp, spectra in the gulp, first_idx): the first gulp is the first
    block; after a gulp of n spectra the pipeline processes n - overlap
    (overlap = boxcar_max + max_delay), which the next gulp carries in front
    of the next block; a block shorter than nsamps_gulp ends the loop
    unsearched."""
    plan = []
    if nsamps_file < nsamps_gulp:
        return plan
    start, n, total = 0, nsamps_gulp, 0
    block = 0
    while True:
        plan.append((start, n, total))
        processed = n - overlap if n > overlap else 0
        carry = n - processed
        total += processed
        block += 1
        if (block + 1) * nsamps_gulp > nsamps_file:
            break
        start = block * nsamps_gulp - carry
        n = carry + nsamps_gulp
    return plan


# ---------------------------------------------------------------------------
# Cross-beam coincidence (Applications/Candidates.C)
# ---------------------------------------------------------------------------
def coincide(beams, sep_time: int, sep_filter: int):
    """compute_coincidence (Candidates.C:236-291) with is_coincident (64-77):
    beams is one list of candidate dicts (snr, samp_idx, filter, dm_trial,
    beam) per beam in list order; returns per beam the list of (nbeams,
    primary_beam, max_snr).  S/N arithmetic in float32 as the reference's."""
    f32 = np.float32
    out = []
    for i, bi in enumerate(beams):
        res = []
        for cj in bi:
            nb, prim, best = 1, int(cj["beam"]), f32(cj["snr"])
            for k, bk in enumerate(beams):
                if k == i:
                    continue
                for cl in bk:
                    fmax = max(int(cl["filter"]), int(cj["filter"]))
                    tol = int(f32(sep_time) * f32(2.0 ** fmax))
                    if abs(int(cl["samp_idx"]) - int(cj["samp_idx"])) > tol:
                        continue
                    if abs(int(cl["dm_trial"]) - int(cj["dm_trial"])) > 9999:
                        continue
                    if abs(int(cl["filter"]) - int(cj["filter"])) > sep_filter:
                        continue
                    a, b = f32(cl["snr"]), f32(cj["snr"])
                    if not (f32(abs(f32(a - b))) / f32(a + b) <= f32(0.4)):
                        continue
                    nb += 1
                    if a > best:
                        prim, best = int(cl["beam"]), a
                    break
            res.append((nb, prim, best))
        out.append(res)
    return out


def ref_coinc_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "coinc_ref"))


def ref_coincide(files, nbeams: int, sep_time: int, sep_filter: int) -> List[str]:
    """The reference's coincidencer (Candidates.C, _ref/coinc_ref) on .cand
    files that sit in one directory; returns the lines of the _all.cand it
    writes there."""
    exe = os.path.join(HERE, "_ref", "coinc_ref")
    d = os.path.dirname(os.path.abspath(files[0]))
    names = [os.path.basename(f) for f in files]
    subprocess.run([exe, str(nbeams), str(sep_time), str(sep_filter)] + names, cwd=d,
                   check=True, capture_output=True)
    out = os.path.join(d, names[0].split("_")[0] + "_all.cand")
    with open(out) as f:
        return f.read().splitlines()


# ---------------------------------------------------------------------------
# Narrow-band RFI (the branch Pipeline/clean_filterbank_rfi.cu:303 disables)
# ---------------------------------------------------------------------------
def measure_bandpass(fb: np.ndarray, ref: bool = False):
    """(bandpass [nchans], rms) of an 8-bit (nsamps, nchans) filterbank:
    the restatement, or (ref=True) the reference's own measure_bandpass."""
    fb = np.ascontiguousarray(fb, dtype=np.uint8)
    nsamps, nchans = fb.shape
    bp = np.zeros(nchans, np.float32)
    rms = np.zeros(1, np.float32)
    if ref:
        ref_lib().ref_measure_bandpass(fb.ctypes.data, nsamps, nchans, _fptr(bp), _fptr(rms))
    else:
        lib().or_measure_bandpass(fb.ctypes.data, nsamps, nchans, _fptr(bp), _fptr(rms))
    return bp, float(rms[0])


def narrow_band(fb: np.ndarray, dt: float, baseline_length: float = 2.0, rfi_tol: float = 5.0,
                ref: bool = False) -> np.ndarray:
    """The narrow-band zapping of an 8-bit filterbank (a copy): the
    restatement, or (ref=True) the reference's own code in index order."""
    out = np.ascontiguousarray(fb, dtype=np.uint8).copy()
    nsamps, nchans = out.shape
    f = ref_lib().ref_narrow_band if ref else lib().or_narrow_band
    if f(out.ctypes.data, nsamps, nchans, dt, baseline_length, rfi_tol) != 0:
        raise ValueError("narrow-band zapping needs nchans a multiple of 4, >= 20")
    return out


def set_narrow_band(enable: bool) -> None:
    """Whether the oracle's cleaning runs the narrow-band branch first."""
    lib().or_set_narrow_band(1 if enable else 0)



# ---------------------------------------------------------------------------
# Candidate profiler restatement (oracle/profiler.c) and the reference's own
# application (oracle/_ref/ref_profiler)
# ---------------------------------------------------------------------------
REF_PROFILER = os.path.join(HERE, "_ref", "ref_profiler")


def profile(fb: np.ndarray, tsamp: float, fch1: float, foff: float, dm_list, samp: int,
            filt: int, dm_idx: int, out_nsamps: int, out_dm_count: int, fscrunch: int,
            do_filter: bool = False) -> dict:
    """or_profile: the candidate profiler's plots and extractions."""
    L = lib()
    fb = np.ascontiguousarray(fb, dtype=np.uint8)
    nsamps, nchans = fb.shape
    dms = np.ascontiguousarray(dm_list, np.float32)
    dm_time = np.zeros((out_dm_count, out_nsamps), np.float32)
    dm0 = np.zeros(out_nsamps, np.float32)
    ft = np.zeros((nchans // fscrunch, out_nsamps), np.float32)
    snr_dm = np.zeros(out_dm_count, np.float32)
    snr_time = np.zeros((out_nsamps, 5), np.float32)
    mx = C.c_size_t(0)
    first = C.c_size_t(0)
    L.or_profile.restype = C.c_size_t
    L.or_profile.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_double, C.c_double,
                             C.c_double, _fp, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t,
                             C.c_size_t, C.c_size_t, C.c_size_t, C.c_int, _fp, _fp, _fp, _szp,
                             _szp, _fp, _fp]
    n = L.or_profile(fb.ctypes.data, nsamps, nchans, tsamp, fch1, foff, _fptr(dms), len(dms),
                     samp, filt, dm_idx, out_nsamps, out_dm_count, fscrunch, int(do_filter),
                     _fptr(dm_time), _fptr(dm0), _fptr(ft), C.byref(mx), C.byref(first),
                     _fptr(snr_dm), _fptr(snr_time))
    return dict(n_dm=int(n), dm_time=dm_time, dm0_time=dm0, freq_time=ft, max_idx=mx.value,
                snr_dm_first=first.value, snr_dm=snr_dm, snr_time=snr_time)


def ref_profiler_available() -> bool:
    return os.path.exists(REF_PROFILER)


def ref_profile(path: str, dm_list, samp: int, filt: int, dm_idx: int, out_nsamps: int,
                out_dm_count: int, fscrunch: int, do_filter: bool = False) -> dict:
    """Runs the reference's candidate_profiler on a sigproc file; returns the
    text of the files it writes (freq_time.dat, snr_dm.dat, snr_time.dat,
    dm_time.pgm) as lists of lines."""
    with tempfile.TemporaryDirectory() as d:
        dml = os.path.join(d, "dm.list")
        with open(dml, "w") as f:
            for v in np.asarray(dm_list, np.float32):
                f.write("%.9g\n" % float(v))
        args = [REF_PROFILER, os.path.abspath(path), dml, str(samp), str(filt), str(dm_idx),
                str(out_nsamps), str(out_dm_count), str(fscrunch), str(int(do_filter))]
        subprocess.run(args, cwd=d, check=True, capture_output=True)
        out = {}
        for name in ("freq_time.dat", "snr_dm.dat", "snr_time.dat", "dm_time.pgm"):
            p = os.path.join(d, name)
            out[name] = open(p).read().splitlines() if os.path.exists(p) else None
    return out
