"""heimdall_multibeam_b200 -- Heimdall's per-gulp single-pulse search on B200.

Python face of ``libhdb200.so``, the C library whose interface
(``include/heimdall_b200.h``, ``include/dedisp.h``) replaces the reference's
``hd_*`` pipeline API (Pipeline/hd/pipeline.h:10-28) and the ``dedisp_*`` calls
it makes.  Everything here is a thin ctypes binding: the computation runs in
the sm_100a kernels of ``csrc/``.  There is no CPU fallback: if the library is
missing or no GPU is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhdb200.so")

# ---- error codes (Pipeline/hd/error.h:19-39) ------------------------------
HD_NO_ERROR = 0
HD_MEM_ALLOC_FAILED = 1
HD_MEM_COPY_FAILED = 2
HD_INVALID_DEVICE_INDEX = 3
HD_DEVICE_ALREADY_SET = 4
HD_INVALID_PIPELINE = 5
HD_INVALID_POINTER = 6
HD_INVALID_STRIDE = 7
HD_INVALID_NBITS = 8
HD_PRIOR_GPU_ERROR = 9
HD_INTERNAL_GPU_ERROR = 10
HD_TOO_FEW_NSAMPS = 11
HD_TOO_MANY_EVENTS = 12
HD_UNKNOWN_ERROR = 13

# fixed scratch limits of hd_clean_filterbank_rfi_noalloc (include/heimdall_b200.h)
HD_NOALLOC_MAX_NSAMPS = 524288
HD_NOALLOC_MAX_BEAMS = 64

DEDISP_NO_ERROR = 0
DEDISP_DEVICE_POINTERS = 1 << 2


class HdError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = code
        super().__init__(f"{where}: {error_string(code)} (hd_error {code})")


class HdRange(C.Structure):
    _fields_ = [("start", C.c_size_t), ("end", C.c_size_t)]


class HdParams(C.Structure):
    """struct hd_params (Pipeline/hd/params.h:19-78), built without HAVE_PSRDADA."""
    _fields_ = [
        ("verbosity", C.c_int),
        ("sigproc_file", C.c_char_p),
        ("yield_cpu", C.c_bool),
        ("nsamps_gulp", C.c_size_t),
        ("dm_gulp_size", C.c_size_t),
        ("baseline_length", C.c_float),
        ("beam", C.c_size_t),
        ("nbeams", C.c_size_t),
        ("override_beam", C.c_bool),
        ("nchans", C.c_size_t),
        ("dt", C.c_float),
        ("f0", C.c_float),
        ("df", C.c_float),
        ("dm_min", C.c_float),
        ("dm_max", C.c_float),
        ("dm_tol", C.c_float),
        ("dm_pulse_width", C.c_float),
        ("dm_nbits", C.c_size_t),
        ("use_scrunching", C.c_bool),
        ("scrunch_tol", C.c_float),
        ("rfi_tol", C.c_float),
        ("rfi_min_beams", C.c_size_t),
        ("boxcar_max", C.c_size_t),
        ("detect_thresh", C.c_float),
        ("cand_sep_time", C.c_size_t),
        ("cand_sep_filter", C.c_size_t),
        ("cand_sep_dm", C.c_size_t),
        ("cand_rfi_dm_cut", C.c_size_t),
        ("max_giant_rate", C.c_float),
        ("min_tscrunch_width", C.c_size_t),
        ("coincidencer_host", C.c_char_p),
        ("coincidencer_port", C.c_int),
        ("num_channel_zaps", C.c_uint),
        ("channel_zaps", C.POINTER(HdRange)),
        ("beam_count", C.c_size_t),
        ("gpu_id", C.c_int),
        ("utc_start", C.c_long),
        ("spectra_per_second", C.c_size_t),
        ("output_dir", C.c_char_p),
    ]


class HdCandidate(C.Structure):
    _fields_ = [("snr", C.c_float), ("samp_idx", C.c_size_t), ("time", C.c_float),
                ("filter", C.c_size_t), ("dm_trial", C.c_size_t), ("dm", C.c_float),
                ("members", C.c_size_t), ("begin", C.c_size_t), ("end", C.c_size_t),
                ("beam", C.c_size_t)]


CANDIDATE_DTYPE = np.dtype([("snr", "<f4"), ("samp_idx", "<u8"), ("time", "<f4"),
                            ("filter", "<u8"), ("dm_trial", "<u8"), ("dm", "<f4"),
                            ("members", "<u8"), ("begin", "<u8"), ("end", "<u8"),
                            ("beam", "<u8")], align=True)

class HdSigprocHeader(C.Structure):
    """hd_sigproc_header (include/heimdall_b200.h)."""
    _fields_ = [("source_name", C.c_char * 80), ("rawdatafile", C.c_char * 80)] + \
        [(k, C.c_double) for k in ("az_start", "za_start", "src_raj", "src_dej", "tstart", "tsamp",
                                   "period", "fch1", "foff", "refdm")] + \
        [(k, C.c_int) for k in ("nchans", "telescope_id", "machine_id", "data_type", "ibeam",
                                "nbeams", "nbits", "barycentric", "pulsarcentric", "nbins",
                                "nsamples", "nifs", "npuls")] + \
        [("signed_data", C.c_ubyte), ("size", C.c_int), ("unknown_keys", C.c_int)]

    def as_dict(self) -> Dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["source_name"] = self.source_name.decode()
        d["rawdatafile"] = self.rawdatafile.decode()
        return d


GULP_CALLBACK = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t)


class RawCandidates(C.Structure):
    """struct RawCandidates (Pipeline/hd/types.h:18-26)."""
    _fields_ = [("peaks", C.POINTER(C.c_float))] + \
        [(k, C.POINTER(C.c_size_t)) for k in ("inds", "begins", "ends", "filter_inds",
                                              "dm_inds", "members")]


class HdCoincidence(C.Structure):
    """hd_coincidence (include/heimdall_b200.h)."""
    _fields_ = [("nbeams", C.c_uint), ("primary_beam", C.c_uint), ("max_snr", C.c_float)]


class HdProfileRequest(C.Structure):
    """hd_profile_request (include/heimdall_b200.h)."""
    _fields_ = [("samp", C.c_size_t), ("filter", C.c_size_t), ("dm_idx", C.c_size_t)]


class HdProfile(C.Structure):
    """hd_profile (include/heimdall_b200.h)."""
    _fields_ = [("dm_time", C.c_void_p), ("dm0_time", C.c_void_p), ("freq_time", C.c_void_p),
                ("snr_dm", C.c_void_p), ("snr_time", C.c_void_p), ("max_idx", C.c_size_t),
                ("n_dm", C.c_size_t), ("dm_begin", C.c_size_t), ("snr_dm_first", C.c_size_t)]


# symbol -> (restype, argtypes); every function include/*.h declares
_P = C.c_void_p
_SZ = C.c_size_t
_SZP = C.POINTER(C.c_size_t)
_FP = C.POINTER(C.c_float)
SYMBOLS = {
    "hd_get_error_string": (C.c_char_p, [C.c_int]),
    "hd_set_default_params": (None, [C.POINTER(HdParams)]),
    "hd_parse_command_line": (C.c_int, [C.c_int, C.POINTER(C.c_char_p), C.POINTER(HdParams)]),
    "hd_print_usage": (None, []),
    "hd_create_pipeline": (C.c_int, [C.POINTER(_P), HdParams]),
    "hd_preallocate": (C.c_int, [_P, _SZ, _SZ]),
    "hd_get_max_overlap": (_SZ, [_P, _SZ]),
    "hd_execute": (C.c_int, [_P, _P, _SZ, _SZ, _SZ, _SZ, _SZP]),
    "hd_destroy_pipeline": (None, [_P]),
    "hd_clean_filterbank_rfi": (C.c_int, [_P, _P, _SZ, _SZ, _P, _P, C.c_float, C.c_float,
                                          C.c_float, _SZ, _SZ]),
    "hd_set_cleaning": (C.c_int, [_P, C.c_int]),
    "hd_set_narrow_band": (C.c_int, [_P, C.c_int]),
    "hd_execute_device": (C.c_int, [_P, _P, _SZ, _SZ, _SZ, _SZ, _SZP]),
    "hd_execute_beams": (C.c_int, [_P, C.POINTER(_P), _SZ, _SZ, _SZ, _SZ, _SZ, _SZP, C.c_int,
                                   C.POINTER(C.c_int), _SZP]),
    "hd_get_beam_candidates": (C.c_int, [_P, _SZ, _P, _SZP]),
    "hd_get_raw_candidates": (C.c_int, [_P, C.c_void_p, _SZP]),
    "hd_prefetch_beams": (C.c_int, [_P, C.POINTER(_P), _SZ, _SZ, _SZ]),
    "hd_execute_prefetched": (C.c_int, [_P, _SZ, _SZ, _SZP, C.POINTER(C.c_int), _SZP]),
    "hd_create_beam_set": (C.c_int, [C.POINTER(_P), C.c_void_p, _SZ, C.c_int]),
    "hd_set_beam_set_cleaning": (C.c_int, [_P, C.c_int]),
    "hd_get_beam_set_config_count": (_SZ, [_P]),
    "hd_execute_beam_set": (C.c_int, [_P, C.POINTER(_P), _SZP, _SZ, _SZ, C.c_int,
                                      C.POINTER(C.c_int), _SZP]),
    "hd_get_beam_set_candidates": (C.c_int, [_P, _SZ, _P, _SZP]),
    "hd_destroy_beam_set": (None, [_P]),
    "hd_get_launch_count": (C.c_ulonglong, []),
    "hd_set_graphs": (C.c_int, [_P, C.c_int]),
    "hd_get_graph_replays": (C.c_ulonglong, [_P]),
    "hd_measure_int_add_rate": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    "hd_clean_filterbank_rfi_noalloc": (C.c_int, [_P, _SZ, _SZ, _SZ, _P, _P, C.c_float,
                                                  C.c_float, C.c_float, _SZ, _SZ, _P, _P]),
    "hd_get_candidates": (C.c_int, [_P, _P, _SZP]),
    "hd_get_giants": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _SZP]),
    "hd_get_timing": (C.c_int, [_P, _FP, C.c_int]),
    "hd_get_dedisp_tile": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)]),
    "hd_get_dedisp_tile_source": (C.c_int, [_P]),
    "hd_read_sigproc_header": (C.c_int, [C.c_char_p, C.POINTER(HdSigprocHeader)]),
    "hd_coincide": (C.c_int, [_P, _SZ, _SZ, C.c_uint, C.c_uint, C.c_int, _P]),
    "hd_profile_candidates": (C.c_int, [_P, _SZ, _SZ, C.c_int, C.c_double, C.c_double,
                                        C.c_double, _FP, _SZ, _P, _SZ, _SZ, _SZ, _SZ, C.c_int,
                                        _P]),
    "hd_write_coincident_candidates": (C.c_int, [C.c_char_p, _P, _P, _SZ]),
    "hd_mjd_to_utc": (C.c_longlong, [C.c_double]),
    "hd_params_from_sigproc": (C.c_int, [C.POINTER(HdSigprocHeader), C.POINTER(HdParams)]),
    "hd_search_sigproc_file": (C.c_int, [_P, C.c_char_p, _SZ, GULP_CALLBACK, C.c_void_p, _SZP,
                                         _SZP]),
    "hd_search_sigproc_files": (C.c_int, [_P, C.POINTER(C.c_char_p), _SZ, _SZ, GULP_CALLBACK,
                                          C.c_void_p, _SZP, _SZP]),
    "hd_extract_patches": (C.c_int, [_P, _FP, _FP, _SZP]),
    "hd_classifier_param_count": (_SZ, []),
    "hd_classifier_create": (C.c_int, [C.POINTER(_P), C.c_int, C.c_ulonglong]),
    "hd_classifier_destroy": (None, [_P]),
    "hd_classifier_get_params": (C.c_int, [_P, _FP, _SZ]),
    "hd_classifier_set_params": (C.c_int, [_P, _FP, _SZ]),
    "hd_classifier_gradients": (C.c_int, [_P, _FP, _FP, C.POINTER(C.c_int), _SZ, _FP, _FP]),
    "hd_classifier_train": (C.c_int, [_P, _FP, _FP, C.POINTER(C.c_int), _SZ, C.c_int, C.c_int,
                                      C.c_float, C.c_ulonglong, _FP]),
    "hd_classifier_score": (C.c_int, [_P, _FP, _FP, _SZ, _FP]),
    "hd_classifier_score_device": (C.c_int, [_P, C.c_void_p, C.c_void_p, _SZ, _FP]),
    "hd_score_candidates": (C.c_int, [_P, _P, _FP, _SZP]),
    "hd_classifier_get_timing": (C.c_int, [_P, _FP]),
    "hd_bf16_gemm": (C.c_int, [C.c_int, C.c_int, C.c_int, _P, C.c_longlong, C.c_longlong, _P,
                               C.c_longlong, C.c_longlong, _FP, C.c_longlong, C.c_longlong,
                               C.c_int, C.c_int]),
    "hd_bf16_gemm_tc": (C.c_int, [C.c_int, C.c_int, C.c_int, _P, C.c_longlong, C.c_longlong, _P,
                               C.c_longlong, C.c_longlong, _FP, C.c_longlong, C.c_longlong,
                               C.c_int, C.c_int]),
    "dedisp_create_plan": (C.c_int, [C.POINTER(_P), _SZ, C.c_float, C.c_float, C.c_float]),
    "dedisp_destroy_plan": (None, [_P]),
    "dedisp_set_dm_list": (C.c_int, [_P, _FP, _SZ]),
    "dedisp_generate_dm_list": (C.c_int, [_P, C.c_float, C.c_float, C.c_float, C.c_float]),
    "dedisp_generate_dm_list_guru": (_FP, [C.c_float, C.c_float, C.c_double, C.c_double,
                                           C.c_double, C.c_double, _SZ, C.c_double, _SZP]),
    "dedisp_set_killmask": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "dedisp_enable_adaptive_dt": (C.c_int, [_P, C.c_float, C.c_float]),
    "dedisp_disable_adaptive_dt": (C.c_int, [_P]),
    "dedisp_get_dm_count": (_SZ, [_P]),
    "dedisp_get_dm_list": (_FP, [_P]),
    "dedisp_get_dt_factors": (_SZP, [_P]),
    "dedisp_get_max_delay": (_SZ, [_P]),
    "dedisp_get_dm_delay": (_SZ, [_P, C.c_int]),
    "dedisp_get_channel_count": (_SZ, [_P]),
    "dedisp_get_dt": (C.c_float, [_P]),
    "dedisp_get_f0": (C.c_float, [_P]),
    "dedisp_get_df": (C.c_float, [_P]),
    "dedisp_execute_adv": (C.c_int, [_P, _SZ, _P, _SZ, _SZ, _P, _SZ, _SZ, C.c_uint]),
    "dedisp_execute": (C.c_int, [_P, _SZ, _P, _SZ, _P, _SZ, C.c_uint]),
    "dedisp_get_error_string": (C.c_char_p, [C.c_int]),
}

_lib = None


def build() -> str:
    """Compiles libhdb200.so (nvcc, sm_100a) in place."""
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(HERE, "csrc")], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    """Loads libhdb200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with "
                              "heimdall_multibeam_b200.build() (there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SYMBOLS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def error_string(code: int) -> str:
    try:
        return lib().hd_get_error_string(code).decode()
    except ImportError:
        return f"hd_error {code}"


def default_params(**overrides) -> HdParams:
    """hd_set_default_params (the reference's defaults) with overrides.  This
    helper turns adaptive dt off unless use_scrunching is given: the search at
    the native sampling time is what the parity tests and the benchmark run."""
    p = HdParams()
    lib().hd_set_default_params(C.byref(p))
    p.use_scrunching = False
    for k, v in overrides.items():
        if k == "output_dir" or k == "sigproc_file":
            v = None if v is None else v.encode()
        setattr(p, k, v)
    return p


def _u8(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a)
    if a.dtype != np.uint8:
        raise TypeError("filterbank must be uint8")
    return a


def read_sigproc_header(path: str) -> Dict:
    """hd_read_sigproc_header as a dict (raises HdError on failure)."""
    h = HdSigprocHeader()
    err = lib().hd_read_sigproc_header(path.encode(), C.byref(h))
    if err != HD_NO_ERROR:
        raise HdError(err, "hd_read_sigproc_header")
    return h.as_dict()


def params_from_sigproc(path: str, params: Optional[HdParams] = None) -> HdParams:
    """hd_params_from_sigproc on the file's header, over default parameters."""
    h = HdSigprocHeader()
    err = lib().hd_read_sigproc_header(path.encode(), C.byref(h))
    if err != HD_NO_ERROR:
        raise HdError(err, "hd_read_sigproc_header")
    p = params if params is not None else default_params()
    err = lib().hd_params_from_sigproc(C.byref(h), C.byref(p))
    if err != HD_NO_ERROR:
        raise HdError(err, "hd_params_from_sigproc")
    return p


def coincide(cands: np.ndarray, nbeams: int, sep_time: int = 3, sep_filter: int = 4,
             gpu_id: int = 0) -> np.ndarray:
    """hd_coincide on a CANDIDATE_DTYPE array: per candidate (nbeams,
    primary_beam, max_snr) as a structured array."""
    c = np.ascontiguousarray(cands, dtype=CANDIDATE_DTYPE)
    out = (HdCoincidence * max(len(c), 1))()
    err = lib().hd_coincide(c.ctypes.data, len(c), nbeams, sep_time, sep_filter, gpu_id,
                            C.cast(out, C.c_void_p))
    if err != HD_NO_ERROR:
        raise HdError(err, "hd_coincide")
    res = np.zeros(len(c), [("nbeams", "<u4"), ("primary_beam", "<u4"), ("max_snr", "<f4")])
    if len(c):
        C.memmove(res.ctypes.data, out, len(c) * C.sizeof(HdCoincidence))
    return res


def write_coincident_candidates(path: str, cands: np.ndarray, co: np.ndarray) -> None:
    c = np.ascontiguousarray(cands, dtype=CANDIDATE_DTYPE)
    o = np.ascontiguousarray(co)
    err = lib().hd_write_coincident_candidates(path.encode(), c.ctypes.data, o.ctypes.data,
                                               len(c))
    if err != HD_NO_ERROR:
        raise HdError(err, "hd_write_coincident_candidates")


def parse_cand_lines(lines) -> np.ndarray:
    """.cand text lines -> CANDIDATE_DTYPE, numbers read as the reference's
    istream does (floats by strtof, integers exactly)."""
    libc = C.CDLL(None)
    libc.strtof.restype = C.c_float
    libc.strtof.argtypes = [C.c_char_p, C.c_void_p]
    out = np.zeros(len(lines), CANDIDATE_DTYPE)
    for i, ln in enumerate(lines):
        f = ln.split()
        out[i]["snr"] = libc.strtof(f[0].encode(), None)
        out[i]["samp_idx"] = int(f[1])
        out[i]["time"] = libc.strtof(f[2].encode(), None)
        out[i]["filter"] = int(f[3])
        out[i]["dm_trial"] = int(f[4])
        out[i]["dm"] = libc.strtof(f[5].encode(), None)
        out[i]["members"] = int(f[6])
        out[i]["begin"] = int(f[7])
        out[i]["end"] = int(f[8])
        out[i]["beam"] = int(f[9])
    return out


class Pipeline:
    """hd_create_pipeline / hd_execute / hd_destroy_pipeline."""

    def __init__(self, params: Optional[HdParams] = None, cleaning: bool = True,
                 channel_zaps: Sequence[Tuple[int, int]] = (), narrow_band: bool = False,
                 **overrides):
        L = lib()
        self._p = None
        if params is None:
            params = default_params(**overrides)
        else:
            for k, v in overrides.items():
                setattr(params, k, v.encode() if isinstance(v, str) else v)
        self._zaps = (HdRange * max(len(channel_zaps), 1))()
        for i, (a, b) in enumerate(channel_zaps):
            self._zaps[i].start, self._zaps[i].end = a, b
        if channel_zaps:
            params.num_channel_zaps = len(channel_zaps)
            params.channel_zaps = C.cast(self._zaps, C.POINTER(HdRange))
        self.params = params
        h = C.c_void_p()
        err = L.hd_create_pipeline(C.byref(h), params)
        if err != HD_NO_ERROR:
            raise HdError(err, "hd_create_pipeline")
        self._p = h
        L.hd_set_cleaning(self._p, 1 if cleaning else 0)
        L.hd_set_narrow_band(self._p, 1 if narrow_band else 0)

    def close(self) -> None:
        if self._p:
            lib().hd_destroy_pipeline(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def max_overlap(self, nbeams: int = 1) -> int:
        return lib().hd_get_max_overlap(self._p, nbeams)

    def set_graphs(self, enable: bool) -> None:
        """hd_set_graphs: the batched device-resident calls replay each gulp
        of a shape seen before as one CUDA graph (on by default)."""
        err = lib().hd_set_graphs(self._p, 1 if enable else 0)
        if err != HD_NO_ERROR:
            raise HdError(err, "hd_set_graphs")

    def graph_replays(self) -> int:
        """hd_get_graph_replays: gulps this pipeline served by a graph replay."""
        return int(lib().hd_get_graph_replays(self._p))

    def execute(self, filterbank: np.ndarray, nbeams: int = 1, first_idx: int = 0,
                raise_on_error: bool = True, nbits: int = 8) -> Tuple[int, int]:
        """One gulp; filterbank is (nsamps, nchans) uint8 (STF for nbeams > 1),
        or with nbits = 1, 2, 4 or 16 one row of packed samples per spectrum
        (synth.pack_filterbank).  Returns (hd_error, nsamps_processed);
        HD_TOO_MANY_EVENTS is soft."""
        fb = _u8(filterbank) if nbits == 8 else np.ascontiguousarray(filterbank)
        proc = C.c_size_t(0)
        err = lib().hd_execute(self._p, fb.ctypes.data, fb.shape[0], nbits, first_idx, nbeams,
                               C.byref(proc))
        if raise_on_error and err not in (HD_NO_ERROR, HD_TOO_MANY_EVENTS):
            raise HdError(err, "hd_execute")
        return err, proc.value

    def execute_ptr(self, host_ptr: int, nsamps: int, nbeams: int = 1,
                    first_idx: int = 0) -> Tuple[int, int]:
        proc = C.c_size_t(0)
        err = lib().hd_execute(self._p, C.c_void_p(host_ptr), nsamps, 8, first_idx, nbeams,
                               C.byref(proc))
        return err, proc.value

    def execute_device(self, dev_ptr: int, nsamps: int, nbeams: int = 1,
                       first_idx: int = 0, nbits: int = 8) -> Tuple[int, int]:
        """hd_execute_device: the filterbank already sits in device memory."""
        proc = C.c_size_t(0)
        err = lib().hd_execute_device(self._p, C.c_void_p(dev_ptr), nsamps, nbits, first_idx,
                                      nbeams, C.byref(proc))
        return err, proc.value

    def execute_beams(self, filterbanks: Sequence, nsamps: Optional[int] = None,
                      nbeams: int = 1, first_idx: int = 0, beams: Optional[Sequence[int]] = None,
                      on_device: bool = False,
                      raise_on_error: bool = True) -> Tuple[int, int, List[int]]:
        """hd_execute_beams over independent filterbanks: uint8 arrays of equal
        shape (nsamps, nchans), or raw pointers (host, or device when
        on_device) with nsamps given.  Returns (hd_error, nsamps_processed,
        per-filterbank statuses)."""
        keep = []
        ptrs = (_P * max(len(filterbanks), 1))()
        for u, fb in enumerate(filterbanks):
            if isinstance(fb, int):
                if nsamps is None:
                    raise ValueError("nsamps is required with raw pointers")
                ptrs[u] = fb
            else:
                a = _u8(fb)
                if nsamps is None:
                    nsamps = a.shape[0]
                if a.shape[0] != nsamps:
                    raise ValueError("all filterbanks need the same number of samples")
                keep.append(a)
                ptrs[u] = a.ctypes.data
        n = len(filterbanks)
        st = (C.c_int * max(n, 1))()
        bm = None
        if beams is not None:
            bm = (C.c_size_t * n)(*beams)
        proc = C.c_size_t(0)
        err = lib().hd_execute_beams(self._p, ptrs, n, nsamps or 0, 8, first_idx, nbeams, bm,
                                     1 if on_device else 0, st, C.byref(proc))
        if raise_on_error and err not in (HD_NO_ERROR, HD_TOO_MANY_EVENTS):
            raise HdError(err, "hd_execute_beams")
        return err, proc.value, [int(st[u]) for u in range(n)]

    def candidates(self, index: Optional[int] = None) -> np.ndarray:
        """Candidates of the last execute (all), or of filterbank `index` of
        the last execute_beams."""
        n = C.c_size_t(0)
        if index is None:
            lib().hd_get_candidates(self._p, None, C.byref(n))
        else:
            err = lib().hd_get_beam_candidates(self._p, index, None, C.byref(n))
            if err != HD_NO_ERROR:
                raise HdError(err, "hd_get_beam_candidates")
        out = np.zeros(n.value, CANDIDATE_DTYPE)
        if n.value:
            if index is None:
                lib().hd_get_candidates(self._p, out.ctypes.data, C.byref(n))
            else:
                lib().hd_get_beam_candidates(self._p, index, out.ctypes.data, C.byref(n))
        return out

    def giants(self) -> Dict[str, np.ndarray]:
        n = C.c_size_t(0)
        lib().hd_get_giants(self._p, None, None, None, None, None, None, None, C.byref(n))
        g = dict(peaks=np.zeros(n.value, np.float32),
                 **{k: np.zeros(n.value, np.uint64) for k in
                    ("inds", "begins", "ends", "filter_inds", "dm_inds", "labels")})
        if n.value:
            lib().hd_get_giants(self._p, g["peaks"].ctypes.data, g["inds"].ctypes.data,
                                g["begins"].ctypes.data, g["ends"].ctypes.data,
                                g["filter_inds"].ctypes.data, g["dm_inds"].ctypes.data,
                                g["labels"].ctypes.data, C.byref(n))
        return g

    def patches(self) -> Tuple[np.ndarray, np.ndarray]:
        """hd_extract_patches: (dm_time [n, 64, 64], freq_time [n, 64, 256]) of
        the last execute's candidates, in candidates() order."""
        n = C.c_size_t(0)
        lib().hd_extract_patches(self._p, None, None, C.byref(n))
        dm = np.zeros((n.value, 64, 64), np.float32)
        ft = np.zeros((n.value, 64, 256), np.float32)
        if n.value:
            err = lib().hd_extract_patches(self._p, dm.ctypes.data_as(_FP), ft.ctypes.data_as(_FP),
                                           C.byref(n))
            if err != HD_NO_ERROR:
                raise HdError(err, "hd_extract_patches")
        return dm, ft

    def scores(self, classifier: "Classifier") -> np.ndarray:
        """hd_score_candidates: the classifier's P(pulse) for each candidate
        of the last execute (patches extracted and scored on the GPU)."""
        n = C.c_size_t(0)
        lib().hd_score_candidates(self._p, classifier._p, None, C.byref(n))
        out = np.zeros(n.value, np.float32)
        if n.value:
            err = lib().hd_score_candidates(self._p, classifier._p, out.ctypes.data_as(_FP),
                                            C.byref(n))
            if err != HD_NO_ERROR:
                raise HdError(err, "hd_score_candidates")
        return out

    def prefetch_beams(self, host_ptrs: Sequence[int], nsamps: int) -> int:
        """hd_prefetch_beams on raw host pointers (pinned for overlap)."""
        ptrs = (_P * len(host_ptrs))(*host_ptrs)
        return lib().hd_prefetch_beams(self._p, ptrs, len(host_ptrs), nsamps, 8)

    def execute_prefetched(self, nunits: int, first_idx: int = 0, nbeams: int = 1,
                           beams: Optional[Sequence[int]] = None) -> Tuple[int, int, List[int]]:
        """hd_execute_prefetched: (hd_error, nsamps_processed, statuses)."""
        st = (C.c_int * max(nunits, 1))()
        bm = (C.c_size_t * nunits)(*beams) if beams is not None else None
        proc = C.c_size_t(0)
        err = lib().hd_execute_prefetched(self._p, first_idx, nbeams, bm, st, C.byref(proc))
        return err, proc.value, list(st)[:nunits]

    def search_sigproc_files(self, paths: Sequence[str], nsamps_gulp: int):
        """hd_search_sigproc_files over files read in lockstep: (hd_error,
        total spectra searched per beam, [(first_idx, candidates of all
        files) per gulp])."""
        gulps = []

        def cb(user, cands, n, first_idx):
            a = np.zeros(n, CANDIDATE_DTYPE)
            if n:
                C.memmove(a.ctypes.data, cands, n * CANDIDATE_DTYPE.itemsize)
            gulps.append((int(first_idx), a))

        fn = GULP_CALLBACK(cb)
        arr = (C.c_char_p * len(paths))(*[p.encode() for p in paths])
        total = C.c_size_t(0)
        ng = C.c_size_t(0)
        err = lib().hd_search_sigproc_files(self._p, arr, len(paths), nsamps_gulp, fn, None,
                                            C.byref(total), C.byref(ng))
        assert ng.value == len(gulps)
        return err, total.value, gulps

    def search_sigproc_file(self, path: str, nsamps_gulp: int):
        """hd_search_sigproc_file: (hd_error, total spectra searched per beam,
        [(first_idx, candidates) per gulp])."""
        gulps = []

        def cb(user, cands, n, first_idx):
            a = np.zeros(n, CANDIDATE_DTYPE)
            if n:
                C.memmove(a.ctypes.data, cands, n * CANDIDATE_DTYPE.itemsize)
            gulps.append((int(first_idx), a))

        fn = GULP_CALLBACK(cb)
        total = C.c_size_t(0)
        ng = C.c_size_t(0)
        err = lib().hd_search_sigproc_file(self._p, path.encode(), nsamps_gulp, fn, None,
                                           C.byref(total), C.byref(ng))
        assert ng.value == len(gulps)
        return err, total.value, gulps

    def dedisp_tile(self) -> Tuple[int, int, int]:
        """hd_get_dedisp_tile: (DM block, time block, rows per stage) of the
        last gulp's dedispersion."""
        v = [C.c_int(0) for _ in range(3)]
        lib().hd_get_dedisp_tile(self._p, *(C.byref(x) for x in v))
        return tuple(int(x.value) for x in v)

    TILE_SOURCES = ("default", "HDB_DEDISP_TILE", "autotuner", "tile cache")

    def dedisp_tile_source(self) -> str:
        """hd_get_dedisp_tile_source as a name: where the last gulp's tile
        came from (the default, HDB_DEDISP_TILE, the autotuner or the
        persistent tile cache)."""
        return self.TILE_SOURCES[lib().hd_get_dedisp_tile_source(self._p)]

    def timing(self) -> Dict[str, float]:
        t = (C.c_float * 8)()
        lib().hd_get_timing(self._p, t, 8)
        names = ("total", "clean", "dedisperse", "baseline_scan", "boxcar_threshold",
                 "giants", "cluster_merge", "h2d")
        return {n: float(v) for n, v in zip(names, t)}

    def clean_filterbank_rfi(self, filterbank: np.ndarray, dt: float, baseline_length=2.0,
                             rfi_tol=5.0, boxcar_max=64, nbeams=1):
        fb = _u8(filterbank)
        out = np.zeros_like(fb)
        mask = np.zeros(fb.shape[0], np.int32)
        err = lib().hd_clean_filterbank_rfi(self._p, fb.ctypes.data, fb.shape[0], 8,
                                            out.ctypes.data, mask.ctypes.data, dt,
                                            baseline_length, rfi_tol, boxcar_max, nbeams)
        if err != HD_NO_ERROR:
            raise HdError(err, "hd_clean_filterbank_rfi")
        return out, mask


def launch_count() -> int:
    return int(lib().hd_get_launch_count())


def int_add_rate(device: int = 0) -> float:
    """Measured 32-bit integer adds per second of the device
    (hd_measure_int_add_rate)."""
    v = C.c_double(0.0)
    err = lib().hd_measure_int_add_rate(device, C.byref(v))
    if err != HD_NO_ERROR:
        raise HdError(err, "hd_measure_int_add_rate")
    return float(v.value)


def cand_lines(c: np.ndarray) -> list:
    """.cand text lines of candidate rows (Pipeline/pipeline.cu:1028-1038)."""
    return ["%g\t%d\t%g\t%d\t%d\t%g\t%d\t%d\t%d\t%d\t" % (
        float(r["snr"]), int(r["samp_idx"]), float(r["time"]), int(r["filter"]),
        int(r["dm_trial"]), float(r["dm"]), int(r["members"]), int(r["begin"]), int(r["end"]),
        int(r["beam"])) for r in c]


class DedispPlan:
    """dedisp_create_plan / ... / dedisp_execute (include/dedisp.h)."""

    def __init__(self, nchans: int, dt: float, f0: float, df: float):
        h = C.c_void_p()
        err = lib().dedisp_create_plan(C.byref(h), nchans, dt, f0, df)
        if err != DEDISP_NO_ERROR:
            raise RuntimeError(lib().dedisp_get_error_string(err).decode())
        self._p = h
        self.nchans = nchans

    def close(self):
        if self._p:
            lib().dedisp_destroy_plan(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, err, what):
        if err != DEDISP_NO_ERROR:
            raise RuntimeError(f"{what}: {lib().dedisp_get_error_string(err).decode()}")

    def generate_dm_list(self, dm_min, dm_max, pulse_width=40.0, tol=1.25):
        self._check(lib().dedisp_generate_dm_list(self._p, dm_min, dm_max, pulse_width, tol),
                    "dedisp_generate_dm_list")

    def set_dm_list(self, dms):
        a = np.ascontiguousarray(dms, np.float32)
        self._check(lib().dedisp_set_dm_list(self._p, a.ctypes.data_as(_FP), len(a)),
                    "dedisp_set_dm_list")

    def set_killmask(self, km):
        a = np.ascontiguousarray(km, np.int32)
        self._check(lib().dedisp_set_killmask(self._p, a.ctypes.data_as(C.POINTER(C.c_int))),
                    "dedisp_set_killmask")

    def enable_adaptive_dt(self, pulse_width=40.0, tol=1.15):
        self._check(lib().dedisp_enable_adaptive_dt(self._p, pulse_width, tol),
                    "dedisp_enable_adaptive_dt")

    def disable_adaptive_dt(self):
        self._check(lib().dedisp_disable_adaptive_dt(self._p), "dedisp_disable_adaptive_dt")

    @property
    def dt_factors(self) -> np.ndarray:
        n = lib().dedisp_get_dm_count(self._p)
        p = lib().dedisp_get_dt_factors(self._p)
        return np.ctypeslib.as_array(p, shape=(n,)).astype(np.uint64) if n else np.zeros(0, np.uint64)

    @property
    def dm_list(self) -> np.ndarray:
        n = lib().dedisp_get_dm_count(self._p)
        p = lib().dedisp_get_dm_list(self._p)
        return np.ctypeslib.as_array(p, shape=(n,)).copy() if n else np.zeros(0, np.float32)

    @property
    def max_delay(self) -> int:
        return lib().dedisp_get_max_delay(self._p)

    def execute(self, filterbank: np.ndarray, nbits: int = 8) -> np.ndarray:
        """dedisp_execute: (nsamps, nchans) uint8, or packed rows of nbits = 1,
        2, 4 or 16-bit samples (synth.pack_filterbank)."""
        fb = _u8(filterbank) if nbits == 8 else np.ascontiguousarray(filterbank)
        nsamps = fb.shape[0]
        nout = nsamps - self.max_delay
        D = lib().dedisp_get_dm_count(self._p)
        out = np.zeros((D, nout), np.float32)
        self._check(lib().dedisp_execute(self._p, nsamps, fb.ctypes.data, nbits, out.ctypes.data,
                                         32, 0), "dedisp_execute")
        return out


def dm_list_guru(dm_min, dm_max, dt, pulse_width, f0, df, nchans, tol) -> np.ndarray:
    n = C.c_size_t(0)
    p = lib().dedisp_generate_dm_list_guru(dm_min, dm_max, dt, pulse_width, f0, df, nchans, tol,
                                           C.byref(n))
    return np.ctypeslib.as_array(p, shape=(n.value,)).copy()


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class BeamSet:
    """hd_create_beam_set / hd_execute_beam_set: beams of different shapes
    (one HdParams each) searched in one call; beam b's results equal a
    separate Pipeline(params[b]).execute of its filterbank."""

    def __init__(self, params: Sequence[HdParams], workers: int = 4, cleaning: bool = True):
        self._p = None
        self._params = (HdParams * len(params))(*params)
        h = C.c_void_p()
        err = lib().hd_create_beam_set(C.byref(h), C.cast(self._params, C.c_void_p), len(params),
                                       workers)
        if err != HD_NO_ERROR:
            raise HdError(err, "hd_create_beam_set")
        self._p = h
        self.nbeams = len(params)
        lib().hd_set_beam_set_cleaning(self._p, 1 if cleaning else 0)

    @property
    def nconfigs(self) -> int:
        return int(lib().hd_get_beam_set_config_count(self._p))

    def close(self) -> None:
        if self._p:
            lib().hd_destroy_beam_set(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def execute(self, filterbanks: Sequence, nsamps: Optional[Sequence[int]] = None,
                first_idx: int = 0, on_device: bool = False) -> Tuple[int, List[int], List[int]]:
        """filterbanks: uint8 arrays (nsamps_b, nchans_b), or raw pointers
        (host, or device when on_device) with nsamps given.  Returns
        (hd_error, per-beam statuses, per-beam nsamps_processed)."""
        n = self.nbeams
        if len(filterbanks) != n:
            raise ValueError(f"{n} filterbanks expected")
        keep = []
        ptrs = (_P * n)()
        ns = (C.c_size_t * n)()
        for b, fb in enumerate(filterbanks):
            if isinstance(fb, int):
                if nsamps is None:
                    raise ValueError("nsamps is required with raw pointers")
                ptrs[b] = fb
                ns[b] = nsamps[b]
            else:
                a = _u8(fb)
                keep.append(a)
                ptrs[b] = a.ctypes.data
                ns[b] = a.shape[0] if nsamps is None else nsamps[b]
        st = (C.c_int * n)()
        proc = (C.c_size_t * n)()
        err = lib().hd_execute_beam_set(self._p, ptrs, ns, 8, first_idx, 1 if on_device else 0,
                                        st, proc)
        return err, list(st), list(proc)

    def candidates(self, beam: int) -> np.ndarray:
        n = C.c_size_t(0)
        err = lib().hd_get_beam_set_candidates(self._p, beam, None, C.byref(n))
        if err != HD_NO_ERROR:
            raise HdError(err, "hd_get_beam_set_candidates")
        out = np.zeros(n.value, CANDIDATE_DTYPE)
        if n.value:
            lib().hd_get_beam_set_candidates(self._p, beam, out.ctypes.data, C.byref(n))
        return out


class Classifier:
    """hd_classifier_*: the candidate classifier (two-branch CNN on the
    DM-time and freq-time patches, BF16 tensor-core GEMMs on the GPU)."""

    def __init__(self, seed: int = 1, gpu_id: int = 0):
        h = C.c_void_p()
        err = lib().hd_classifier_create(C.byref(h), gpu_id, seed)
        if err != HD_NO_ERROR:
            raise HdError(err, "hd_classifier_create")
        self._p = h
        self.nparam = int(lib().hd_classifier_param_count())

    def close(self) -> None:
        if self._p:
            lib().hd_classifier_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def params(self) -> np.ndarray:
        out = np.zeros(self.nparam, np.float32)
        err = lib().hd_classifier_get_params(self._p, out.ctypes.data_as(_FP), self.nparam)
        if err != HD_NO_ERROR:
            raise HdError(err, "hd_classifier_get_params")
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = _f32(p)
        err = lib().hd_classifier_set_params(self._p, p.ctypes.data_as(_FP), self.nparam)
        if err != HD_NO_ERROR:
            raise HdError(err, "hd_classifier_set_params")

    def gradients(self, dm_time, freq_time, labels) -> Tuple[np.ndarray, float]:
        dm, ft = _f32(dm_time), _f32(freq_time)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        g = np.zeros(self.nparam, np.float32)
        loss = C.c_float(0)
        err = lib().hd_classifier_gradients(self._p, dm.ctypes.data_as(_FP), ft.ctypes.data_as(_FP),
                                            lab.ctypes.data_as(C.POINTER(C.c_int)), len(lab),
                                            g.ctypes.data_as(_FP), C.byref(loss))
        if err != HD_NO_ERROR:
            raise HdError(err, "hd_classifier_gradients")
        return g, loss.value

    def train(self, dm_time, freq_time, labels, epochs: int = 10, batch: int = 128,
              lr: float = 1e-3, seed: int = 7) -> np.ndarray:
        dm, ft = _f32(dm_time), _f32(freq_time)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        losses = np.zeros(epochs, np.float32)
        err = lib().hd_classifier_train(self._p, dm.ctypes.data_as(_FP), ft.ctypes.data_as(_FP),
                                        lab.ctypes.data_as(C.POINTER(C.c_int)), len(lab), epochs,
                                        batch, lr, seed, losses.ctypes.data_as(_FP))
        if err != HD_NO_ERROR:
            raise HdError(err, "hd_classifier_train")
        return losses

    def score(self, dm_time, freq_time) -> np.ndarray:
        dm, ft = _f32(dm_time), _f32(freq_time)
        n = dm.shape[0]
        out = np.zeros(n, np.float32)
        if n:
            err = lib().hd_classifier_score(self._p, dm.ctypes.data_as(_FP), ft.ctypes.data_as(_FP),
                                            n, out.ctypes.data_as(_FP))
            if err != HD_NO_ERROR:
                raise HdError(err, "hd_classifier_score")
        return out

    def last_score_ms(self) -> float:
        """hd_classifier_get_timing: device ms of the last scoring call."""
        ms = C.c_float(0.0)
        lib().hd_classifier_get_timing(self._p, C.byref(ms))
        return float(ms.value)

    def score_device(self, dm_ptr: int, ft_ptr: int, n: int) -> np.ndarray:
        """hd_classifier_score_device on device pointers (n patch pairs)."""
        out = np.zeros(n, np.float32)
        if n:
            err = lib().hd_classifier_score_device(self._p, C.c_void_p(dm_ptr), C.c_void_p(ft_ptr),
                                                   n, out.ctypes.data_as(_FP))
            if err != HD_NO_ERROR:
                raise HdError(err, "hd_classifier_score_device")
        return out


def profile_candidates(filterbank, tsamp: float, fch1: float, foff: float, dm_list,
                       requests: Sequence[Tuple[int, int, int]], out_nsamps: int = 64,
                       out_dm_count: int = 32, fscrunch: int = 16, do_filter: bool = False,
                       nsamps: Optional[int] = None, nchans: Optional[int] = None,
                       on_device: bool = False) -> List[Dict]:
    """hd_profile_candidates: the candidate profiler's arrays for each
    (samp, filter, dm_idx) request.  filterbank: (nsamps, nchans) uint8, or a
    device pointer with nsamps, nchans and on_device."""
    if isinstance(filterbank, int):
        ptr, ns, nc = filterbank, nsamps, nchans
        keep = None
    else:
        keep = _u8(filterbank)
        ptr, (ns, nc) = keep.ctypes.data, keep.shape
    dms = np.ascontiguousarray(dm_list, np.float32)
    n = len(requests)
    reqs = (HdProfileRequest * n)(*[HdProfileRequest(int(a), int(b), int(c))
                                    for a, b, c in requests])
    outs = (HdProfile * n)()
    arrays = []
    for i in range(n):
        a = dict(dm_time=np.zeros((out_dm_count, out_nsamps), np.float32),
                 dm0_time=np.zeros(out_nsamps, np.float32),
                 freq_time=np.zeros((nc // fscrunch, out_nsamps), np.float32),
                 snr_dm=np.zeros(out_dm_count, np.float32),
                 snr_time=np.zeros((out_nsamps, 5), np.float32))
        for k, v in a.items():
            setattr(outs[i], k, v.ctypes.data)
        arrays.append(a)
    err = lib().hd_profile_candidates(C.c_void_p(ptr), ns, nc, 1 if on_device else 0, tsamp,
                                      fch1, foff, dms.ctypes.data_as(_FP), len(dms),
                                      C.cast(reqs, C.c_void_p), n, out_nsamps, out_dm_count,
                                      fscrunch, 1 if do_filter else 0, C.cast(outs, C.c_void_p))
    if err != HD_NO_ERROR:
        raise HdError(err, "hd_profile_candidates")
    for i in range(n):
        arrays[i].update(max_idx=outs[i].max_idx, n_dm=outs[i].n_dm, dm_begin=outs[i].dm_begin,
                         snr_dm_first=outs[i].snr_dm_first)
    return arrays
