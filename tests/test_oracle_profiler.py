"""The candidate-profiler restatement (oracle/profiler.c) against the
reference's own application (Applications/candidate_profiler.C, compiled
unchanged by `make -C oracle ref` and linked with the CPU dedisperser).

The application reads a sigproc file and a DM list and writes freq_time.dat,
snr_dm.dat, snr_time.dat and dm_time.pgm; the restatement's arrays are
printed the way the application prints them and compared as text, for both
filtering modes and for candidates of several widths and DMs.  Rows with no
deviation are NaN in both (the application divides by zero)."""
import os

import numpy as np
import pytest

import oracle
from heimdall_multibeam_b200 import synth

needs_ref = pytest.mark.skipif(not oracle.ref_profiler_available(),
                               reason="reference profiler (oracle/_ref) not present")


def _num(v, prec):
    """A float as std::ostream prints it at precision `prec` (glibc: -nan
    for a NaN with the sign bit set)."""
    v = np.float32(v)
    if np.isnan(v):
        return "-nan" if np.signbit(v) else "nan"
    if np.isinf(v):
        return "-inf" if v < 0 else "inf"
    return "%.*g" % (prec, float(v))


def _files(r, dms, fscrunch, out_nsamps, out_dm_count):
    ft = []
    for c in range(r["freq_time"].shape[0]):
        row = r["freq_time"][c].copy()
        row[np.isnan(row)] = 0
        if c * fscrunch < 150:  # candidate_profiler.C:545-547
            row[:] = 0
        ft.append("".join(_num(v, 6) + "\t" for v in row))
    first = r["snr_dm_first"]
    sd = ["#dm_trial\tDM\tSNR"]
    for d in range(min(out_dm_count, len(dms))):
        sd.append("%d\t%s\t%s" % (first + d, _num(dms[first + d], 10), _num(r["snr_dm"][d], 10)))
    st = ["#sample\ttime\tSNR\tSNR@DM-1\tSNR@DM+1\tSNR@DM0"]
    for t in range(out_nsamps):
        row = r["snr_time"][t]
        st.append("\t".join([_num(row[0], 6 if t == 0 else 10)] +
                            [_num(x, 10) for x in row]))
    pgm = ["P2 %d %d 255" % (out_nsamps, out_dm_count)]
    for d in range(out_dm_count):
        vals = []
        for v in r["dm_time"][d]:
            x = np.float32(v) / np.float32(8.0) * np.float32(255.0)
            x = min(max(x, np.float32(0.0)), np.float32(255.0)) if not np.isnan(x) else x
            # a NaN level converts to size_t as x86 converts it: 2^63
            vals.append("%d" % int(x) if not np.isnan(x) else str(1 << 63))
        pgm.append("".join(s + "\t" for s in vals))
    return {"freq_time.dat": ft, "snr_dm.dat": sd, "snr_time.dat": st, "dm_time.pgm": pgm}


CASES = [  # pulse index of the 256-channel workload, filter, out_nsamps, out_dm_count, fscrunch
    (1, 4, 64, 32, 16),
    (0, 2, 64, 16, 8),
    (2, 7, 128, 8, 16),
]


@needs_ref
@pytest.mark.parametrize("do_filter", [0, 1])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_profiler_equals_reference(oracle_lib, tmp_path, case, do_filter):
    w = synth.SEARCH_C0
    b = synth.make_c0()
    path = str(tmp_path / "c0.fil")
    synth.write_sigproc(path, b.data, nchans=w.nchans, nbits=8, tsamp=w.dt, fch1=w.f0,
                        foff=w.df, tstart=60000.0)
    dms = oracle.dm_list(0.0, 1000.0, w.dt, 40.0, w.f0, w.df, w.nchans, 1.25)
    k, filt, out_n, out_d, fs = CASES[case]
    p = b.pulses[k]
    dm_idx = int(np.argmin(np.abs(dms - p.dm)))
    samp = int(p.t0)
    r = oracle.profile(b.data, w.dt, w.f0, w.df, dms, samp, filt, dm_idx, out_n, out_d, fs,
                       bool(do_filter))
    assert r["n_dm"] == out_d
    dmax = r["max_idx"] // out_n
    assert 0 < dmax < out_d - 1   # the application reads rows dmax - 1 and dmax + 1
    ref = oracle.ref_profile(path, dms, samp, filt, dm_idx, out_n, out_d, fs, bool(do_filter))
    ours = _files(r, dms, fs, out_n, out_d)
    for name in ("freq_time.dat", "snr_dm.dat", "snr_time.dat", "dm_time.pgm"):
        assert ours[name] == ref[name], name
