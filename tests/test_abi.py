"""The C-ABI boundary: the library loads, exports every function the headers
declare, and the Python mirror's struct layouts match the C compiler's."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import heimdall_multibeam_b200 as hdb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in ("heimdall_b200.h", "dedisp.h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b((?:hd|dedisp)_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(hdb):
    L = hdb.lib()
    declared = declared_functions()
    assert len(declared) >= 30
    missing = [n for n in sorted(declared) if not hasattr(L, n)]
    assert not missing, missing
    assert declared == set(hdb.SYMBOLS), declared ^ set(hdb.SYMBOLS)


def _c_layout(struct, fields):
    body = "\n".join(f'  printf("%zu %zu\\n", offsetof({struct}, {f}), sizeof(((({struct}*)0))->{f}));'
                     for f in fields)
    prog = f"""#include <stdio.h>
#include <stddef.h>
#include "heimdall_b200.h"
int main(void) {{
  printf("%zu\\n", sizeof({struct}));
{body}
  return 0;
}}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        open(c, "w").write(prog)
        exe = os.path.join(d, "l")
        subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe],
                       check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    size = int(out[0])
    lay = [tuple(int(x) for x in ln.split()) for ln in out[1:] if ln.strip()]
    return size, lay


@pytest.mark.parametrize("cls,cname", [(hdb.HdParams, "struct hd_params"),
                                       (hdb.HdCandidate, "hd_candidate"),
                                       (hdb.HdSigprocHeader, "hd_sigproc_header"),
                                       (hdb.HdCoincidence, "hd_coincidence"),
                                       (hdb.HdProfileRequest, "hd_profile_request"),
                                       (hdb.HdProfile, "hd_profile"),
                                       (hdb.RawCandidates, "struct RawCandidates")])
def test_struct_layout_matches_c(cls, cname):
    fields = [f for f, _ in cls._fields_]
    size, lay = _c_layout(cname, fields)
    assert size == C.sizeof(cls)
    for (f, t), (off, sz) in zip(cls._fields_, lay):
        assert getattr(cls, f).offset == off, f
        assert C.sizeof(t) == sz, f


def test_candidate_dtype_matches_struct():
    assert hdb.CANDIDATE_DTYPE.itemsize == C.sizeof(hdb.HdCandidate)
    for f, _ in hdb.HdCandidate._fields_:
        assert hdb.CANDIDATE_DTYPE.fields[f][1] == getattr(hdb.HdCandidate, f).offset


def test_default_params_and_errors(hdb):
    p = hdb.default_params()
    assert p.nchans == 1024 and p.boxcar_max == 4096 and abs(p.detect_thresh - 6.0) < 1e-6
    assert p.cand_sep_dm == 200 and p.min_tscrunch_width == 4096
    assert hdb.error_string(hdb.HD_TOO_MANY_EVENTS) == "Too many events"
    assert hdb.error_string(hdb.HD_TOO_FEW_NSAMPS) == "No. samples < maximum delay"


def test_parse_command_line(hdb):
    L = hdb.lib()
    p = hdb.default_params()
    args = [b"heimdall", b"-f", b"x.fil", b"-dm", b"10", b"500", b"-boxcar_max", b"1024",
            b"-zap_chans", b"5", b"9", b"-V", b"-beam", b"3"]
    argv = (C.c_char_p * len(args))(*args)
    assert L.hd_parse_command_line(len(args), argv, C.byref(p)) == 0
    assert p.dm_min == 10.0 and p.dm_max == 500.0 and p.boxcar_max == 1024
    assert p.num_channel_zaps == 1 and p.channel_zaps[0].start == 5 and p.channel_zaps[0].end == 9
    assert p.verbosity == 2 and p.beam == 2 and p.override_beam


def test_dm_list_guru_matches_golden(hdb):
    """The product's generator reproduces Share/dm2000.list (host code, no GPU)."""
    golden = open(os.path.join(ROOT, "tests", "golden", "dm2000.list")).read().split()
    dms = hdb.dm_list_guru(0.0, 2000.0, 64e-6, 40.0, 1581.804688, -0.390625, 1024, 1.25)
    assert ["%g" % float(x) for x in dms[1:]] == golden


def test_header_compiles_as_cxx_with_reference_types():
    """The reference's C++ Candidates type (Pipeline/hd/types.h:38-43) derives
    from RawCandidates as there."""
    prog = """#include "heimdall_b200.h"
int main() {
  Candidates c;
  RawCandidates* r = &c;
  r->peaks = 0;
  c.dms = 0;
  ConstRawCandidates k;
  k.inds = 0;
  hd_range_t z = {1, 2};
  return (int)(z.end - z.start) - 1;
}
"""
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.cpp")
        open(src, "w").write(prog)
        exe = os.path.join(d, "t")
        subprocess.run(["/usr/bin/g++", "-I", os.path.join(ROOT, "include"), src, "-o", exe],
                       check=True)
        assert subprocess.run([exe]).returncode == 0



def test_c_caller_links_with_documented_line(hdb, tmp_path):
    """A plain C caller built with the include and link flags given to C
    callers (-I include, -L ... -lhdb200 with an rpath) links and runs the
    calls that need no GPU: default parameters, command-line parsing, error
    strings and the sigproc header reader."""
    from heimdall_multibeam_b200 import synth
    fil = str(tmp_path / "h.fil")
    synth.write_sigproc(fil, np.zeros((50, 64), np.uint8), nchans=64, nbits=8, tsamp=1e-4,
                        fch1=1400.0, foff=-1.0, tstart=60000.25, nbeams=3, ibeam=2)
    src = tmp_path / "caller.c"
    src.write_text(r'''#include <stdio.h>
#include "heimdall_b200.h"
int main(int argc, char** argv) {
  struct hd_params p;
  hd_set_default_params(&p);
  char* args[] = {"heimdall", "-dm", "0", "500", "-boxcar_max", "256", "-f", argv[1]};
  if (hd_parse_command_line(8, args, &p) != 0) return 2;
  if (p.sigproc_file == NULL) return 3;
  hd_sigproc_header h;
  hd_error e = hd_read_sigproc_header(argv[1], &h);
  printf("%d %g %zu %d %d %d %s\n", (int)e, (double)p.dm_max, (size_t)p.boxcar_max,
         (int)h.nchans, (int)h.nbeams, (int)h.ibeam, hd_get_error_string(HD_TOO_FEW_NSAMPS));
  return e == HD_NO_ERROR ? 0 : 1;
}
''')
    libdir = os.path.join(ROOT, "heimdall_multibeam_b200")
    exe = str(tmp_path / "caller")
    subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", exe,
                    "-L" + libdir, "-lhdb200", "-Wl,-rpath," + libdir], check=True)
    out = subprocess.run([exe, fil], capture_output=True, text=True, check=True).stdout.split()
    assert out[:6] == ["0", "500", "256", "64", "3", "2"], out
    assert " ".join(out[6:]) == hdb.lib().hd_get_error_string(hdb.HD_TOO_FEW_NSAMPS).decode()


def _layout_probe(tmp, include_line, defines, extra_inc):
    """sizeof(hd_params) and every field's offset/size, as a C++ compiler
    lays out the struct that `include_line` declares."""
    import oracle
    names = [f for f, _ in hdb.HdParams._fields_]
    if "HAVE_PSRDADA" in defines:
        names = names[:1] + ["dada_id"] + names[1:]
    body = "\n".join(
        f'  printf("{n} %zu %zu\\n", offsetof(hd_params, {n}), sizeof(((hd_params*)0)->{n}));'
        for n in names)
    src = os.path.join(tmp, "probe.cpp")
    with open(src, "w") as f:
        f.write(f"""#include <cstdio>
#include <cstddef>
{include_line}
int main() {{
  printf("size %zu\\n", sizeof(hd_params));
{body}
  return 0;
}}
""")
    exe = os.path.join(tmp, "probe")
    cmd = ["/usr/bin/g++", "-w"] + [f"-D{d}" for d in defines]
    for d in extra_inc:
        cmd += ["-I", d]
    subprocess.run(cmd + [src, "-o", exe], check=True)
    return subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")


@pytest.mark.parametrize("psrdada", [False, True])
def test_params_layout_equals_reference_headers(tmp_path, psrdada):
    """include/heimdall_b200.h lays out hd_params field for field as the
    reference's own Pipeline/hd/params.h and hd/types.h, compiled here with
    stand-ins for what they pull in (config.h; dada_hdu.h, which only needs
    to supply key_t), with HAVE_PSRDADA off and on."""
    import oracle
    ref = oracle.reference_dir()
    if not os.path.exists(os.path.join(ref, "Pipeline", "hd", "params.h")):
        pytest.skip("reference tree not present")
    stub = tmp_path / "stub"
    stub.mkdir()
    (stub / "config.h").write_text("/* stand-in for the autotools config.h */\n")
    (stub / "dada_hdu.h").write_text("#include <sys/types.h>\n")
    defines = ["HAVE_PSRDADA"] if psrdada else []
    theirs = _layout_probe(str(tmp_path), '#include "hd/params.h"', defines,
                           [str(stub), os.path.join(ref, "Pipeline")])
    (tmp_path / "ours").mkdir()
    ours = _layout_probe(str(tmp_path / "ours"), '#include "heimdall_b200.h"', defines,
                         [os.path.join(ROOT, "include")])
    assert len(ours) > 30
    assert ours == theirs
    if not psrdada:
        assert ours[0] == f"size {C.sizeof(hdb.HdParams)}"
