"""The autotuner's tile choice persists across processes (the tile cache).

A first process searches a gulp with HDB_TUNE_CACHE pointing at a fresh file:
the autotuner times the candidate tiles and appends its choice.  A second
process with the same file and shape reads the tile from the cache without
timing anything, picks the same tile and finds the same candidates (every
tile gives the same sums).  A different shape is a different key, and
HDB_TUNE_CACHE=0 writes nothing.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import heimdall_multibeam_b200 as H
from heimdall_multibeam_b200 import synth
nsamps = int(sys.argv[2])
w = synth.SEARCH_C0
b = synth.make_beam(nsamps, 64, w.dt, w.f0, w.df * 4,
                    [synth.Pulse(3000.0, 150.0, 1e-3, 30.0)], seed=5)
p = H.default_params(nchans=64, output_dir=None, dt=w.dt, f0=w.f0, df=w.df * 4,
                     dm_min=0.0, dm_max=300.0, boxcar_max=256)
with H.Pipeline(p) as pl:
    pl.execute(b.data)
    print(json.dumps({"tile": pl.dedisp_tile(), "source": pl.dedisp_tile_source(),
                      "cands": H.cand_lines(pl.candidates())}))
"""


def _run(cache, nsamps=1 << 14, **extra):
    env = dict(os.environ)
    env.pop("HDB_DEDISP_TILE", None)
    env.pop("HDB_DEDISP_TUNE", None)
    env.pop("HDB_TUNE_CACHE", None)
    if cache is not None:
        env["HDB_TUNE_CACHE"] = cache
    env.update(extra)
    out = subprocess.run([sys.executable, "-c", SCRIPT, ROOT, str(nsamps)], env=env,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_tile_choice_persists_across_processes(hdb, tmp_path):
    cache = str(tmp_path / "sub" / "tiles.txt")
    first = _run(cache)
    assert first["source"] == "autotuner"
    lines = open(cache).read().splitlines()
    assert len(lines) == 1
    key, db, tb, rows = lines[0].split()
    assert len(key) == 16 and [int(db), int(tb), int(rows)] == first["tile"]
    second = _run(cache)
    assert second["source"] == "tile cache"
    assert second["tile"] == first["tile"]
    assert second["cands"] == first["cands"] and len(first["cands"]) >= 1
    assert len(open(cache).read().splitlines()) == 1
    # another gulp length is another shape: timed again, a second line
    third = _run(cache, nsamps=(1 << 14) + 4096)
    assert third["source"] == "autotuner"
    assert len(open(cache).read().splitlines()) == 2


def test_tile_cache_off_and_default_location(hdb, tmp_path):
    """HDB_TUNE_CACHE=0: the default locations under the home and cache
    directories stay untouched; unset: the XDG cache directory is used."""
    r = _run("0", HOME=str(tmp_path), XDG_CACHE_HOME=str(tmp_path / "xdg"))
    assert r["source"] == "autotuner"
    assert not (tmp_path / "xdg" / "heimdall_b200").exists()
    assert not (tmp_path / ".cache" / "heimdall_b200").exists()
    # unset: the choice lands in the XDG cache directory
    unset = _run(None, HOME=str(tmp_path), XDG_CACHE_HOME=str(tmp_path / "xdg"))
    assert unset["source"] == "autotuner"
    assert len((tmp_path / "xdg" / "heimdall_b200" / "dedisp_tiles.txt").read_text().splitlines()) == 1
