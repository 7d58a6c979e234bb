"""The cross-beam coincidence restatement (oracle.coincide) against the
reference's own coincidencer (Applications/Candidates.C, compiled into
oracle/_ref/coinc_ref) on synthetic per-beam candidate lists (no GPU)."""
import os
import sys

import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import coinc_data as D  # noqa: E402

pytestmark = pytest.mark.skipif(not oracle.ref_coinc_available(),
                                reason="oracle/_ref/coinc_ref is built from the reference "
                                       "(make -C oracle ref)")


@pytest.mark.parametrize("seed,sep_time,sep_filter", [(3, 3, 4), (4, 3, 4), (5, 1, 1),
                                                       (6, 6, 8)])
def test_restatement_matches_reference(hdb, tmp_path, seed, sep_time, sep_filter):
    bl = D.lines_by_beam(5, seed)
    files = D.write_files(tmp_path, bl)
    ref = oracle.ref_coincide(files, len(bl), sep_time, sep_filter)
    rows = [H.parse_cand_lines(ls) for ls in bl]
    co = oracle.coincide(rows, sep_time, sep_filter)
    mine = []
    for r, c in zip(rows, co):
        mine += D.format_all(r, c)
    assert mine == ref
    if sep_time == 3:
        # the boundary pair (|dt| = 3 * 2^2, S/N ratio exactly 0.4) is coincident
        r0 = rows[0]
        k = int(np.where((r0["samp_idx"] == 50000) & (r0["snr"] == 7.0))[0][0])
        assert co[0][k][0] >= 2
