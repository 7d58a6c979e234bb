"""The narrow-band RFI stage on the GPU (hd_set_narrow_band: the branch of
Pipeline/clean_filterbank_rfi.cu:303-351 the reference disables) against the
oracle, whose restatement equals the reference's own code for it
(tests/test_oracle_narrowband.py): the cleaned filterbank and mask bit for
bit, the candidates of whole gulps, and batched units equal to separate
calls."""
import os
import sys

import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from test_oracle_narrowband import narrowband_beam  # noqa: E402

pytestmark = pytest.mark.gpu

DT, F0 = 64e-6, 1500.0


@pytest.fixture
def narrow_oracle(oracle_lib):
    oracle.set_narrow_band(True)
    try:
        yield
    finally:
        oracle.set_narrow_band(False)


@pytest.mark.parametrize("nsamps,nchans", [(1 << 16, 256), (40000, 120), (20000, 1140)])
def test_clean_with_narrow_band_bit_exact(hdb, narrow_oracle, nsamps, nchans):
    fb = narrowband_beam(nsamps, nchans, 5)
    ref_out, ref_mask = oracle.clean_filterbank(fb, DT)
    with H.Pipeline(H.default_params(nchans=nchans, output_dir=None), narrow_band=True) as pl:
        out, mask = pl.clean_filterbank_rfi(fb, DT)
    np.testing.assert_array_equal(mask, ref_mask)
    np.testing.assert_array_equal(out, ref_out)
    # the narrow stage changed the data the broadband stage saw
    oracle.set_narrow_band(False)
    plain_out, _ = oracle.clean_filterbank(fb, DT)
    assert (plain_out != out).any()


def test_gulps_with_narrow_band(hdb, narrow_oracle):
    nchans, nsamps = 256, 1 << 16
    df = -1.5625
    kw = dict(dt=DT, f0=F0, df=df, dm_min=0.0, dm_max=300.0, boxcar_max=256)
    beams = []
    for b in range(3):
        x = narrowband_beam(nsamps, nchans, 10 + b).astype(np.float32)
        for t0, dm in ((15000.0 + 9000 * b, 150.0), (40000.0, 60.0 + 40 * b)):
            synth.inject_pulse(x, synth.Pulse(t0, dm, 1e-3, 30.0), DT, F0, df)
        beams.append(np.clip(np.rint(x), 0, 255).astype(np.uint8))
    p = H.default_params(nchans=nchans, output_dir=None, **kw)
    per_beam = []
    with H.Pipeline(p, cleaning=True, narrow_band=True) as pl:
        for fb in beams:
            err, proc = pl.execute(fb)
            per_beam.append(H.cand_lines(pl.candidates()))
        # same beam number for every unit, as the separate calls have
        err, _, st = pl.execute_beams(beams, beams=[0, 0, 0])
        batched = [H.cand_lines(pl.candidates(u)) for u in range(3)]
    assert batched == per_beam
    r = oracle.execute(beams[0], clean=1, **kw)
    lines = oracle.cand_lines(r["groups"], nsamps, 1, 0, r["nsamps_processed"], 256, DT)
    assert per_beam[0] == lines and len(lines) >= 2
