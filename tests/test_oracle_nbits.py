"""Packed and 16-bit input (nbits = 1, 2, 4, 16) on the CPU.

* The packing order of synth.pack_filterbank against the reference's own
  writer, restated loop for loop (Formats/giant_maker.C:258-262,385-392:
  channel c into the unsigned 32-bit word c / chans_per_word at bit
  (c % chans_per_word) * nbits).
* The reference's own pipeline (oracle/_ref, the shipped build without
  cleaning, over the restated dedisp) on packed data writes the same .cand
  lines as on the same sample values given as bytes: hd_execute passes
  nbits to dedisp (Pipeline/pipeline.cu:453-462), which sums sample values
  whatever their width.
"""
import numpy as np
import pytest

import oracle
from heimdall_multibeam_b200 import synth

needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference build (oracle/_ref) not present")


def _giant_maker_pack(values, nbits):
    nsamps, nchans = values.shape
    cpw = 32 // nbits
    q = np.zeros((nsamps, nchans // cpw), dtype=np.uint32)
    for t in range(nsamps):
        for c in range(nchans):
            q[t, c // cpw] |= np.uint32(int(values[t, c]) << ((c % cpw) * nbits))
    return q.astype("<u4").view(np.uint8).reshape(nsamps, -1)


@pytest.mark.parametrize("nbits", [1, 2, 4, 8, 16])
def test_pack_order_matches_reference_writer(nbits):
    rng = np.random.default_rng(nbits)
    v = rng.integers(0, 1 << nbits, size=(7, 64))
    np.testing.assert_array_equal(synth.pack_filterbank(v, nbits), _giant_maker_pack(v, nbits))


def test_pack_rejects_bad_shapes():
    with pytest.raises(ValueError):
        synth.pack_filterbank(np.zeros((4, 20), np.uint8), 2)  # 40 bits per spectrum
    with pytest.raises(ValueError):
        synth.pack_filterbank(np.full((4, 32), 4, np.uint8), 2)  # value >= 2^nbits


def _quantised_beam(nbits):
    """The single-beam workload's samples requantised to nbits (the top
    bits of each byte; 16 bits: the byte value, so the search matches the
    8-bit one exactly)."""
    w = synth.SEARCH_C0
    b = synth.make_beam(1 << 14, 64, w.dt, w.f0, w.df * 4,
                        [synth.Pulse(3000.0, 150.0, 1e-3, 40.0),
                         synth.Pulse(9000.0, 60.0, 2e-3, 30.0)], seed=40 + nbits)
    v = b.data if nbits >= 8 else (b.data >> (8 - nbits))
    kw = dict(dt=w.dt, f0=w.f0, df=w.df * 4, dm_min=0.0, dm_max=300.0, boxcar_max=256)
    return v.astype(np.uint16 if nbits == 16 else np.uint8), kw


@needs_ref
@pytest.mark.parametrize("nbits", [1, 2, 4, 16])
def test_reference_pipeline_packed_equals_bytes(oracle_lib, nbits):
    v, kw = _quantised_beam(nbits)
    packed = synth.pack_filterbank(v, nbits)
    err, proc, lines, _ = oracle.ref_execute(packed, nbits=nbits, nchans=v.shape[1],
                                             nthreads=1, **kw)
    err8, proc8, lines8, _ = oracle.ref_execute(v.astype(np.uint8), nthreads=1, **kw)
    assert err == err8 == 0 and proc == proc8
    assert lines == lines8
    if nbits >= 4:
        assert len(lines) >= 1
