"""The classifier's CPU checker (oracle/classifier.c) against independent
restatements and known answers (no GPU)."""
import numpy as np
import pytest

import oracle


def _np_normalise(row: np.ndarray) -> np.ndarray:
    """Applications/candidate_profiler.C:88-134 in numpy float32/float64, the
    same types and order as the reference (a zero deviation gives zeros)."""
    n = len(row)
    x = row.astype(np.float32).copy()
    m1 = np.sort(x[: n // 2])[n // 4]
    m2 = np.sort(x[n // 2:])[n // 4]
    grad = float(np.float32(np.float32(m2 - m1) / np.float32(n // 2)))
    m0 = np.float32(float(m1) - grad * (n // 4))
    base = np.array([np.float32(float(m0) + j * grad) for j in range(n)], np.float32)
    x = (x - base).astype(np.float32)
    mad = np.sort(np.abs(x))[n // 2]
    sd = np.float32(float(mad) * 1.4826)
    if not sd > 0:
        return np.zeros(n, np.float32)
    val = np.float32(1.0 / float(sd))
    return (x * val).astype(np.float32)


@pytest.mark.parametrize("n", [64, 256])
def test_normalise_rows_bit_exact(oracle_lib, n):
    rng = np.random.default_rng(n)
    rows = (rng.standard_normal((20, n)) * 7 + np.linspace(0, 30, n)).astype(np.float32)
    rows[3] = 5.0  # constant row: zero deviation
    got = oracle.normalise_rows(rows)
    for r in range(rows.shape[0]):
        np.testing.assert_array_equal(got[r], _np_normalise(rows[r]), err_msg=f"row {r}")
    assert np.all(got[3] == 0)


def test_patch_dm_impulse(oracle_lib):
    """A unit impulse at sample 500 of DM trial 10: the patch's row 32 (the
    candidate's trial) peaks at column 32 for width 1 and is the only
    non-flat row."""
    D, n = 40, 2000
    x = np.zeros((D, n), np.float32)
    x[10, 500] = 1.0
    x += np.random.default_rng(1).standard_normal((D, n)).astype(np.float32) * 1e-3
    scans = np.zeros((D, n + 1), np.float32)
    for d in range(D):
        scans[d, 1:] = np.cumsum(x[d], dtype=np.float32)
    p = oracle.patch_dm(scans, dm=10, ind=500, filt=0)
    assert int(np.argmax(p[32])) == 32
    assert p[32].max() > 10 * np.abs(p[33]).max()
    # rows for trials below 0 are zero
    assert np.all(p[:22] == 0)


def test_patch_ft_shows_the_sweep(oracle_lib):
    """A dispersed pulse: the brightest time bin moves later from the top
    sub-band to the bottom one (the dispersion sweep of the undispersed
    data); a zero-DM burst lies at one time bin in every sub-band."""
    from heimdall_multibeam_b200 import synth
    w = synth.TRAIN
    dm = 300.0
    b = synth.make_beam(w.nsamps, w.nchans, w.dt, w.f0, w.df,
                        [synth.Pulse(9000.0, dm, 2e-3, 200.0)], seed=5)
    table = oracle.delay_table(w.nchans, w.dt, w.f0, w.df)
    md = int(oracle.delays(np.array([dm], np.float32), table).max())
    p = oracle.patch_ft(b.data, md, 9000, 2)
    peaks = np.argmax(p, axis=1)
    assert np.corrcoef(np.arange(64), peaks)[0, 1] > 0.9
    x = b.data.astype(np.float32)
    x[20000:20004] += 100
    q = oracle.patch_ft(np.clip(x, 0, 255).astype(np.uint8), 0, 20001, 0)
    # window starts 128 bins before sample 20001: the burst is bins 127..130
    assert set(np.argmax(q, axis=1).tolist()) <= {127, 128, 129, 130}


def test_cnn_gradient_finite_differences(oracle_lib):
    """Head parameters (FC2 weights and biases, FC1 biases) against central
    differences of the loss; these enter in FP32, after every BF16 rounding."""
    rng = np.random.default_rng(3)
    npar = oracle.cnn_param_count()
    assert npar == 175666
    params = (rng.standard_normal(npar) * 0.05).astype(np.float32)
    n = 3
    dm = rng.standard_normal((n, 64, 64)).astype(np.float32)
    ft = rng.standard_normal((n, 64, 256)).astype(np.float32)
    lab = np.array([1, 0, 1], np.int32)
    _, g, loss = oracle.cnn_run(params, dm, ft, lab)
    assert np.isfinite(loss) and np.all(np.isfinite(g))
    nhead = 16 + 32 + 2
    idx = list(range(npar - nhead, npar))
    eps = 1e-2
    for i in idx[::3]:
        p1 = params.copy(); p1[i] += eps
        p0 = params.copy(); p0[i] -= eps
        l1 = oracle.cnn_run(p1, dm, ft, lab)[2]
        l0 = oracle.cnn_run(p0, dm, ft, lab)[2]
        fd = (l1 - l0) / (2 * eps)
        assert abs(fd - g[i]) <= 2e-3 + 2e-2 * abs(g[i]), (i, fd, g[i])
