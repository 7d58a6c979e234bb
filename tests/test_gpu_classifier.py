"""GPU classifier: the BF16 tensor-core GEMM against numpy, the candidate
patches against the oracle (bit-exact), the network's forward pass and
gradients against the CPU network (oracle/classifier.c), and training on
candidates the pipeline itself produces.

Tolerances: the GEMMs accumulate BF16 products in FP32 (relative error
~1e-6 of the operands' scale, asserted at 1e-4); the tensor-core GEMM
(tcgen05, hd_bf16_gemm_tc) is also checked for the same bits on a second run;
the network's gradients
agree with the CPU network (double sums, same BF16 rounding points) to 3e-2
relative L2 per parameter tensor and its probabilities to 2e-3, because a
different FP32 summation order can move an activation across a BF16 rounding
boundary."""
import numpy as np
import pytest

import heimdall_multibeam_b200 as H
import oracle
from heimdall_multibeam_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _bf16(shape, rng):
    return torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).to(torch.bfloat16).cuda()


@pytest.mark.parametrize("case", ["nn", "tn", "nt", "splitk"])
def test_gemm_matches_numpy(hdb, case):
    rng = np.random.default_rng(11)
    M, N, K = 40, 300, 1000
    if case == "nn":      # A [M][K], B [K][N]
        A, B = _bf16((M, K), rng), _bf16((K, N), rng)
        sa, sb = (K, 1), (N, 1)
        a, b = A.float().cpu().numpy(), B.float().cpu().numpy()
    elif case == "tn":    # A stored [K][M]
        A, B = _bf16((K, M), rng), _bf16((K, N), rng)
        sa, sb = (1, M), (N, 1)
        a, b = A.float().cpu().numpy().T, B.float().cpu().numpy()
    else:                 # B stored [N][K]
        A, B = _bf16((M, K), rng), _bf16((N, K), rng)
        sa, sb = (K, 1), (1, K)
        a, b = A.float().cpu().numpy(), B.float().cpu().numpy().T
    ref = a.astype(np.float64) @ b.astype(np.float64)
    Cd = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    splits = 8 if case == "splitk" else 1
    err = H.lib().hd_bf16_gemm(M, N, K, A.data_ptr(), sa[0], sa[1], B.data_ptr(), sb[0], sb[1],
                               H.C.cast(Cd.data_ptr(), H.C.POINTER(H.C.c_float)), N, 1, 0, splits)
    assert err == H.HD_NO_ERROR
    got = Cd.cpu().numpy()
    scale = np.abs(a).max() * np.abs(b).max() * np.sqrt(K)
    assert np.abs(got - ref).max() <= 1e-4 * scale


@pytest.mark.parametrize("M,N,K,splits,acc", [
    (1000, 16, 80, 1, 0),        # conv layer 2 shape: M tail, K = 80 (one partial block)
    (333, 32, 144, 1, 1),        # conv layer 3 shape, accumulate into C
    (12305, 8, 16, 1, 0),        # conv layer 1 shape: N = 8 padded to 16, K = 16
    (256, 16, 10240, 64, 0),     # fully connected layer: split K
    (144, 32, 65536, 37, 1),     # weight gradient: K = pixels, 37 splits, accumulate
    (200, 128, 512, 3, 0),       # widest N, splits that do not divide the K blocks
])
def test_gemm_tensor_cores_match_numpy(hdb, M, N, K, splits, acc):
    """hd_bf16_gemm_tc (tcgen05.mma, TMEM accumulators, TMA-staged K-major
    operands) against float64 products of the same BF16 values, and the same
    bits on a second run (split K is reduced in a fixed order)."""
    rng = np.random.default_rng(M + N + K)
    A, B = _bf16((M, K), rng), _bf16((N, K), rng)
    a, b = A.float().cpu().numpy(), B.float().cpu().numpy()
    c0 = rng.standard_normal((N, M)).astype(np.float32)
    ref = (a.astype(np.float64) @ b.astype(np.float64).T).T + (c0 if acc else 0.0)
    outs = []
    for _ in range(2):
        Cd = torch.from_numpy(c0.copy()).cuda()  # C(m, n) at n * M + m
        err = H.lib().hd_bf16_gemm_tc(M, N, K, A.data_ptr(), K, 1, B.data_ptr(), 1, K,
                                      H.C.cast(Cd.data_ptr(), H.C.POINTER(H.C.c_float)), 1, M,
                                      acc, splits)
        assert err == H.HD_NO_ERROR, H.error_string(err)
        outs.append(Cd.cpu().numpy())
    scale = np.abs(a).max() * np.abs(b).max() * np.sqrt(K)
    assert np.abs(outs[0] - ref).max() <= 1e-4 * scale
    np.testing.assert_array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


def test_gemm_tensor_cores_reject_unsupported(hdb):
    """Operands that are not K-major, or N above 128, are refused."""
    rng = np.random.default_rng(3)
    A, B = _bf16((64, 64), rng), _bf16((200, 64), rng)
    Cd = torch.zeros((64, 200), dtype=torch.float32, device="cuda")
    cp = H.C.cast(Cd.data_ptr(), H.C.POINTER(H.C.c_float))
    assert H.lib().hd_bf16_gemm_tc(64, 200, 64, A.data_ptr(), 64, 1, B.data_ptr(), 1, 64, cp,
                                   200, 1, 0, 1) == H.HD_INVALID_STRIDE
    assert H.lib().hd_bf16_gemm_tc(64, 64, 64, A.data_ptr(), 1, 64, B.data_ptr(), 1, 64, cp,
                                   64, 1, 0, 1) == H.HD_INVALID_STRIDE


def test_patches_match_oracle(hdb, oracle_lib):
    w = synth.SEARCH_C0
    b = synth.make_c0()
    kw = dict(dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min, dm_max=w.dm_max,
              boxcar_max=w.boxcar_max)
    with H.Pipeline(H.default_params(nchans=w.nchans, output_dir=None, **kw), cleaning=False) as pl:
        pl.execute(b.data)
        cands = pl.candidates()
        dm, ft = pl.patches()
    assert len(cands) >= 3 and dm.shape == (len(cands), 64, 64)
    r, scans, dms, table = oracle.execute_with_scans(b.data, clean=0, **kw)
    for i, c in enumerate(cands):
        d, ind, f = int(c["dm_trial"]), int(c["samp_idx"]), int(c["filter"])
        np.testing.assert_array_equal(dm[i], oracle.patch_dm(scans, d, ind, f), err_msg=f"dm {i}")
        md = int(oracle.delays(dms[d:d + 1], table).max())
        np.testing.assert_array_equal(ft[i], oracle.patch_ft(b.data, md, ind, f), err_msg=f"ft {i}")


def test_score_candidates_matches_host_path(hdb):
    """hd_score_candidates (patches extracted and scored on the GPU) gives the
    same scores as hd_extract_patches + hd_classifier_score through host
    memory, and hd_classifier_score_device the same on device patches."""
    w = synth.SEARCH_C0
    b = synth.make_c0()
    kw = dict(dt=w.dt, f0=w.f0, df=w.df, dm_min=w.dm_min, dm_max=w.dm_max,
              boxcar_max=w.boxcar_max)
    with H.Pipeline(H.default_params(nchans=w.nchans, output_dir=None, **kw), cleaning=False) as pl, \
            H.Classifier(seed=7) as clf:
        pl.execute(b.data)
        n = len(pl.candidates())
        assert n >= 3
        fused = pl.scores(clf)
        dm, ft = pl.patches()
        host = clf.score(dm, ft)
        ddm = torch.from_numpy(dm).cuda()
        dft = torch.from_numpy(ft).cuda()
        torch.cuda.synchronize()
        dev = clf.score_device(ddm.data_ptr(), dft.data_ptr(), n)
    assert fused.shape == (n,)
    np.testing.assert_array_equal(fused, host)
    np.testing.assert_array_equal(dev, host)
    assert np.all((fused >= 0) & (fused <= 1))


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)


def test_forward_and_gradients_match_oracle(hdb, oracle_lib):
    rng = np.random.default_rng(21)
    n = 4
    dm = rng.standard_normal((n, 64, 64)).astype(np.float32)
    ft = rng.standard_normal((n, 64, 256)).astype(np.float32)
    dm[1, 30:34, 30:34] += 6.0
    ft[2, :, 100:104] += 4.0
    lab = np.array([0, 1, 1, 0], np.int32)
    with H.Classifier(seed=5) as clf:
        params = clf.params()
        assert params.size == oracle.cnn_param_count() == 175666
        g, loss = clf.gradients(dm, ft, lab)
        probs = clf.score(dm, ft)
    p_cpu, g_cpu, loss_cpu = oracle.cnn_run(params, dm, ft, lab)
    assert abs(loss - loss_cpu) <= 2e-3 * abs(loss_cpu)
    np.testing.assert_allclose(probs, p_cpu, atol=2e-3)
    # per tensor: conv layers (W, b) x 6, W1, b1, W2, b2
    sizes = []
    for ci, co in [(1, 8), (8, 16), (16, 32)] * 2:
        sizes += [co * ci * 9, co]
    sizes += [16 * 10240, 16, 32, 2]
    o = 0
    for k, s in enumerate(sizes):
        assert _rel(g[o:o + s], g_cpu[o:o + s]) < 3e-2, (k, _rel(g[o:o + s], g_cpu[o:o + s]))
        o += s
    assert o == params.size


def test_gradients_and_training_reproducible(hdb):
    """Every reduction of the backward pass runs in a fixed order (split-K
    weight gradients added split by split, bias and head gradients summed
    sample by sample), so the same batch gives the same gradient bits, and
    the same training run the same weights."""
    rng = np.random.default_rng(8)
    n = 64
    dm = rng.standard_normal((n, 64, 64)).astype(np.float32)
    ft = rng.standard_normal((n, 64, 256)).astype(np.float32)
    lab = (rng.random(n) < 0.5).astype(np.int32)
    runs = []
    for _ in range(2):
        with H.Classifier(seed=9) as clf:
            g, loss = clf.gradients(dm, ft, lab)
            clf.train(dm, ft, lab, epochs=2, batch=32, seed=4)
            runs.append((g, np.float32(loss), clf.params()))
    np.testing.assert_array_equal(runs[0][0].view(np.uint32), runs[1][0].view(np.uint32))
    assert runs[0][1] == runs[1][1]
    np.testing.assert_array_equal(runs[0][2].view(np.uint32), runs[1][2].view(np.uint32))


def test_training_keeps_pulses_and_rejects_rfi(hdb):
    """Trained on candidates the pipeline produces from seeded gulps (4
    injected pulses and 2 RFI events each: zero-DM bursts, narrowband bursts,
    baseline drifts; cleaning off), the classifier must keep >= 99 % of the
    plain candidate list's recall of injected S/N >= 8 pulses at a score
    threshold that removes >= 90 % of the RFI candidates (held-out gulps)."""
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import classifier_data as CD
    tr, _ = CD.build(range(0, 320))
    ev, pev = CD.build(range(1000, 1120))
    assert tr["label"].sum() > 500 and tr["rfi"].sum() > 2000
    rng = np.random.default_rng(0)
    pos = np.where(tr["label"] == 1)[0]
    neg = np.where(tr["label"] == 0)[0]
    neg = rng.choice(neg, size=min(len(neg), 2 * len(pos)), replace=False)
    sel = np.concatenate([pos, neg])
    with H.Classifier(seed=1) as clf:
        losses = clf.train(tr["dm"][sel], tr["ft"][sel], tr["label"][sel], epochs=40, batch=32,
                           lr=3e-4)
        assert losses[-1] < 0.5 * losses[0]
        scores = clf.score(ev["dm"], ev["ft"])
    ok = None
    for th in (0.005, 0.01, 0.02, 0.05, 0.1, 0.2, 0.3, 0.5):
        r0, r1, kept_other, kept_rfi, total = CD.recall_and_reduction(ev, pev, scores, th)
        if kept_rfi <= 0.1:
            ok = (th, r0, r1, kept_rfi, total)
            break
    assert ok is not None, "no threshold removes 90 % of the RFI candidates"
    th, r0, r1, kept_rfi, total = ok
    print(f"threshold {th}: plain recall {r0:.4f}, classified {r1:.4f} of {total} pulses, "
          f"RFI kept {kept_rfi:.4f}")
    assert r0 > 0.9
    assert r1 >= 0.99 * r0
