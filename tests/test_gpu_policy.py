"""Learned (nw, ns) policy on the GPU: the hand-written forward, backward
and training kernels against the numpy restatement of the MLP (FP32, so
relative tolerance 1e-4), the feature kernel against its numpy
restatement, and a full solve driven by the network, which must keep the
backward error <= 50*n*eps (a prediction can only change the speed)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def test_mlp_forward_backward_match_numpy(pkg):
    import torch
    lrn = pkg.learned
    L = pkg.lib()
    rng = np.random.default_rng(3)
    B = 37
    P = lrn.init_params(5)
    P[lrn.NHID * lrn.NIN:lrn.NHID * lrn.NIN + lrn.NHID] = rng.standard_normal(lrn.NHID) * 0.1
    X = rng.random((B, lrn.NIN)).astype(np.float32)
    T = rng.random((B, lrn.NOUT)).astype(np.float32)
    p, x, t = _dev(torch, P), _dev(torch, X), _dev(torch, T)
    a1 = torch.empty(B, lrn.NHID, device="cuda")
    a2 = torch.empty(B, lrn.NHID, device="cuda")
    y = torch.empty(B, lrn.NOUT, device="cuda")
    dy = torch.empty(B, lrn.NOUT, device="cuda")
    d2 = torch.empty(B, lrn.NHID, device="cuda")
    d1 = torch.empty(B, lrn.NHID, device="cuda")
    g = torch.empty(P.size, device="cuda")
    vp = lambda z: ctypes.c_void_p(z.data_ptr())
    assert L.b200qz_mlp_forward(vp(p), vp(x), B, vp(a1), vp(a2), vp(y), None) == 0
    assert L.b200qz_mlp_backward(vp(p), vp(x), vp(t), B, vp(a1), vp(a2), vp(y), vp(dy), vp(d2), vp(d1), vp(g),
                                 None) == 0
    torch.cuda.synchronize()
    A1, A2, Y = lrn.forward_np(P, X)
    G = lrn.backward_np(P, X, T)
    assert np.allclose(y.cpu().numpy(), Y, rtol=1e-4, atol=1e-5)
    assert np.allclose(a2.cpu().numpy(), A2, rtol=1e-4, atol=1e-5)
    gg = g.cpu().numpy()
    assert np.allclose(gg, G, rtol=1e-4, atol=1e-6 * np.abs(G).max())


def test_mlp_training_reduces_loss(pkg):
    lrn = pkg.learned
    rng = np.random.default_rng(4)
    X = rng.random((200, lrn.NIN)).astype(np.float32)
    T = np.stack([X[:, :8].mean(1), X[:, 8:16].mean(1)], 1).astype(np.float32)
    P0 = lrn.init_params(2)
    l0 = lrn.loss_np(P0, X, T)
    P1, l1 = lrn.train_device(P0, X, T, epochs=500, lr=1e-3)
    assert abs(l1 - lrn.loss_np(P1, X, T)) <= 1e-4 * max(1.0, l1)
    assert l1 < 0.05 * l0, (l0, l1)


def test_feature_kernel_matches_numpy(pkg):
    import torch
    lrn = pkg.learned
    H, T = pkg.pencils.clustered_ht(700, 11, every=50, scale=1e-8)
    H[300, 299] = 0.0
    dH = torch.from_numpy(np.ascontiguousarray(H.T)).cuda()
    s = pkg.Solver(0)
    try:
        for ktop, kbot, fr in ((0, 699, 0.0), (120, 650, 0.25), (10, 12, 1.0)):
            f = s.policy_features(dH.data_ptr(), 700, ktop, kbot, fr)
            ref = lrn.features_np(H, ktop, kbot, fr)
            assert np.allclose(f, ref, rtol=1e-5, atol=1e-6), (ktop, kbot, np.abs(f - ref).max())
    finally:
        s.close()


def test_policy_driven_solve_is_backward_stable(pkg, lapack):
    lrn = pkg.learned
    P = lrn.load_weights()
    if P is None:
        P = lrn.init_params(7)  # an untrained network is still a valid policy
    n = 1500
    H, T = pkg.pencils.clustered_ht(n, 21, every=50, scale=1e-8)
    S, Pm, Q, Z = (np.array(M, order="F", copy=True) for M in (H, T, np.eye(n), np.eye(n)))
    s = pkg.Solver(0)
    try:
        s.set_policy(P)
        ar, ai, be, info = s.solve_host(S, Pm, Q, Z)
        st = s.stats()
    finally:
        s.close()
    assert info == 0
    assert st["policy_calls"] > 0
    r = lapack.residuals(H, T, S, Pm, Q, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])
    assert lapack.schur_structure_ok(S, Pm)
