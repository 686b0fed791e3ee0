"""Learned (nw, ns) policy, host side: the numpy restatement of the MLP
(the reference for the CUDA kernels) against finite differences, the
output decoding, and the offline gain of the committed network on the
committed traces."""
import numpy as np
import pytest


def test_numpy_gradient_matches_finite_differences(pkg):
    lrn = pkg.learned
    rng = np.random.default_rng(0)
    P = lrn.init_params(1).astype(np.float64)
    X = rng.random((7, lrn.NIN))
    T = rng.random((7, lrn.NOUT))
    g = lrn.backward_np(P, X, T)
    idx = rng.choice(P.size, 60, replace=False)
    idx = np.concatenate([idx, [P.size - 1, P.size - 2, lrn.NHID * lrn.NIN]])  # output and first-layer biases
    h = 1e-6
    for i in idx:
        e = np.zeros_like(P)
        e[i] = h
        fd = (lrn.loss_np(P + e, X, T) - lrn.loss_np(P - e, X, T)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_decode_and_table(pkg):
    lrn = pkg.learned
    assert lrn.decode([0.0, 0.0], 10000) == (16, 2)
    assert lrn.decode([1.0, 1.0], 10000) == (80, 80)
    assert lrn.decode([2.0, 0.5], 50) == (50, 40)
    assert lrn.decode([0.5, 0.5], 10000) == (48, 24)
    assert lrn.table_choice(10000) == (80, 1.0)
    assert lrn.nparams() == 25090


def test_learned_policy_gains_offline(pkg):
    """On held-out decision points (every 5th training pencil), the trained
    network's (nw, ns) scores at least as many deflations per flop as the
    fixed table's choice, on average."""
    lrn = pkg.learned
    P = lrn.load_weights()
    if P is None:
        pytest.skip("no trained weights committed")
    tr = np.load(lrn.TRACES)
    hold = tr["pencil"] % 5 == 0
    g = lrn.offline_gain(P, tr["features"][hold], tr["scores"][hold], tr["nh"][hold])
    assert g >= 1.0, g
