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
    assert lrn.table_choice(10000) == (48, 1.0)
    assert lrn.table_choice(10000, 80) == (80, 1.0)
    assert lrn.nparams() == 25090


def test_learned_policy_gains_offline(pkg):
    """What the committed network gains over the fixed table, scored on the
    committed traces in deflations per device second at the nearest grid
    candidate: a gain on the decision points it was trained on (4 of every
    5 pencils), and at most a 5% loss on the held-out ones."""
    lrn = pkg.learned
    P = lrn.load_weights()
    if P is None:
        pytest.skip("no trained weights committed")
    tr = np.load(lrn.TRACES)
    grid = lrn.trace_grid(tr)
    hold = tr["pencil"] % 5 == 0
    g_train = lrn.offline_gain(P, tr["features"][~hold], tr["scores"][~hold], tr["nh"][~hold], grid)
    g_hold = lrn.offline_gain(P, tr["features"][hold], tr["scores"][hold], tr["nh"][hold], grid)
    print("offline gain over the table: train %.3f, held-out %.3f" % (g_train, g_hold))
    assert g_train > 1.0, g_train
    assert g_hold >= 0.95, g_hold
