"""Pins the oracle's C restatement of the reference path (oracle/qzref.c)
against LAPACK DHGEQZ: backward errors and orthogonality <= 50*n*eps,
standardised Schur form, eigenvalue sets within the condition-scaled
chordal tolerance.  CPU only."""
import numpy as np
import pytest

from conftest import EPS


@pytest.fixture(scope="module")
def qzref():
    from oracle import qzref as R
    R.lib()
    return R


@pytest.mark.parametrize("n,seed,zf,kind", [(1, 0, 0.0, "r"), (2, 1, 0.0, "r"), (40, 2, 0.0, "r"),
                                             (230, 3, 0.05, "r"), (300, 4, 0.0, "g"), (400, 5, 0.0, "c"),
                                             (600, 6, 0.0, "r")])
def test_restatement_matches_lapack(pkg, lapack, qzref, n, seed, zf, kind):
    P_ = pkg.pencils
    if kind == "g":
        H, T = P_.graded_ht(n, seed)
    elif kind == "c":
        H, T = P_.clustered_ht(n, seed)
    else:
        H, T = P_.random_ht(n, seed, zf)
    S, P, Q, Z, ar, ai, be, info, st = qzref.pdhgeqz(H, T, nb=60)
    assert info == 0
    r = lapack.residuals(H, T, S, P, Q, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])
    assert lapack.schur_structure_ok(S, P)
    So, Po, lar, lai, lbe, _, _, _ = lapack.dhgeqz(H, T)
    tol = lapack.eig_tolerance(So, Po, H, T)
    ok, ratio, _ = lapack.match_eigenvalues((lar, lai, lbe), (ar, ai, be), tol)
    assert ok, ratio
    if n >= 300:
        assert st["aeds"] > 0  # the AED path really ran
    if n >= 600:
        assert st["sweeps"] > 0  # and the multishift sweep


def test_restatement_sweep_is_orthogonal_equivalence(pkg, qzref):
    n = 60
    H, T = pkg.pencils.random_ht(n, 9)
    rng = np.random.default_rng(1)
    sr = rng.standard_normal(8)
    si = np.zeros(8)
    sb = np.ones(8)
    S, P, Q, Z = qzref.sweep(H, T, sr, si, sb)
    assert np.linalg.norm(Q @ S @ Z.T - H) <= 50 * n * EPS * np.linalg.norm(H)
    # introduction then chase equals the whole sweep
    H1, T1, Q1, Z1 = qzref.sweep(H, T, sr, si, sb, phase=1)
    S2, P2, Q2, Z2 = qzref.sweep(H1, T1, sr, si, sb, phase=2)
    assert np.allclose(S2, S, rtol=0, atol=1e-12 * np.linalg.norm(S))
    assert np.linalg.norm(Q @ P @ Z.T - T) <= 50 * n * EPS * np.linalg.norm(T)
    assert np.all(np.tril(S, -2) == 0) and np.all(np.tril(P, -1) == 0)
