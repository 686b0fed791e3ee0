"""End-to-end parity of the GPU solver against the FP64 LAPACK DHGEQZ
oracle: backward errors and orthogonality <= 50*n*eps, generalized Schur
structure, and eigenvalue sets matched in the chordal metric within
50*n*eps*||(H,T)||_F / s_j (s_j: DTGSNA reciprocal condition numbers)."""
import numpy as np
import pytest

from conftest import EPS

pytestmark = pytest.mark.gpu


def check(lapack, H, T, S, P, Q, Z, ar, ai, be, info, eig=True):
    assert info == 0
    r = lapack.residuals(H, T, S, P, Q, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])
    assert lapack.schur_structure_ok(S, P)
    e = lapack.eig_from_schur(S, P)
    assert np.allclose(e[0], ar, rtol=1e-12, atol=1e-300) and np.allclose(e[2], be, rtol=1e-12, atol=1e-300)
    assert np.all(be >= 0)
    if eig:
        So, Po, lar, lai, lbe, _, _, _ = lapack.dhgeqz(H, T)
        tol = lapack.eig_tolerance(So, Po, H, T)
        ok, ratio, _ = lapack.match_eigenvalues((lar, lai, lbe), (ar, ai, be), tol)
        assert ok, ratio


@pytest.mark.parametrize("n,seed,zf,kind", [
    (1, 0, 0.0, "r"), (2, 1, 0.0, "r"), (3, 2, 0.0, "r"), (50, 3, 0.0, "r"), (81, 4, 0.0, "r"),
    (200, 5, 0.0, "r"), (400, 6, 0.05, "r"), (300, 7, 0.0, "g"), (500, 8, 0.0, "c"), (1000, 0, 0.0, "r")])
def test_solve_matches_lapack(pkg, lapack, n, seed, zf, kind):
    P_ = pkg.pencils
    if kind == "g":
        H, T = P_.graded_ht(n, seed)
    elif kind == "c":
        H, T = P_.clustered_ht(n, seed)
    else:
        H, T = P_.random_ht(n, seed, zf)
    S, P, Q, Z, ar, ai, be, info = pkg.solve(H, T)
    check(lapack, H, T, S, P, Q, Z, ar, ai, be, info)
    if zf > 0:
        # adjacent zeros on T's diagonal can carry fewer infinite
        # eigenvalues than zeros: count against LAPACK's exact zeros
        lbe = lapack.dhgeqz(H, T)[4]
        assert np.sum(be == 0) >= np.sum(lbe == 0) > 0


def test_pdhgeqz_dropin_accumulates_V(pkg, lapack):
    """COMPQ=COMPZ='V': Q1*H*Z1^T = Q*S*Z^T with Q1, Z1 on entry."""
    n = 150
    H, T = pkg.pencils.random_ht(n, 11)
    rng = np.random.default_rng(0)
    Q1 = np.asfortranarray(np.linalg.qr(rng.standard_normal((n, n)))[0])
    Z1 = np.asfortranarray(np.linalg.qr(rng.standard_normal((n, n)))[0])
    S, P, Q, Z = H.copy(order="F"), T.copy(order="F"), Q1.copy(order="F"), Z1.copy(order="F")
    pkg.kkqzconf()
    ar, ai, be, info = pkg.pdhgeqz("S", "V", "V", S, P, Q, Z, nb=64)
    assert info == 0
    r = lapack.residuals(H, T, S, P, Q, Z, Q0=Q1, Z0=Z1)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])


def test_pdhgeqz_dropin_ilo_ihi(pkg, lapack):
    """Rows/cols outside ILO:IHI already triangular (PDHGEQZ.f:155-161)."""
    n, ilo, ihi = 120, 11, 100
    H, T = pkg.pencils.random_ht(n, 12)
    H[ilo - 1, ilo - 2] = 0.0
    H[ihi, ihi - 1] = 0.0
    H[np.arange(1, ilo - 1), np.arange(0, ilo - 2)] = 0.0
    H[np.arange(ihi + 1, n), np.arange(ihi, n - 1)] = 0.0
    S, P, Q, Z = H.copy(order="F"), T.copy(order="F"), np.eye(n, order="F"), np.eye(n, order="F")
    ar, ai, be, info = pkg.pdhgeqz("S", "I", "I", S, P, Q, Z, ilo=ilo, ihi=ihi)
    check(lapack, H, T, S, P, Q, Z, ar, ai, be, info)


def test_compq_n_eigenvalues_only(pkg, lapack):
    n = 200
    H, T = pkg.pencils.random_ht(n, 13)
    S, P = H.copy(order="F"), T.copy(order="F")
    ar, ai, be, info = pkg.pdhgeqz("E", "N", "N", S, P, None, None)
    assert info == 0
    So, Po, lar, lai, lbe, _, _, _ = lapack.dhgeqz(H, T)
    tol = lapack.eig_tolerance(So, Po, H, T)
    ok, ratio, _ = lapack.match_eigenvalues((lar, lai, lbe), (ar, ai, be), tol)
    assert ok, ratio


@pytest.mark.parametrize("scale", [1e-200, 1e150])
def test_solve_with_T_far_from_H(pkg, lapack, scale):
    """T scaled far from H: the library balances T by a power of two for the
    iteration (shift polynomials stay in range) and undoes it at the end."""
    n = 200
    H, T = pkg.pencils.random_ht(n, 31)
    T = T * scale
    S, P, Q, Z, ar, ai, be, info = pkg.solve(H, T)
    check(lapack, H, T, S, P, Q, Z, ar, ai, be, info)
