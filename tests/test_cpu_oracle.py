"""CPU tests of the LAPACK oracle wrapper and of the seeded generators."""
import numpy as np
import pytest

from conftest import EPS


def test_generators_shapes_and_structure(pkg):
    P = pkg.pencils
    H, T = P.random_ht(50, 0)
    assert H.flags.f_contiguous and T.flags.f_contiguous
    assert np.all(np.tril(H, -2) == 0) and np.all(np.tril(T, -1) == 0)
    assert np.all(np.diag(H, -1) != 0)
    H2, T2 = P.random_ht(50, 0)
    assert np.array_equal(H, H2) and np.array_equal(T, T2)
    _, Tz = P.random_ht(400, 1, zero_frac=0.05)
    assert np.sum(np.diag(Tz) == 0) == 20
    Hg, Tg = P.graded_ht(60, 2)
    assert np.all(np.tril(Hg, -2) == 0) and np.all(np.tril(Tg, -1) == 0)
    assert np.max(np.abs(Hg)) / np.min(np.abs(np.diag(Hg, -1))) > 1e3
    Hc, _ = P.clustered_ht(200, 3)
    assert abs(Hc[50, 49]) < 1e-6
    sizes = P.batch_sizes(2048, 4)
    assert sizes.min() >= 32 and sizes.max() <= 512


@pytest.mark.parametrize("n,zf", [(40, 0.0), (120, 0.05)])
def test_lapack_dhgeqz_oracle(lapack, pkg, n, zf):
    H, T = pkg.pencils.random_ht(n, 7, zf)
    S, P, ar, ai, be, Q, Z, info = lapack.dhgeqz(H, T)
    assert info == 0
    r = lapack.residuals(H, T, S, P, Q, Z)
    assert r["h"] <= 50 * r["neps"] and r["t"] <= 50 * r["neps"]
    assert r["q"] <= 50 * r["neps"] and r["z"] <= 50 * r["neps"]
    assert lapack.schur_structure_ok(S, P)
    e = lapack.eig_from_schur(S, P)
    tol = lapack.eig_tolerance(S, P, H, T)
    ok, ratio, _ = lapack.match_eigenvalues((ar, ai, be), e, tol)
    assert ok, ratio
    assert np.sum(be == 0) == round(zf * n)


def test_matching_detects_wrong_eigenvalue(lapack, pkg):
    H, T = pkg.pencils.random_ht(30, 3)
    S, P, ar, ai, be, Q, Z, info = lapack.dhgeqz(H, T)
    tol = lapack.eig_tolerance(S, P, H, T)
    bad = ar.copy()
    j = int(np.argmax(np.abs(be)))
    bad[j] += 1e-3 * max(1.0, abs(be[j]))
    ok, ratio, _ = lapack.match_eigenvalues((ar, ai, be), (bad, ai, be), tol)
    assert not ok and ratio > 1.0


def test_residuals_detect_perturbation(lapack, pkg):
    H, T = pkg.pencils.random_ht(30, 4)
    S, P, ar, ai, be, Q, Z, info = lapack.dhgeqz(H, T)
    S[0, 5] += 1e-10
    r = lapack.residuals(H, T, S, P, Q, Z)
    assert r["h"] > 50 * r["neps"]


@pytest.mark.parametrize("n", [30, 150])
def test_lapack_ht_reductions_agree(lapack, n):
    """The two LAPACK Hessenberg-triangular reductions the tests and the
    bench use: DGGHRD (the parity oracle of the GPU reduction) and DGGHD3
    (the blocked form timed as its CPU baseline) both return a
    Hessenberg-triangular form of the same pencil within 50 n eps, with
    the same eigenvalues."""
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n))
    B = np.triu(rng.standard_normal((n, n)))
    forms = []
    for f in (lapack.dgghrd, lapack.dgghd3):
        H, T, Q, Z, info = f(A, B)
        assert info == 0
        assert not np.any(np.tril(H, -2)) and not np.any(np.tril(T, -1))
        r = lapack.residuals(A, B, H, T, Q, Z)
        for key in ("h", "t", "q", "z"):
            assert r[key] <= 50 * r["neps"], (f.__name__, key, r[key] / r["neps"])
        forms.append((H, T))
    S0, P0, ar0, ai0, be0, _, _, i0 = lapack.dhgeqz(*forms[0])
    _, _, ar1, ai1, be1, _, _, i1 = lapack.dhgeqz(*forms[1])
    assert i0 == 0 and i1 == 0
    tol = lapack.eig_tolerance(S0, P0, *forms[0])
    ok, ratio, _ = lapack.match_eigenvalues((ar0, ai0, be0), (ar1, ai1, be1), tol)
    assert ok, ratio
