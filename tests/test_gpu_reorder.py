"""Reordering of a generalized real Schur form on the GPU (DTGSEN
semantics; the reference's PDTGSEN/PDTGORD, src/reorder/PDTGSEN.f:1)
against LAPACK DTGSEN on the same Schur form: the same dimension m, the
selected eigenvalues leading in the same order, the same deflating
subspaces (principal angles), backward errors and orthogonality within
50 n eps of the original pencil, Schur structure with non-negative 1x1
T entries, the projection norms PL, PR (IJOB = 1, 5) and the 1-norm Dif
estimates (IJOB = 3, 5)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver(pkg):
    s = pkg.Solver(0)
    yield s
    s.close()


def _schur(lapack, pkg, n, seed, zf=0.0):
    H, T = pkg.pencils.random_ht(n, seed, zf)
    S, P, ar, ai, be, Q, Z, info = lapack.dhgeqz(H, T)
    assert info == 0
    return H, T, S, P, Q, Z, ar, ai, be


def _select(ar, ai, be, rule, seed):
    n = len(ar)
    lam = np.abs(ar + 1j * ai) / np.maximum(np.abs(be), 1e-300)
    if rule == "small":
        sel = lam < np.median(lam)
    elif rule == "random":
        sel = np.random.default_rng(seed).random(n) < 0.4
    elif rule == "bottom":
        sel = np.zeros(n, bool)
        sel[-max(1, n // 10):] = True
    elif rule == "all":
        sel = np.ones(n, bool)
    else:
        sel = np.zeros(n, bool)
    return sel.astype(np.int32)


def _sin_angle(X, Y, m):
    """Largest sine of the principal angles between span X[:, :m] and span Y[:, :m]."""
    if m == 0 or m == X.shape[0]:
        return 0.0
    return float(np.linalg.norm(Y[:, m:].T @ X[:, :m], 2))


@pytest.mark.parametrize("n,seed,rule,ijob", [(8, 1, "small", 0), (40, 2, "random", 1), (120, 3, "small", 1),
                                               (200, 4, "random", 0), (300, 5, "bottom", 1), (60, 6, "all", 1),
                                               (60, 7, "none", 1), (1, 8, "all", 1), (500, 9, "random", 1)])
def test_tgsen_matches_lapack(solver, lapack, pkg, n, seed, rule, ijob):
    H, T, S, P, Q, Z, ar, ai, be = _schur(lapack, pkg, n, seed)
    sel = _select(ar, ai, be, rule, seed)
    # ijob 4: the same reordering, plus Dif estimates that bound how far the
    # deflating subspaces may move under rounding
    La, Lb, lar, lai, lbe, Lq, Lz, lm, lpl, lpr, dif, linfo = lapack.dtgsen(S, P, Q, Z, sel, ijob=4)
    assert linfo == 0
    eps = np.finfo(np.float64).eps
    nrm = np.hypot(np.linalg.norm(H), np.linalg.norm(T))
    sub_tol = min(1.0, 1e3 * n * eps * nrm / max(float(np.min(dif)), 1e-300)) if 0 < lm < n else 1e-12
    Gs, Gt, Gq, Gz = (np.array(M, order="F", copy=True) for M in (S, P, Q, Z))
    gar, gai, gbe, m, pl, pr, info, ret = solver.tgsen(Gs, Gt, Gq, Gz, sel, ijob=ijob)
    assert ret == 0 and info == 0
    assert m == lm
    # a generalized Schur form of the original pencil
    r = lapack.residuals(H, T, Gs, Gt, Gq, Gz)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])
    assert lapack.schur_structure_ok(Gs, Gt)
    one = [k for k in range(n) if (k == 0 or Gs[k, k - 1] == 0) and (k == n - 1 or Gs[k + 1, k] == 0)]
    assert np.all(Gt[one, one] >= 0)
    # the same leading eigenvalues, in the same order
    if n > 1:
        tol = lapack.eig_tolerance(La, Lb, H, T)
        ok, ratio, _ = lapack.match_eigenvalues((lar[:m], lai[:m], lbe[:m]), (gar[:m], gai[:m], gbe[:m]), tol[:m])
        assert ok, ratio
        # position by position (a conjugate pair may list its members in
        # either order): real parts and moduli of the imaginary parts
        g = (gar + 1j * gai) / gbe
        l = (lar + 1j * lai) / lbe
        scale = np.maximum(np.abs(l[:m]), 1.0)
        assert np.all(np.abs(g[:m].real - l[:m].real) <= 1e-8 * scale)
        assert np.all(np.abs(np.abs(g[:m].imag) - np.abs(l[:m].imag)) <= 1e-8 * scale)
    # the same deflating subspaces
    assert _sin_angle(Gz, Lz, m) <= sub_tol
    assert _sin_angle(Gq, Lq, m) <= sub_tol
    if ijob == 1:
        assert abs(pl - lpl) <= max(1e-9, sub_tol) * lpl + 1e-14
        assert abs(pr - lpr) <= max(1e-9, sub_tol) * lpr + 1e-14
    else:
        assert pl == 1.0 and pr == 1.0


def test_tgsen_with_gpu_schur_form(solver, lapack, pkg):
    """Solve on the GPU, then reorder the GPU's Schur form on the GPU: the
    selected eigenvalues lead and the result is still a Schur form of the
    input pencil."""
    n = 400
    H, T = pkg.pencils.random_ht(n, 41, 0.0)
    S, P, Q, Z, ar, ai, be, info = pkg.solve(H, T)
    assert info == 0
    lam = np.abs(ar + 1j * ai) / np.maximum(np.abs(be), 1e-300)
    sel = (lam > np.median(lam)).astype(np.int32)
    gar, gai, gbe, m, pl, pr, rinfo, ret = solver.tgsen(S, P, Q, Z, sel, ijob=1)
    assert ret == 0 and rinfo == 0
    r = lapack.residuals(H, T, S, P, Q, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])
    g = np.abs(gar + 1j * gai) / np.maximum(np.abs(gbe), 1e-300)
    assert m == int(sel.sum()) or m == int(sel.sum()) + 1
    assert np.min(g[:m]) >= np.median(lam) * (1 - 1e-9)
    assert 0.0 < pl <= 1.0 and 0.0 < pr <= 1.0


def test_tgsen_argument_errors(solver, pkg):
    L = pkg.lib()
    A = np.zeros((4, 4), order="F")
    sel = np.zeros(4, dtype=np.int32)
    v = np.zeros(4)
    m, info = pkg.ctypes.c_int(0), pkg.ctypes.c_int(0)
    pl, pr = pkg.ctypes.c_double(0), pkg.ctypes.c_double(0)
    vp = pkg._vp(A.ctypes.data)

    def call(ijob, n, lds, ldt, ldq, ldz):
        return L.b200qz_tgsen_host(solver.handle, ijob, 1, 1, sel.ctypes.data_as(pkg._pi), n, vp, lds, vp, ldt, vp,
                                   ldq, vp, ldz, pkg._p(v), pkg._p(v), pkg._p(v), pkg.ctypes.byref(m),
                                   pkg.ctypes.byref(pl), pkg.ctypes.byref(pr), pkg._p(v), pkg.ctypes.byref(info))

    assert call(2, 4, 4, 4, 4, 4) == -1
    assert call(4, 4, 4, 4, 4, 4) == -1
    assert call(6, 4, 4, 4, 4, 4) == -1
    assert call(0, -1, 4, 4, 4, 4) == -5
    assert call(0, 4, 3, 4, 4, 4) == -7
    assert call(0, 4, 4, 3, 4, 4) == -9
    assert call(0, 4, 4, 4, 3, 4) == -14
    assert call(0, 4, 4, 4, 4, 3) == -16


@pytest.mark.parametrize("n,seed,rule,ijob", [(12, 21, "small", 3), (40, 22, "random", 5), (14, 4, "small", 5),
                                               (30, 24, "bottom", 3), (60, 25, "all", 5), (60, 26, "none", 3)])
def test_tgsen_dif_estimates(solver, lapack, pkg, n, seed, rule, ijob):
    """Difu and Difl by Higham's 1-norm estimator over generalized Sylvester
    solves and their transposes (DTGSEN IJOB 3 and 5).  The estimator is
    LAPACK DLACN2's (pinned by the host test against DLACN2 itself); its
    sign-vector iteration can take another path when a solution entry that
    is zero in exact arithmetic comes out +0 in one solve and -1e-17 in
    another, so against LAPACK's DTGSEN the estimates agree within a factor
    of 3 (exactly in most cases), and each is checked against the true
    value it estimates: 1/Dif <= ||Z^-1||_1 for the Sylvester operator Z,
    i.e. the estimate is never below the true 1-norm separation.  With
    nothing or everything selected DTGSEN returns ||(S, T)||_F, to rounding."""
    H, T, S, P, Q, Z, ar, ai, be = _schur(lapack, pkg, n, seed)
    sel = _select(ar, ai, be, rule, seed)
    La, Lb, lar, lai, lbe, Lq, Lz, lm, lpl, lpr, ldif, linfo = lapack.dtgsen(S, P, Q, Z, sel, ijob=ijob)
    assert linfo == 0
    Gs, Gt, Gq, Gz = (np.array(M, order="F", copy=True) for M in (S, P, Q, Z))
    dif = np.zeros(2)
    gar, gai, gbe, m, pl, pr, info, ret = solver.tgsen(Gs, Gt, Gq, Gz, sel, ijob=ijob, dif=dif)
    assert ret == 0 and info == 0 and m == lm
    if m == 0 or m == n:
        assert np.allclose(dif, ldif, rtol=1e-12), (dif, ldif)
        return
    assert np.all(dif > 0)
    assert np.all(dif >= ldif / 3) and np.all(dif <= 3 * ldif), (dif, ldif)

    def op(A, D, B, E):
        p_, q_ = A.shape[0], B.shape[0]
        return np.block([[np.kron(np.eye(q_), A), -np.kron(B.T, np.eye(p_))],
                         [np.kron(np.eye(q_), D), -np.kron(E.T, np.eye(p_))]])

    S11, T11, S22, T22 = Gs[:m, :m], Gt[:m, :m], Gs[m:, m:], Gt[m:, m:]
    for k, Zop in enumerate((op(S11, T11, S22, T22), op(S22, T22, S11, T11))):
        true_sep = 1.0 / np.abs(np.linalg.inv(Zop)).sum(axis=0).max()
        assert dif[k] >= true_sep * (1 - 1e-9), (k, dif[k], true_sep)
    if ijob == 5:
        assert abs(pl - lpl) <= 1e-9 * lpl and abs(pr - lpr) <= 1e-9 * lpr
