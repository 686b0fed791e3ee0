"""Balancing on the GPU (DGGBAL / DGGBAK semantics) against LAPACK's own
DGGBAL / DGGBAK (the routines that produce the ILO/IHI the reference's
driver takes, PDHGEQZ.f:155-161): the same ILO/IHI, the same recorded
interchanges and power-of-ten scale factors, the same balanced pencil bit
for bit, and the same back-transformed vectors.  A balanced pencil reduced
to Hessenberg-triangular form and solved with its ILO/IHI gives LAPACK's
eigenvalues of the original pencil."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _block_permuted(n, seed, k1, k2, density=1.0):
    """[[T1 X Y]; [0 M W]; [0 0 T2]] (T1, T2 upper triangular of orders
    k1, k2) for A and B, rows and columns then shuffled by random
    permutations: DGGBAL isolates k1 + k2 eigenvalues."""
    rng = np.random.default_rng(seed)

    def one():
        S = rng.standard_normal((n, n))
        if density < 1.0:
            S *= rng.random((n, n)) < density
        S[k1:, :k1] = 0.0
        S[n - k2:, :n - k2] = 0.0
        S[:k1, :k1] = np.triu(S[:k1, :k1])
        S[n - k2:, n - k2:] = np.triu(S[n - k2:, n - k2:])
        return S

    A, B = one(), one()
    pr, pc = rng.permutation(n), rng.permutation(n)
    return A[pr][:, pc], B[pr][:, pc]


def _pencil(kind, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "dense":
        return rng.standard_normal((n, n)), rng.standard_normal((n, n))
    if kind == "graded":
        A = rng.standard_normal((n, n)) * np.logspace(-8, 8, n)[:, None] * np.logspace(3, -3, n)[None, :]
        B = rng.standard_normal((n, n)) * np.logspace(5, -5, n)[None, :]
        return A, B
    if kind == "block":
        return _block_permuted(n, seed, n // 5, n // 4)
    if kind == "blockgraded":
        A, B = _block_permuted(n, seed, n // 6, n // 7)
        d = np.logspace(-5, 5, n)
        return A * d[:, None], B * d[None, :]
    if kind == "sparse":
        A = rng.standard_normal((n, n)) * (rng.random((n, n)) < 0.03)
        B = rng.standard_normal((n, n)) * (rng.random((n, n)) < 0.03)
        return A, B
    if kind == "zeros":
        A, B = rng.standard_normal((n, n)), rng.standard_normal((n, n))
        for r in rng.choice(n, 3, replace=False):
            A[r, :] = 0.0
            B[r, :] = 0.0
        for c in rng.choice(n, 2, replace=False):
            A[:, c] = 0.0
            B[:, c] = 0.0
        return A, B
    if kind == "triangular":
        return np.triu(rng.standard_normal((n, n))), np.triu(rng.standard_normal((n, n)))
    raise ValueError(kind)


@pytest.fixture(scope="module")
def solver(pkg):
    s = pkg.Solver(0)
    yield s
    s.close()


CASES = [("dense", 120, 1, "B"), ("graded", 150, 2, "S"), ("graded", 150, 3, "B"), ("block", 200, 4, "P"),
         ("block", 200, 5, "B"), ("blockgraded", 240, 6, "B"), ("sparse", 160, 7, "P"), ("sparse", 160, 8, "B"),
         ("zeros", 90, 9, "B"), ("triangular", 60, 10, "B"), ("dense", 2, 11, "B"), ("dense", 1, 12, "B"),
         ("graded", 700, 13, "B"), ("block", 600, 14, "B"), ("dense", 50, 15, "N")]


@pytest.mark.parametrize("kind,n,seed,job", CASES)
def test_ggbal_matches_lapack(solver, lapack, kind, n, seed, job):
    A, B = _pencil(kind, n, seed)
    La, Lb, lilo, lihi, lls, lrs, linfo = lapack.dggbal(A, B, job)
    assert linfo == 0
    Ga = np.array(A, order="F", copy=True)
    Gb = np.array(B, order="F", copy=True)
    ilo, ihi, ls, rs, info = solver.ggbal(Ga, Gb, job)
    assert info == 0
    assert (ilo, ihi) == (lilo, lihi)
    assert np.array_equal(ls, lls) and np.array_equal(rs, lrs), (ls, lls, rs, lrs)
    assert np.array_equal(Ga, La) and np.array_equal(Gb, Lb)
    if job in "PB" and n > 1:
        # outside ILO..IHI the balanced pencil is upper triangular
        lo, hi = ilo - 1, ihi - 1
        for M in (Ga, Gb):
            assert not np.any(M[hi + 1:, :hi + 1])
            assert not np.any(M[lo:, :lo])


def test_ggbal_empty_pencil(solver):
    A = np.zeros((1, 1), order="F")
    ilo, ihi, ls, rs, info = solver.ggbal(A[:0, :0], A[:0, :0].copy(), "B")
    assert info == 0 and (ilo, ihi) == (1, 0)


@pytest.mark.parametrize("job,side", [("B", "R"), ("B", "L"), ("P", "R"), ("S", "L"), ("N", "R")])
def test_ggbak_matches_lapack(solver, lapack, job, side):
    A, B = _pencil("blockgraded", 240, 21)
    _, _, ilo, ihi, ls, rs, _ = lapack.dggbal(A, B, job)
    rng = np.random.default_rng(22)
    V = np.array(rng.standard_normal((240, 37)), order="F")
    ref, linfo = lapack.dggbak(V, ilo, ihi, ls, rs, side=side, job=job)
    assert linfo == 0
    G = V.copy(order="F")
    assert solver.ggbak(G, ilo, ihi, ls, rs, side=side, job=job) == 0
    assert np.array_equal(G, ref)


def test_ggbal_argument_errors(solver, pkg):
    L = pkg.lib()
    A = np.zeros((4, 4), order="F")
    ls = np.zeros(4)
    i1, i2 = pkg.ctypes.c_int(0), pkg.ctypes.c_int(0)
    args = lambda job, n, lda, ldb: L.b200qz_ggbal_host(solver.handle, job, n, pkg._vp(A.ctypes.data), lda,
                                                        pkg._vp(A.ctypes.data), ldb, pkg.ctypes.byref(i1),
                                                        pkg.ctypes.byref(i2), pkg._p(ls), pkg._p(ls))
    assert args(b"X", 4, 4, 4) == -1
    assert args(b"B", -1, 4, 4) == -2
    assert args(b"B", 4, 3, 4) == -4
    assert args(b"B", 4, 4, 3) == -6
    V = np.zeros((4, 2), order="F")
    bak = lambda job, side, n, ilo, ihi, m, ldv: L.b200qz_ggbak_host(solver.handle, job, side, n, ilo, ihi,
                                                                     pkg._p(ls), pkg._p(ls), m,
                                                                     pkg._vp(V.ctypes.data), ldv)
    assert bak(b"X", b"R", 4, 1, 4, 2, 4) == -1
    assert bak(b"B", b"X", 4, 1, 4, 2, 4) == -2
    assert bak(b"B", b"R", -1, 1, 4, 2, 4) == -3
    assert bak(b"B", b"R", 4, 0, 4, 2, 4) == -4
    assert bak(b"B", b"R", 4, 3, 2, 2, 4) == -5
    assert bak(b"B", b"R", 4, 1, 4, -1, 4) == -8
    assert bak(b"B", b"R", 4, 1, 4, 2, 3) == -10


@pytest.mark.parametrize("kind,n,seed", [("blockgraded", 300, 31), ("graded", 400, 32)])
def test_balanced_solve_with_ilo_ihi(solver, lapack, pkg, kind, n, seed):
    """Balance on the GPU, reduce to Hessenberg-triangular form (QR of B,
    then DGGHRD from the test harness), solve on the GPU with the ILO/IHI
    the balancing returned: LAPACK's eigenvalues of the same balanced
    pencil within the condition-scaled tolerance, and the isolated
    eigenvalues exactly the diagonal ratios outside ILO..IHI."""
    A, B = _pencil(kind, n, seed)
    Ga, Gb = np.array(A, order="F"), np.array(B, order="F")
    ilo, ihi, ls, rs, info = solver.ggbal(Ga, Gb, "B")
    assert info == 0
    q, r = np.linalg.qr(Gb)
    H0, T0, _, _, hinfo = lapack.dgghrd(q.T @ Ga, np.triu(r))
    assert hinfo == 0
    H, T = np.array(H0, order="F"), np.array(T0, order="F")
    Q, Z = np.eye(n, order="F"), np.eye(n, order="F")
    ar, ai, be, sinfo = solver.solve_host(H, T, Q, Z, ilo=ilo, ihi=ihi)
    assert sinfo == 0
    So, Po, lar, lai, lbe, _, _, linfo = lapack.dhgeqz(H0, T0, ilo=ilo, ihi=ihi)
    assert linfo == 0
    tol = lapack.eig_tolerance(So, Po, H0, T0)
    ok, ratio, _ = lapack.match_eigenvalues((lar, lai, lbe), (ar, ai, be), tol)
    assert ok, ratio
