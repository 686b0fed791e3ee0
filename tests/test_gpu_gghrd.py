"""Hessenberg-triangular reduction on the GPU (DGGHRD semantics; the role
of the reference's PDGGHRD, src/ab2ht/PDGGHRD.f:13, which its examples call
after a QR factorisation of B, examples/EXRAND2.f:296-336) against LAPACK
DGGHRD on the same inputs: the same H, T, Q, Z to rounding (the same
rotations in the same order and sign convention), exact Hessenberg-
triangular structure, backward errors and orthogonality within 50 n eps;
the ILO/IHI and COMPQ/COMPZ modes; the PDGGHRD drop-in with its
transposed Q; a general pencil reduced and solved on the GPU, whose
eigenvalues match LAPACK's within the condition-scaled tolerance; and the
same for the reference's own example pencil (examples/sparseA.mtx,
sparseB.mtx, n = 4800)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver(pkg):
    s = pkg.Solver(0)
    yield s
    s.close()


def _pencil(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, n)), np.triu(rng.standard_normal((n, n)))


@pytest.mark.parametrize("n,seed,win", [(1, 1, 128), (2, 2, 128), (3, 3, 128), (17, 4, 4), (64, 5, 128),
                                        (130, 6, 7), (300, 7, 128), (700, 8, 160), (400, 9, 2), (1000, 10, 128)])
def test_gghrd_matches_dgghrd(solver, lapack, n, seed, win):
    A, B = _pencil(n, seed)
    H0, T0, Q0, Z0, info = lapack.dgghrd(A, B)
    assert info == 0
    solver.set_param("hr_win", win)
    H, T = np.array(A, order="F"), np.array(B, order="F")
    Q, Z = np.zeros((n, n), order="F"), np.zeros((n, n), order="F")
    try:
        assert solver.gghrd(H, T, Q, Z) == 0
    finally:
        solver.set_param("hr_win", 128)
    assert not np.any(np.tril(H, -2)) and not np.any(np.tril(T, -1))
    # the same rotations as DGGHRD: entrywise agreement to rounding
    tol = 1e-12 * max(1, n)
    assert np.abs(H - H0).max() <= tol * np.abs(H0).max()
    assert np.abs(T - T0).max() <= tol * np.abs(T0).max()
    assert np.abs(Q - Q0).max() <= tol and np.abs(Z - Z0).max() <= tol
    r = lapack.residuals(A, B, H, T, Q, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])


def test_gghrd_ilo_ihi_and_modes(solver, lapack):
    rng = np.random.default_rng(11)
    n, ilo, ihi = 90, 12, 71  # 1-based
    A = np.triu(rng.standard_normal((n, n)))
    A[ilo - 1:ihi, ilo - 1:ihi] = rng.standard_normal((ihi - ilo + 1,) * 2)
    B = np.triu(rng.standard_normal((n, n))) + np.tril(rng.standard_normal((n, n)), -1)  # lower part is ignored
    Qi, _ = np.linalg.qr(rng.standard_normal((n, n)))
    Zi, _ = np.linalg.qr(rng.standard_normal((n, n)))
    for cq, cz in (("V", "V"), ("N", "I"), ("I", "N"), ("N", "N")):
        Hl, Tl, Ql, Zl, info = lapack.dgghrd(A, np.triu(B), cq, cz, ilo, ihi, Qi, Zi)
        assert info == 0
        H, T = np.array(A, order="F"), np.array(B, order="F")
        Q, Z = np.array(Qi, order="F"), np.array(Zi, order="F")
        assert solver.gghrd(H, T, Q, Z, compq=cq, compz=cz, ilo=ilo, ihi=ihi) == 0
        assert np.abs(H - Hl).max() <= 1e-11 and np.abs(T - Tl).max() <= 1e-11
        assert not np.any(np.tril(T, -1))
        if cq != "N":
            assert np.abs(Q - Ql).max() <= 1e-12
        else:
            assert np.array_equal(Q, Qi)
        if cz != "N":
            assert np.abs(Z - Zl).max() <= 1e-12
        else:
            assert np.array_equal(Z, Zi)


def test_gghrd_argument_errors(solver, pkg):
    L = pkg.lib()
    A = np.zeros((4, 4), order="F")
    vp = pkg._vp(A.ctypes.data)

    def call(cq, cz, n, ilo, ihi, lda, ldb, ldq, ldz):
        return L.b200qz_gghrd_host(solver.handle, cq, cz, n, ilo, ihi, vp, lda, vp, ldb, vp, ldq, vp, ldz)

    assert call(b"X", b"I", 4, 1, 4, 4, 4, 4, 4) == -1
    assert call(b"I", b"X", 4, 1, 4, 4, 4, 4, 4) == -2
    assert call(b"I", b"I", -1, 1, 4, 4, 4, 4, 4) == -3
    assert call(b"I", b"I", 4, 0, 4, 4, 4, 4, 4) == -4
    assert call(b"I", b"I", 4, 2, 5, 4, 4, 4, 4) == -5
    assert call(b"I", b"I", 4, 3, 1, 4, 4, 4, 4) == -5
    assert call(b"I", b"I", 4, 1, 4, 3, 4, 4, 4) == -7
    assert call(b"I", b"I", 4, 1, 4, 4, 3, 4, 4) == -9
    assert call(b"I", b"I", 4, 1, 4, 4, 4, 3, 4) == -11
    assert call(b"N", b"I", 4, 1, 4, 4, 4, 1, 4) == 0
    assert call(b"I", b"I", 4, 1, 4, 4, 4, 4, 3) == -13


def test_pdgghrd_dropin_transposed_q(pkg, lapack):
    """The reference's calling sequence (examples/EXRAND2.f:282-356): Q1 = I,
    B = QR, Q1 <- Q_B^T (PDORMQR 'L','T'), A <- Q_B^T A, PDGGHRD('V','V'),
    then Q1 transposed.  The drop-in returns the transposed Q, so the
    transposed result reconstructs the original pencil."""
    import ctypes
    n, nb = 200, 32
    rng = np.random.default_rng(12)
    A0 = rng.standard_normal((n, n))
    B0 = rng.standard_normal((n, n))
    qb, rb = np.linalg.qr(B0)
    A = np.array(qb.T @ A0, order="F")
    B = np.array(np.triu(rb), order="F")
    Q = np.array(qb.T, order="F")
    Z = np.eye(n, order="F")
    d = pkg.descriptor(n, nb, n)
    dp = d.ctypes.data_as(pkg._pi)
    info = ctypes.c_int(7)
    work = np.zeros(max(1, nb))
    L = pkg.lib()
    lw = ctypes.c_int(-1)
    L.pdgghrd_(b"V", b"V", pkg._ip(n), pkg._ip(1), pkg._ip(n), pkg._vp(A.ctypes.data), dp, pkg._vp(B.ctypes.data),
               dp, pkg._vp(Q.ctypes.data), dp, pkg._vp(Z.ctypes.data), dp, pkg._p(work), ctypes.byref(lw),
               ctypes.byref(info), 1, 1)
    assert info.value == 0 and work[0] == nb
    lw = ctypes.c_int(nb)
    L.pdgghrd_(b"V", b"V", pkg._ip(n), pkg._ip(1), pkg._ip(n), pkg._vp(A.ctypes.data), dp, pkg._vp(B.ctypes.data),
               dp, pkg._vp(Q.ctypes.data), dp, pkg._vp(Z.ctypes.data), dp, pkg._p(work), ctypes.byref(lw),
               ctypes.byref(info), 1, 1)
    assert info.value == 0
    assert not np.any(np.tril(A, -2)) and not np.any(np.tril(B, -1))
    Qt = Q.T  # EXRAND2.f:352 transposes Q1 after the call
    r = lapack.residuals(A0, B0, A, B, Qt, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])
    # argument errors in PDGGHRD's numbering; N <= 1 returns before any check
    bad = d.copy()
    bad[5] = nb + 1
    for args, want in (((b"X", b"V", n, 1, n, d, nb), -1), ((b"V", b"X", n, 1, n, d, nb), -2),
                       ((b"V", b"V", n, 0, n, d, nb), -4), ((b"V", b"V", n, 1, n + 1, d, nb), -5),
                       ((b"V", b"V", n, 1, n, bad, nb), -6), ((b"V", b"V", n, 1, n, d, nb - 1), -7),
                       ((b"X", b"V", 1, 1, 1, d, nb), 0)):
        cq, cz, nn, ilo, ihi, dd, lwv = args
        info = ctypes.c_int(7)
        dpp = dd.ctypes.data_as(pkg._pi)
        L.pdgghrd_(cq, cz, pkg._ip(nn), pkg._ip(ilo), pkg._ip(ihi), pkg._vp(A.ctypes.data), dpp,
                   pkg._vp(B.ctypes.data), dp, pkg._vp(Q.ctypes.data), dp, pkg._vp(Z.ctypes.data), dp,
                   pkg._p(work), ctypes.byref(ctypes.c_int(lwv)), ctypes.byref(info), 1, 1)
        assert info.value == want, (args, info.value)


def test_gghrd_large_backward_error(solver, pkg):
    """n = 2500 on device arrays: structure and backward errors (products in
    FP64 on the GPU)."""
    import torch
    n = 2500
    A, B = _pencil(n, 13)
    dev = torch.device("cuda:0")
    tA = torch.tensor(A.T.copy(), dtype=torch.float64, device=dev)  # row-major of A^T = column-major of A
    tB = torch.tensor(B.T.copy(), dtype=torch.float64, device=dev)
    tQ = torch.empty((n, n), dtype=torch.float64, device=dev)
    tZ = torch.empty((n, n), dtype=torch.float64, device=dev)
    H, T = tA.clone(), tB.clone()
    torch.cuda.synchronize()
    assert solver.gghrd_device(H.data_ptr(), T.data_ptr(), tQ.data_ptr(), tZ.data_ptr(), n, n) == 0
    torch.cuda.synchronize()
    # the tensors hold the transposes: H^T, T^T, Q^T, Z^T
    Hm, Tm, Qm, Zm = H.T, T.T, tQ.T, tZ.T
    assert not torch.any(torch.tril(Hm, -2)) and not torch.any(torch.tril(Tm, -1))
    eps = np.finfo(np.float64).eps
    ra = torch.linalg.norm(Qm @ Hm @ Zm.T - tA.T) / torch.linalg.norm(tA)
    rb = torch.linalg.norm(Qm @ Tm @ Zm.T - tB.T) / torch.linalg.norm(tB)
    eye = torch.eye(n, dtype=torch.float64, device=dev)
    oq = torch.linalg.norm(Qm.T @ Qm - eye)
    oz = torch.linalg.norm(Zm.T @ Zm - eye)
    for v in (ra, rb, oq, oz):
        assert float(v) <= 50 * n * eps, float(v) / (n * eps)


def test_general_pencil_reduced_and_solved_on_gpu(solver, lapack, pkg):
    """A general (A, B): QR of B on the host (the step before PDGGHRD in the
    reference's examples), reduction and solve on the GPU: a Schur form of
    the original pencil whose eigenvalues match LAPACK's (DGGHRD + DHGEQZ)
    within the condition-scaled tolerance."""
    n = 600
    rng = np.random.default_rng(14)
    A0 = rng.standard_normal((n, n))
    B0 = rng.standard_normal((n, n))
    qb, rb = np.linalg.qr(B0)
    A1 = qb.T @ A0
    B1 = np.triu(rb)
    H, T = np.array(A1, order="F"), np.array(B1, order="F")
    Q, Z = np.array(qb, order="F"), np.eye(n, order="F")
    assert solver.gghrd(H, T, Q, Z, compq="V", compz="V") == 0
    ar, ai, be, info = solver.solve_host(H, T, Q, Z, compq="V", compz="V")
    assert info == 0
    r = lapack.residuals(A0, B0, H, T, Q, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])
    Hl, Tl, _, _, hinfo = lapack.dgghrd(A1, B1)
    assert hinfo == 0
    So, Po, lar, lai, lbe, _, _, linfo = lapack.dhgeqz(Hl, Tl)
    assert linfo == 0
    tol = lapack.eig_tolerance(So, Po, Hl, Tl)
    ok, ratio, _ = lapack.match_eigenvalues((lar, lai, lbe), (ar, ai, be), tol)
    assert ok, ratio


def test_reference_example_pencil_reduced_and_solved_on_gpu(solver, lapack, pkg):
    """The reference's own example pair (examples/sparseA.mtx, sparseB.mtx,
    4800 x 4800, read by examples/EXRAND3.f:297-316; entries committed in
    tests/golden/mhd4800.npz by tests/golden/make_mhd_fixture.py): QR of B
    on the host, then the Hessenberg-triangular reduction and the QZ solve
    on the GPU.  The result is a generalized Schur form of the original
    pencil within 50 n eps, and its eigenvalues match LAPACK's (DGGHD3 +
    DHGEQZ of the same pencil) within the condition-scaled tolerance."""
    import os
    import torch
    fx = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mhd4800.npz"))
    n = 4800
    A0 = np.zeros((n, n))
    np.add.at(A0, (fx["a_i"], fx["a_j"]), fx["a_v"])
    B0 = np.zeros((n, n))
    np.add.at(B0, (fx["b_i"], fx["b_j"]), fx["b_v"])
    off = fx["b_i"] != fx["b_j"]
    np.add.at(B0, (fx["b_j"][off], fx["b_i"][off]), fx["b_v"][off])
    qb, rb = np.linalg.qr(B0)
    dev = torch.device("cuda:0")
    # device buffers hold the transposes of the column-major matrices
    tA = torch.tensor((qb.T @ A0).T.copy(), dtype=torch.float64, device=dev)
    tB = torch.tensor(np.triu(rb).T.copy(), dtype=torch.float64, device=dev)
    tQ = torch.tensor(qb.T.copy(), dtype=torch.float64, device=dev)
    tZ = torch.empty((n, n), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    assert solver.gghrd_device(tA.data_ptr(), tB.data_ptr(), tQ.data_ptr(), tZ.data_ptr(), n, n,
                               compq="V", compz="I") == 0
    de = torch.empty(3 * n, dtype=torch.float64, device=dev)
    info = solver.solve_device(tA.data_ptr(), tB.data_ptr(), tQ.data_ptr(), tZ.data_ptr(), n, n, de.data_ptr(),
                               de.data_ptr() + 8 * n, de.data_ptr() + 16 * n, compq="V", compz="V")
    torch.cuda.synchronize()
    assert info == 0
    S, P, Q, Z = tA.T, tB.T, tQ.T, tZ.T
    gA0 = torch.tensor(A0, dtype=torch.float64, device=dev)
    gB0 = torch.tensor(B0, dtype=torch.float64, device=dev)
    eps = np.finfo(np.float64).eps
    I = torch.eye(n, dtype=torch.float64, device=dev)
    r = {"a": float(torch.linalg.norm(Q @ S @ Z.T - gA0) / torch.linalg.norm(gA0)),
         "b": float(torch.linalg.norm(Q @ P @ Z.T - gB0) / torch.linalg.norm(gB0)),
         "q": float(torch.linalg.norm(Q.T @ Q - I)), "z": float(torch.linalg.norm(Z.T @ Z - I))}
    for key, v in r.items():
        assert v <= 50 * n * eps, (key, v / (n * eps))
    assert not bool(torch.any(torch.tril(S, -2))) and not bool(torch.any(torch.tril(P, -1)))
    e = de.cpu().numpy()
    tol = np.clip(50.0 * n * eps * float(fx["norm"]) / np.maximum(fx["rcond"], 1e-300), 50.0 * n * eps, 2.0)
    ok, ratio, _ = lapack.match_eigenvalues((fx["alphar"], fx["alphai"], fx["beta"]), (e[:n], e[n:2 * n], e[2 * n:]),
                                            tol)
    assert ok, ratio
