"""Kernel-level parity on the GPU through the C-ABI.

Tolerances: the off-diagonal update is an FP64 product with k-term dot
products, checked to 8*k*eps relative to |W|*|M|; window kernels are checked
through backward error (<= 50*n*eps) and orthogonality of their factors."""
import ctypes

import numpy as np
import pytest
import torch

from conftest import EPS

pytestmark = pytest.mark.gpu


def colmajor_cuda(A):
    """device buffer holding the column-major storage of A"""
    return torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()


def to_np(t, n, m):
    return t.cpu().numpy().T.copy(order="F")


@pytest.fixture(scope="module")
def solver(pkg):
    s = pkg.Solver(0)
    yield s
    s.close()


@pytest.mark.parametrize("k,side,len_", [(16, "L", 100), (37, "L", 65), (80, "R", 300), (80, "L", 1000),
                                          (128, "R", 257), (200, "L", 90), (200, "R", 33)])
def test_update_matches_fp64_product(pkg, solver, k, side, len_):
    rng = np.random.default_rng(k + len_)
    W = np.linalg.qr(rng.standard_normal((k, k)))[0]
    rows, cols = (k + 7, len_ + 5) if side == "L" else (len_ + 3, k + 9)
    M = rng.standard_normal((rows, cols))
    r0, c0 = (5, 3) if side == "L" else (2, 6)
    dM = colmajor_cuda(M)
    dW = colmajor_cuda(W)
    rc = pkg.lib().b200qz_update(solver.handle, side.encode(), dM.data_ptr(), rows, r0, c0, len_, dW.data_ptr(), k, k)
    assert rc == 0
    out = to_np(dM, rows, cols)
    ref = M.copy()
    if side == "L":
        ref[r0:r0 + k, c0:c0 + len_] = W.T @ M[r0:r0 + k, c0:c0 + len_]
        scale = np.abs(W.T) @ np.abs(M[r0:r0 + k, c0:c0 + len_])
        sl = (slice(r0, r0 + k), slice(c0, c0 + len_))
    else:
        ref[r0:r0 + len_, c0:c0 + k] = M[r0:r0 + len_, c0:c0 + k] @ W
        scale = np.abs(M[r0:r0 + len_, c0:c0 + k]) @ np.abs(W)
        sl = (slice(r0, r0 + len_), slice(c0, c0 + k))
    err = np.abs(out[sl] - ref[sl])
    assert np.all(err <= 8 * k * EPS * scale + 1e-300)
    # untouched outside the slab
    mask = np.ones_like(M, dtype=bool)
    mask[sl] = False
    assert np.array_equal(out[mask], M[mask])


@pytest.mark.parametrize("n,seed,zf", [(5, 1, 0.0), (24, 2, 0.0), (60, 3, 0.1), (80, 4, 0.0)])
def test_window_full_schur(pkg, lapack, solver, n, seed, zf):
    """AED kernel with the window = whole active block: full small QZ."""
    H, T = pkg.pencils.random_ht(n, seed, zf)
    dH, dT = colmajor_cuda(H), colmajor_cuda(T)
    dQ = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    dZ = torch.zeros_like(dQ)
    dS = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    info = (ctypes.c_int * 3)()
    rc = pkg.lib().b200qz_aed_window(solver.handle, dH.data_ptr(), dT.data_ptr(), n, 0, 0, n - 1,
                                     dQ.data_ptr(), dZ.data_ptr(), dS.data_ptr(), info)
    assert rc == 0 and info[1] == 0 and info[0] == 0 and info[2] == 1
    S, P = to_np(dH, n, n), to_np(dT, n, n)
    Q = dQ.cpu().numpy().reshape(n, n).T
    Z = dZ.cpu().numpy().reshape(n, n).T
    r = lapack.residuals(H, T, S, P, Q, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r)
    assert np.all(np.tril(S, -2) == 0) and np.all(np.tril(P, -1) == 0)
    e = lapack.eig_from_schur(S, P)
    So, Po, ar, ai, be, _, _, _ = lapack.dhgeqz(H, T)
    tol = lapack.eig_tolerance(So, Po, H, T)
    ok, ratio, _ = lapack.match_eigenvalues((ar, ai, be), e, tol)
    assert ok, ratio


@pytest.mark.parametrize("n,nw,seed", [(200, 40, 5), (300, 80, 6)])
def test_aed_window(pkg, lapack, solver, n, nw, seed):
    H, T = pkg.pencils.clustered_ht(n, seed, every=17)
    kwtop = n - nw
    dH, dT = colmajor_cuda(H), colmajor_cuda(T)
    dQ = torch.zeros(nw * nw, dtype=torch.float64, device="cuda")
    dZ = torch.zeros_like(dQ)
    dS = torch.zeros(3 * nw, dtype=torch.float64, device="cuda")
    info = (ctypes.c_int * 3)()
    rc = pkg.lib().b200qz_aed_window(solver.handle, dH.data_ptr(), dT.data_ptr(), n, 0, kwtop, n - 1,
                                     dQ.data_ptr(), dZ.data_ptr(), dS.data_ptr(), info)
    assert rc == 0 and info[1] == 0
    m = info[0]
    assert 0 < m < nw and info[2] == 1
    Hn, Tn = to_np(dH, n, n), to_np(dT, n, n)
    Q = dQ.cpu().numpy().reshape(nw, nw).T
    Z = dZ.cpu().numpy().reshape(nw, nw).T
    W0, T0 = H[kwtop:, kwtop:], T[kwtop:, kwtop:]
    W1, T1 = Hn[kwtop:, kwtop:], Tn[kwtop:, kwtop:]
    assert np.linalg.norm(Q @ W1 @ Z.T - W0) <= 50 * nw * EPS * np.linalg.norm(W0)
    assert np.linalg.norm(Q @ T1 @ Z.T - T0) <= 50 * nw * EPS * np.linalg.norm(T0)
    assert np.linalg.norm(Q.T @ Q - np.eye(nw)) <= 50 * nw * EPS
    # spike: new H(kwtop, kwtop-1) = s*Q(0,0); deflated rows decoupled
    s = H[kwtop, kwtop - 1]
    assert np.isclose(Hn[kwtop, kwtop - 1], s * Q[0, 0], rtol=1e-14, atol=0)
    spike = s * Q[0, :]
    assert np.all(np.abs(spike[m:]) <= max(EPS * abs(s) * 10, 1e-300) + EPS * np.abs(np.diag(W1)[m:]) * 10)
    assert np.all(np.tril(W1[:m, :m], -2) == 0) and np.all(np.tril(T1, -1) == 0)
    assert np.all(W1[m:, :m] == 0)
    # nothing outside the window changed
    assert np.array_equal(Hn[:kwtop, :], H[:kwtop, :]) and np.array_equal(Hn[:, :kwtop - 1], H[:, :kwtop - 1])


def _shift_set(rng, nb, cplx):
    """nb shift pairs as (sr, si, sb) lists and polynomial coefficients."""
    sr, si, sb, coef = [], [], [], []
    for b in range(nb):
        if cplx and b % 2 == 0:
            ar, ai = rng.standard_normal(), abs(rng.standard_normal()) + 0.1
            sr += [ar, ar]; si += [ai, -ai]; sb += [1.0, 1.0]
            coef += [1.0, 2 * ar, ar * ar + ai * ai]
        else:
            a1, a2 = rng.standard_normal(2)
            sr += [a1, a2]; si += [0.0, 0.0]; sb += [1.0, 1.0]
            coef += [1.0, a1 + a2, a1 * a2]
    return np.array(sr), np.array(si), np.array(sb), np.array(coef)


@pytest.mark.parametrize("n,nb,cplx", [(12, 1, False), (30, 3, False), (50, 5, True), (60, 6, True), (80, 12, True)])
def test_chase_window_matches_restatement(pkg, solver, n, nb, cplx):
    """Chase of an introduced chain through one window (lockstep, GPU)
    against the oracle's bulge-by-bulge PDHGEQZB/DHGEQZ5 restatement from
    the same state (the oracle's PDHGEQZA introduction).  Both apply the
    same reflectors in exact arithmetic, so H, T, U (=Q), V (=Z) agree to
    rounding: 1e-9 relative.  (Whole sweeps are not compared element-wise:
    the two codes form the shift polynomial's first column with different
    roundings, and a long chase amplifies that difference.)"""
    from oracle import qzref as R
    H, T = pkg.pencils.random_ht(n, 20 + n)
    rng = np.random.default_rng(n)
    sr, si, sb, coef = _shift_set(rng, nb, cplx)
    H1, T1, _, _ = R.sweep(H, T, sr, si, sb, phase=1)
    S_ref, P_ref, Q_ref, Z_ref = R.sweep(H1, T1, sr, si, sb, phase=2)
    bul, tmax = [], 0
    for k in range(nb):
        base = 3 * (nb - 1 - k) + 1   # next step row of bulge k (0 = deepest)
        thi = (n - 1) - base           # chase to the bottom and push off
        bul += [base, 0, thi, 0]
        tmax = max(tmax, thi)
    bul = (ctypes.c_int * len(bul))(*bul)
    cf = (ctypes.c_double * len(coef))(*coef.tolist())
    dH, dT = colmajor_cuda(H1), colmajor_cuda(T1)
    dU = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    dV = torch.zeros_like(dU)
    rc = pkg.lib().b200qz_chase_window(solver.handle, dH.data_ptr(), dT.data_ptr(), n, 0, n, n - 1, bul, cf, nb,
                                       tmax, dU.data_ptr(), dV.data_ptr())
    assert rc == 0
    S, P = to_np(dH, n, n), to_np(dT, n, n)
    U = dU.cpu().numpy().reshape(n, n).T
    V = dV.cpu().numpy().reshape(n, n).T
    assert np.linalg.norm(U @ S @ V.T - H1) <= 50 * n * EPS * np.linalg.norm(H1)
    assert np.linalg.norm(U @ P @ V.T - T1) <= 50 * n * EPS * np.linalg.norm(T1)
    assert np.all(np.tril(S, -2) == 0) and np.all(np.tril(P, -1) == 0)
    for a, b in ((S, S_ref), (P, P_ref), (U, Q_ref), (V, Z_ref)):
        assert np.linalg.norm(a - b) <= 1e-9 * max(1.0, np.linalg.norm(b)), np.linalg.norm(a - b)


@pytest.mark.parametrize("n,nb,cplx", [(40, 4, True), (80, 12, False)])
def test_chase_window_full_sweep_backward_stable(pkg, solver, n, nb, cplx):
    """Introduction + chase + push-off in one window: an orthogonal
    equivalence to 50*n*eps that returns a Hessenberg-triangular pencil."""
    H, T = pkg.pencils.random_ht(n, 40 + n)
    rng = np.random.default_rng(n + 1)
    sr, si, sb, coef = _shift_set(rng, nb, cplx)
    bul, tmax = [], 0
    for k in range(nb):
        base, tlo = -3 * k, 3 * k
        thi = (n - 1) - base
        bul += [base, tlo, thi, 1]
        tmax = max(tmax, thi)
    bul = (ctypes.c_int * len(bul))(*bul)
    cf = (ctypes.c_double * len(coef))(*coef.tolist())
    dH, dT = colmajor_cuda(H), colmajor_cuda(T)
    dU = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    dV = torch.zeros_like(dU)
    rc = pkg.lib().b200qz_chase_window(solver.handle, dH.data_ptr(), dT.data_ptr(), n, 0, n, n - 1, bul, cf, nb,
                                       tmax, dU.data_ptr(), dV.data_ptr())
    assert rc == 0
    S, P = to_np(dH, n, n), to_np(dT, n, n)
    U = dU.cpu().numpy().reshape(n, n).T
    V = dV.cpu().numpy().reshape(n, n).T
    assert np.linalg.norm(U @ S @ V.T - H) <= 50 * n * EPS * np.linalg.norm(H)
    assert np.linalg.norm(U @ P @ V.T - T) <= 50 * n * EPS * np.linalg.norm(T)
    assert np.linalg.norm(U.T @ U - np.eye(n)) <= 50 * n * EPS
    assert np.all(np.tril(S, -2) == 0) and np.all(np.tril(P, -1) == 0)
