"""Split-precision (INT8 Ozaki, 7 slices, tcgen05) off-diagonal updates.

Kernel level: the in-place update through b200qz_update_split against the
FP64 product, entrywise within 2^-44 (7 slices) or 2^-51 (8 slices) times
k * max|a_i| * max|w_j| (the slice truncation is about 2^-48 or 2^-55
relative to those scales), for left and right updates, graded slabs, every
window size class and ragged tiles.  Solver level: full solves with the
split updates keep the backward error and orthogonality within 50*n*eps
and the Schur structure, and their eigenvalues match LAPACK's."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _split_update(pkg, side, M, r0, c0, length, W, slices):
    import torch
    k = W.shape[0]
    dM = torch.from_numpy(np.ascontiguousarray(M.T)).cuda()  # column-major storage
    dW = torch.from_numpy(np.ascontiguousarray(W.T)).cuda()
    s = pkg.Solver(0)
    try:
        rc = pkg.lib().b200qz_update_split(s.handle, side.encode(), ctypes.c_void_p(dM.data_ptr()), M.shape[0], r0,
                                           c0, length, ctypes.c_void_p(dW.data_ptr()), k, k, slices)
    finally:
        s.close()
    assert rc == 0, rc
    return dM.cpu().numpy().T


@pytest.mark.parametrize("slices,tol", [(7, 2.0 ** -44), (8, 2.0 ** -51)])
@pytest.mark.parametrize("k", [1, 7, 16, 33, 64, 80])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("n", [400, 401])
def test_split_update_matches_fp64(pkg, k, side, slices, tol, n):
    """n = 400: the slab tile comes in by TMA (even leading dimension; the
    odd row offset 37 exercises the box start rounded down to an even row);
    n = 401: odd leading dimension, plain loads."""
    rng = np.random.default_rng(100 + k)
    M = rng.standard_normal((n, n)) * 10.0 ** rng.uniform(-6, 6, size=(n, 1))
    M *= 10.0 ** rng.uniform(-3, 3, size=(1, n))
    W = np.linalg.qr(rng.standard_normal((k, k)))[0]
    r0, c0 = 37, 101
    length = 257 if side == "L" else 299
    out = _split_update(pkg, side, M, r0, c0, length, W, slices)
    ref = M.copy()
    if side == "L":
        X = M[r0:r0 + k, c0:c0 + length]
        ref[r0:r0 + k, c0:c0 + length] = W.T @ X
        A = X.T                      # rows of the product's A operand
        D_err = np.abs(out[r0:r0 + k, c0:c0 + length] - ref[r0:r0 + k, c0:c0 + length]).T
    else:
        X = M[r0:r0 + length, c0:c0 + k]
        ref[r0:r0 + length, c0:c0 + k] = X @ W
        A = X
        D_err = np.abs(out[r0:r0 + length, c0:c0 + k] - ref[r0:r0 + length, c0:c0 + k])
    scale = np.abs(A).max(axis=1, keepdims=True) * np.abs(W).max(axis=0, keepdims=True) * k
    assert np.all(D_err <= tol * scale), float((D_err / scale).max())
    # everything outside the slab is untouched
    mask = np.ones_like(M, dtype=bool)
    if side == "L":
        mask[r0:r0 + k, c0:c0 + length] = False
    else:
        mask[r0:r0 + length, c0:c0 + k] = False
    assert np.array_equal(out[mask], M[mask])


@pytest.mark.parametrize("n,seed,kind", [(600, 1, "r"), (1200, 2, "g"), (1500, 3, "z")])
def test_split_solve_backward_stable(pkg, lapack, n, seed, kind):
    P_ = pkg.pencils
    if kind == "g":
        H, T = P_.graded_ht(n, seed)
    elif kind == "z":
        H, T = P_.random_ht(n, seed, 0.05)
    else:
        H, T = P_.random_ht(n, seed)
    S, P, Q, Z = (np.array(M, order="F", copy=True) for M in (H, T, np.eye(n), np.eye(n)))
    s = pkg.Solver(0)
    try:
        s.set_param("split", 8)
        ar, ai, be, info = s.solve_host(S, P, Q, Z)
    finally:
        s.close()
    assert info == 0
    r = lapack.residuals(H, T, S, P, Q, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])
    assert lapack.schur_structure_ok(S, P)
    So, Po, lar, lai, lbe, _, _, _ = lapack.dhgeqz(H, T)
    ok, ratio, _ = lapack.match_eigenvalues((lar, lai, lbe), (ar, ai, be), lapack.eig_tolerance(So, Po, H, T))
    assert ok, ratio
