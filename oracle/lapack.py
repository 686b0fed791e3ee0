"""LAPACK side of the oracle (test infrastructure only).

This module is part of the oracle, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it.

It calls FP64 LAPACK through ctypes in the OpenBLAS build that ships inside
scipy (``scipy.libs/libscipy_openblas-*.so``, symbols prefixed
``scipy_``).  The reference links LAPACK/ScaLAPACK unpinned
(``make.inc:5``, ``make_inc/make.inc_openmpi:6-7``; user guide: LAPACK >=
3.4.0); the routines used here are the ones the reference's path calls or
names:

* ``DHGEQZ``  -- the serial QZ the reference's kkqz replaces; its
  commented-out call is still in ``src/kkqz/qzearly.f:224-227``.  It is the
  eigenvalue-set oracle.
* ``DTGEVC`` + ``DTGSNA`` -- eigenvectors and reciprocal eigenvalue
  condition numbers used to scale the eigenvalue matching tolerance.
* ``DGGHRD``  -- Hessenberg-triangular reduction (``qzearly.f:449``; the
  semantics of the reference's PDGGHRD, ``src/ab2ht/PDGGHRD.f:13``), and
  ``DGGHD3``, its blocked form, as the host timing baseline.
* ``DTGSEN`` -- reordering of a generalized Schur form and the
  projection norms PL/PR (the role of the reference's PDTGSEN,
  ``src/reorder/PDTGSEN.f:1``), through scipy's wrapper of the same
  LAPACK.
* ``DGGBAL`` / ``DGGBAK`` -- balancing that produces the ILO/IHI the
  reference's driver takes (``PDHGEQZ.f:155-161``) and its back
  transformation; not in the reference, called from LAPACK.

Residual definitions follow ``tools/PQZHLPS.f`` (PCOMPRES):
||S - Q^T A Z||_F / ||A||_F, ||P - Q^T B Z||_F / ||B||_F and
||Q Q^T - I||_F / (n eps), the same for Z.
"""
from __future__ import annotations

import ctypes
import glob
import os

import numpy as np

_LIB = None


def openblas_path() -> str:
    import scipy
    d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError("scipy's bundled OpenBLAS was not found in %s" % d)
    return cands[0]


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(openblas_path(), mode=ctypes.RTLD_GLOBAL)
    return _LIB


_c = ctypes.c_char_p
_i = ctypes.POINTER(ctypes.c_int)
_d = ctypes.POINTER(ctypes.c_double)


def _ip(x: int):
    return ctypes.byref(ctypes.c_int(int(x)))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_d)


def set_threads(n: int) -> None:
    lib().scipy_openblas_set_num_threads(ctypes.c_int(int(n)))


def dhgeqz(H, T, job="S", compq="I", compz="I", Q=None, Z=None, ilo=1, ihi=None):
    """LAPACK DHGEQZ.  Returns (S, P, alphar, alphai, beta, Q, Z, info).

    Inputs are copied; arrays come back column-major."""
    n = H.shape[0]
    if ihi is None:
        ihi = n
    S = np.array(H, dtype=np.float64, order="F", copy=True)
    P = np.array(T, dtype=np.float64, order="F", copy=True)
    Qm = np.array(Q if Q is not None else np.eye(n), dtype=np.float64, order="F", copy=True)
    Zm = np.array(Z if Z is not None else np.eye(n), dtype=np.float64, order="F", copy=True)
    ar = np.zeros(n)
    ai = np.zeros(n)
    be = np.zeros(n)
    info = ctypes.c_int(0)
    ld = max(1, n)
    f = lib().scipy_dhgeqz_
    # workspace query
    wq = np.zeros(1)
    f(_c(job.encode()), _c(compq.encode()), _c(compz.encode()), _ip(n), _ip(ilo), _ip(ihi),
      _dp(S), _ip(ld), _dp(P), _ip(ld), _dp(ar), _dp(ai), _dp(be), _dp(Qm), _ip(ld),
      _dp(Zm), _ip(ld), _dp(wq), _ip(-1), ctypes.byref(info),
      ctypes.c_size_t(1), ctypes.c_size_t(1), ctypes.c_size_t(1))
    lw = max(1, int(wq[0]))
    work = np.zeros(lw)
    f(_c(job.encode()), _c(compq.encode()), _c(compz.encode()), _ip(n), _ip(ilo), _ip(ihi),
      _dp(S), _ip(ld), _dp(P), _ip(ld), _dp(ar), _dp(ai), _dp(be), _dp(Qm), _ip(ld),
      _dp(Zm), _ip(ld), _dp(work), _ip(lw), ctypes.byref(info),
      ctypes.c_size_t(1), ctypes.c_size_t(1), ctypes.c_size_t(1))
    return S, P, ar, ai, be, Qm, Zm, info.value


def dgghrd(A, B, compq="I", compz="I", ilo=1, ihi=None, Q=None, Z=None):
    """LAPACK DGGHRD on (A, B) with B already upper triangular (1-based
    ilo/ihi; Q, Z are the input matrices for compq/compz = 'V')."""
    n = A.shape[0]
    ihi = n if ihi is None else ihi
    H = np.array(A, dtype=np.float64, order="F", copy=True)
    T = np.array(B, dtype=np.float64, order="F", copy=True)
    Q = np.array(Q if Q is not None else np.eye(n), dtype=np.float64, order="F", copy=True)
    Z = np.array(Z if Z is not None else np.eye(n), dtype=np.float64, order="F", copy=True)
    info = ctypes.c_int(0)
    ld = max(1, n)
    lib().scipy_dgghrd_(_c(compq.encode()), _c(compz.encode()), _ip(n), _ip(ilo), _ip(ihi),
                        _dp(H), _ip(ld), _dp(T), _ip(ld), _dp(Q), _ip(ld), _dp(Z), _ip(ld),
                        ctypes.byref(info), ctypes.c_size_t(1), ctypes.c_size_t(1))
    return H, T, Q, Z, info.value


def dgghd3(A, B, compq="I", compz="I"):
    """LAPACK DGGHD3 (the blocked Hessenberg-triangular reduction, the
    host baseline for timing) on (A, B) with B upper triangular."""
    n = A.shape[0]
    H = np.array(A, dtype=np.float64, order="F", copy=True)
    T = np.array(B, dtype=np.float64, order="F", copy=True)
    Q = np.eye(n, order="F")
    Z = np.eye(n, order="F")
    info = ctypes.c_int(0)
    ld = max(1, n)

    def call(work, lwork):
        lib().scipy_dgghd3_(_c(compq.encode()), _c(compz.encode()), _ip(n), _ip(1), _ip(n), _dp(H), _ip(ld),
                            _dp(T), _ip(ld), _dp(Q), _ip(ld), _dp(Z), _ip(ld), _dp(work), ctypes.byref(lwork),
                            ctypes.byref(info), ctypes.c_size_t(1), ctypes.c_size_t(1))

    w = np.zeros(1)
    call(w, ctypes.c_int(-1))
    lw = max(1, int(w[0]))
    call(np.zeros(lw), ctypes.c_int(lw))
    return H, T, Q, Z, info.value


def dggbal(A, B, job="B"):
    """LAPACK DGGBAL.  Returns (A', B', ilo, ihi, lscale, rscale, info)
    with 1-based ilo/ihi and LAPACK's lscale/rscale (permutation indices,
    1-based, outside ilo..ihi; scale factors inside)."""
    n = A.shape[0]
    Ab = np.array(A, dtype=np.float64, order="F", copy=True)
    Bb = np.array(B, dtype=np.float64, order="F", copy=True)
    ilo = ctypes.c_int(0)
    ihi = ctypes.c_int(0)
    ls = np.zeros(max(1, n))
    rs = np.zeros(max(1, n))
    work = np.zeros(max(1, 6 * n))
    info = ctypes.c_int(0)
    ld = max(1, n)
    lib().scipy_dggbal_(_c(job.encode()), _ip(n), _dp(Ab), _ip(ld), _dp(Bb), _ip(ld), ctypes.byref(ilo),
                        ctypes.byref(ihi), _dp(ls), _dp(rs), _dp(work), ctypes.byref(info), ctypes.c_size_t(1))
    return Ab, Bb, ilo.value, ihi.value, ls[:n], rs[:n], info.value


def dtgsen(S, P, Q, Z, select, ijob=0):
    """LAPACK DTGSEN.  Returns (S', P', alphar, alphai, beta, Q', Z', m,
    pl, pr, dif, info); dif holds the Dif estimates for ijob >= 2."""
    import scipy.linalg.lapack as SL
    n = S.shape[0]
    lw = 4 * n + 16 + 2 * n * n
    r = SL.dtgsen(np.asarray(select, dtype=np.int32), np.array(S, order="F"), np.array(P, order="F"),
                  np.array(Q, order="F"), np.array(Z, order="F"), ijob=ijob, lwork=lw, liwork=n + 6 + 2 * n * n)
    a, b, ar, ai, be, q, z, m, pl, pr, dif, info = r
    return a, b, ar, ai, be, q, z, int(m), float(pl), float(pr), np.array(dif), int(info)


def dggbak(V, ilo, ihi, lscale, rscale, side="R", job="B"):
    """LAPACK DGGBAK: back-transform the columns of V (n x m)."""
    n, m = V.shape
    Vb = np.array(V, dtype=np.float64, order="F", copy=True)
    ls = np.array(lscale, dtype=np.float64, copy=True)
    rs = np.array(rscale, dtype=np.float64, copy=True)
    info = ctypes.c_int(0)
    lib().scipy_dggbak_(_c(job.encode()), _c(side.encode()), _ip(n), _ip(ilo), _ip(ihi), _dp(ls), _dp(rs),
                        _ip(m), _dp(Vb), _ip(max(1, n)), ctypes.byref(info), ctypes.c_size_t(1), ctypes.c_size_t(1))
    return Vb, info.value


def eig_condition(S, P, Q=None, Z=None):
    """Reciprocal condition numbers s(j) of the eigenvalues of the
    generalized Schur form (S, P) (DTGEVC + DTGSNA, JOB='E', HOWMNY='A').

    Returns an array of length n (one entry per eigenvalue, a complex pair
    shares its value)."""
    n = S.shape[0]
    S = np.array(S, dtype=np.float64, order="F", copy=True)
    P = np.array(P, dtype=np.float64, order="F", copy=True)
    VL = np.eye(n, order="F")
    VR = np.eye(n, order="F")
    ld = max(1, n)
    m = ctypes.c_int(0)
    info = ctypes.c_int(0)
    sel = np.ones(n, dtype=np.int32)
    work = np.zeros(6 * n + 16)
    lib().scipy_dtgevc_(_c(b"B"), _c(b"A"), sel.ctypes.data_as(_i), _ip(n), _dp(S), _ip(ld),
                        _dp(P), _ip(ld), _dp(VL), _ip(ld), _dp(VR), _ip(ld), _ip(n),
                        ctypes.byref(m), _dp(work), ctypes.byref(info),
                        ctypes.c_size_t(1), ctypes.c_size_t(1))
    if info.value != 0:
        raise RuntimeError("DTGEVC info=%d" % info.value)
    s = np.zeros(n)
    dif = np.zeros(n)
    lwork = 2 * n * (n + 2) + 16
    work2 = np.zeros(lwork)
    iwork = np.zeros(n + 6, dtype=np.int32)
    lib().scipy_dtgsna_(_c(b"E"), _c(b"A"), sel.ctypes.data_as(_i), _ip(n), _dp(S), _ip(ld),
                        _dp(P), _ip(ld), _dp(VL), _ip(ld), _dp(VR), _ip(ld), _dp(s), _dp(dif),
                        _ip(n), ctypes.byref(m), _dp(work2), _ip(lwork),
                        iwork.ctypes.data_as(_i), ctypes.byref(info),
                        ctypes.c_size_t(1), ctypes.c_size_t(1))
    if info.value != 0:
        raise RuntimeError("DTGSNA info=%d" % info.value)
    return s


# ----------------------------------------------------------------------------
# residuals (tools/PQZHLPS.f PCOMPRES definitions)
# ----------------------------------------------------------------------------

def residuals(H0, T0, S, P, Q, Z, Q0=None, Z0=None):
    """Backward errors and orthogonality of a generalized Schur form.

    Q0 H0 Z0^T = Q S Z^T is checked (Q0 = Z0 = I for COMPQ = COMPZ = 'I').
    Returns dict with keys ``h``, ``t`` (relative Frobenius backward errors),
    ``q``, ``z`` (||Q^T Q - I||_F) -- all unscaled -- and the n*eps unit."""
    n = H0.shape[0]
    eps = np.finfo(np.float64).eps
    if Q0 is None:
        lhsH = Q.T @ H0 @ Z
        lhsT = Q.T @ T0 @ Z
    else:
        lhsH = Q.T @ (Q0 @ H0 @ Z0.T) @ Z
        lhsT = Q.T @ (Q0 @ T0 @ Z0.T) @ Z
    hn = np.linalg.norm(H0) or 1.0
    tn = np.linalg.norm(T0) or 1.0
    I = np.eye(n)
    return dict(
        h=float(np.linalg.norm(lhsH - S) / hn),
        t=float(np.linalg.norm(lhsT - P) / tn),
        q=float(np.linalg.norm(Q.T @ Q - I)),
        z=float(np.linalg.norm(Z.T @ Z - I)),
        neps=float(n * eps),
    )


def schur_structure_ok(S, P, tol=0.0):
    """S quasi upper triangular (no two consecutive nonzero subdiagonals,
    nothing below the first subdiagonal), P upper triangular, and P's 2x2
    diagonal blocks diagonal with positive entries (DLAGV2 normalisation)."""
    n = S.shape[0]
    if n == 0:
        return True
    if np.any(np.tril(S, -2) != 0.0) or np.any(np.tril(P, -1) != 0.0):
        return False
    sub = np.diag(S, -1)
    nz = sub != 0.0
    if np.any(nz[1:] & nz[:-1]):
        return False
    for j in np.nonzero(nz)[0]:
        if P[j, j + 1] != 0.0 or P[j, j] <= 0.0 or P[j + 1, j + 1] <= 0.0:
            return False
    return True


def eig_from_schur(S, P):
    """(alphar, alphai, beta) read from a standardised Schur form."""
    n = S.shape[0]
    ar = np.zeros(n)
    ai = np.zeros(n)
    be = np.zeros(n)
    j = 0
    while j < n:
        if j + 1 < n and S[j + 1, j] != 0.0:
            a = S[j:j + 2, j:j + 2]
            b11, b22 = P[j, j], P[j + 1, j + 1]
            # eigenvalues of the 2x2 pencil with diagonal B, computed on
            # diag(B)^-1 A scaled by a power of two (eigenvalues far from 1
            # in magnitude), the scale folded back into beta's factor
            m = np.linalg.solve(np.diag([b11, b22]), a)
            mx = np.abs(m).max()
            e = int(np.frexp(mx)[1]) if mx > 0 and np.isfinite(mx) else 0
            lam = np.linalg.eigvals(np.ldexp(m, -e))
            lam = lam[np.argsort(-lam.imag)]
            s11, s22 = np.ldexp(b11, e), np.ldexp(b22, e)
            ar[j], ai[j], be[j] = lam[0].real * s11, abs(lam[0].imag) * s11, b11
            ar[j + 1], ai[j + 1], be[j + 1] = lam[0].real * s22, -abs(lam[0].imag) * s22, b22
            j += 2
        else:
            ar[j], ai[j], be[j] = S[j, j], 0.0, P[j, j]
            j += 1
    return ar, ai, be


# ----------------------------------------------------------------------------
# eigenvalue-set matching
# ----------------------------------------------------------------------------

def _sphere(ar, ai, be):
    """Map (alpha, beta) to the unit-diameter Riemann sphere; the chordal
    distance between two eigenvalues is the Euclidean distance of the
    images."""
    a = ar + 1j * ai
    b = be.astype(np.complex128)
    # scale by the larger modulus first so that the squares below neither
    # underflow nor overflow (pencils with entries near the range limits)
    sc = np.maximum(np.abs(a), np.abs(b))
    sc[sc == 0] = 1.0
    a = a / sc
    b = b / sc
    nrm = np.sqrt(np.abs(a) ** 2 + np.abs(b) ** 2)
    nrm[nrm == 0] = 1.0
    a = a / nrm
    b = b / nrm
    # make beta real non-negative (projective normalisation)
    ph = np.where(np.abs(b) > 0, np.conj(b) / np.maximum(np.abs(b), 1e-300), 1.0)
    a = a * ph
    b = np.abs(b)
    # stereographic image of lambda = a/b on sphere of diameter 1
    d = np.abs(a) ** 2 + b ** 2
    x = (a.real * b) / d
    y = (a.imag * b) / d
    z = (np.abs(a) ** 2) / d - 0.5
    return np.stack([x, y, z], axis=1)


def chordal(ar1, ai1, be1, ar2, ai2, be2):
    p = _sphere(np.atleast_1d(ar1), np.atleast_1d(ai1), np.atleast_1d(be1))
    q = _sphere(np.atleast_1d(ar2), np.atleast_1d(ai2), np.atleast_1d(be2))
    return np.linalg.norm(p - q, axis=1)


def match_eigenvalues(e1, e2, tol):
    """Match two eigenvalue sets e = (alphar, alphai, beta) as multisets.

    ``tol`` is an array of per-eigenvalue chordal tolerances for e1.
    Returns (ok, max_ratio, dist) where max_ratio = max_j dist_j / tol_j
    over the optimal assignment (minimum total chordal distance)."""
    from scipy.optimize import linear_sum_assignment
    from scipy.spatial import cKDTree

    p = _sphere(*e1)
    q = _sphere(*e2)
    n = p.shape[0]
    if n == 0:
        return True, 0.0, np.zeros(0)
    if q.shape[0] != n:
        return False, np.inf, np.full(n, np.inf)
    tol = np.broadcast_to(np.asarray(tol, dtype=np.float64), (n,))
    k = min(n, 12)
    tree = cKDTree(q)
    dist, idx = tree.query(p, k=k)
    if k == 1:
        dist = dist[:, None]
        idx = idx[:, None]
    # greedy by increasing distance, measured in units of each tolerance
    scaled = dist / np.maximum(tol, 1e-300)[:, None]
    order = np.argsort(scaled, axis=None, kind="stable")
    used_p = np.zeros(n, dtype=bool)
    used_q = np.zeros(n, dtype=bool)
    dd = np.full(n, np.inf)
    for flat in order:
        i, j = divmod(int(flat), k)
        qi = int(idx[i, j])
        if used_p[i] or used_q[qi]:
            continue
        used_p[i] = True
        used_q[qi] = True
        dd[i] = dist[i, j]
    rest_p = np.nonzero(~used_p)[0]
    if rest_p.size:
        # optimal assignment among what greedy left over (small, dense)
        rest_q = np.nonzero(~used_q)[0]
        C = np.linalg.norm(p[rest_p][:, None, :] - q[rest_q][None, :, :], axis=2)
        r, c = linear_sum_assignment(C / np.maximum(tol[rest_p], 1e-300)[:, None])
        dd[rest_p[r]] = C[r, c]
    ratio = dd / np.maximum(tol, 1e-300)
    return bool(np.all(ratio <= 1.0)), float(ratio.max()), dd


def eig_tolerance(S, P, H0, T0, factor=50.0):
    """Per-eigenvalue chordal tolerance factor * n * eps * ||(H,T)||_F / s_j,
    s_j the DTGSNA reciprocal condition number of eigenvalue j in the
    oracle's Schur form (S, P).  Clamped to [factor * n * eps, 2]."""
    n = S.shape[0]
    eps = np.finfo(np.float64).eps
    s = eig_condition(S, P)
    # orthogonal equivalence keeps ||(S,P)||_F = ||(H0,T0)||_F; LAPACK's
    # first-order bound is chord <= eps * ||(A,B)||_F / s_j per unit of
    # relative backward error
    nrm = np.hypot(np.linalg.norm(H0), np.linalg.norm(T0))
    s = np.maximum(s, 1e-300)
    tol = factor * n * eps * nrm / s
    return np.clip(tol, factor * n * eps, 2.0)
