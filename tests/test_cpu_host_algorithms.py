"""The library's window algorithms and iteration driver, built for the host
(tests/host_qz.cpp: one host thread, the same template source as the device
kernels, and a host backend in place of the kernels), checked against the
LAPACK DHGEQZ oracle without a GPU: backward errors and orthogonality
within 50*n*eps, generalized Schur structure, and eigenvalue sets within
the condition-scaled chordal tolerance."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("hostqz") / "libhostqz.so")
    cmd = ["g++", "-O2", "-shared", "-fPIC", "-std=c++17", "-Wno-unknown-pragmas", os.path.join(HERE, "host_qz.cpp"),
           "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, timeout=300)
    L = ctypes.CDLL(out)
    L.host_small_qz.argtypes = [ctypes.c_int] + [_pd] * 4
    L.host_small_qz.restype = ctypes.c_int
    L.host_small_qz_ms.argtypes = [ctypes.c_int] + [_pd] * 4
    L.host_small_qz_ms.restype = ctypes.c_int
    L.host_aed.argtypes = [ctypes.c_int] + [_pd] * 4 + [ctypes.c_double, ctypes.c_int, _pd, _pi]
    L.host_aed.restype = None
    L.host_solve.argtypes = [ctypes.c_int] + [_pd] * 4 + [ctypes.c_int] * 4 + [_pd] * 3 + [_pi]
    L.host_solve.restype = ctypes.c_int
    L.host_chase.argtypes = [ctypes.c_int] + [_pd] * 4 + [_pi, _pd] + [ctypes.c_int] * 3
    L.host_chase.restype = None
    L.host_solve_p.argtypes = [ctypes.c_int] + [_pd] * 4 + [_pi] + [_pd] * 3 + [_pi]
    L.host_solve_p.restype = ctypes.c_int
    L.host_barriers.argtypes = [ctypes.POINTER(ctypes.c_long), ctypes.c_int]
    L.host_barriers.restype = None
    L.host_gghrd.argtypes = [ctypes.c_int] * 3 + [_pd] * 4 + [ctypes.c_int] * 5
    L.host_gghrd.restype = ctypes.c_int
    L.host_hr_lartg.argtypes = [ctypes.c_double, ctypes.c_double, _pd]
    L.host_hr_lartg.restype = None
    L.host_onenorm_est.argtypes = [ctypes.c_int, _pd]
    L.host_onenorm_est.restype = ctypes.c_double
    L.host_set_pipe.argtypes = [ctypes.c_int]
    L.host_set_pipe.restype = None
    L.host_pipe_far_done.restype = ctypes.c_int
    L.host_swap11.argtypes = [_pd, _pd, ctypes.c_int, _pd]
    L.host_swap11.restype = None
    return L


def _p(a):
    return a.ctypes.data_as(_pd)


def _check(lapack, H, T, S, P, Q, Z, eig=None):
    r = lapack.residuals(H, T, S, P, Q, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])
    So, Po, lar, lai, lbe, _, _, _ = lapack.dhgeqz(H, T)
    e = eig if eig is not None else lapack.eig_from_schur(S, P)
    ok, ratio, _ = lapack.match_eigenvalues((lar, lai, lbe), e, lapack.eig_tolerance(So, Po, H, T))
    assert ok, ratio


@pytest.mark.parametrize("n,seed,zf", [(1, 0, 0.0), (2, 1, 0.0), (3, 2, 0.0), (17, 3, 0.0), (60, 4, 0.05),
                                       (80, 5, 0.0), (120, 6, 0.02)])
def test_host_window_qz(pkg, lapack, host, n, seed, zf):
    H, T = pkg.pencils.random_ht(n, seed, zf)
    S, P, Q, Z = (np.array(M, order="F", copy=True) for M in (H, T, np.eye(n), np.eye(n)))
    assert host.host_small_qz(n, _p(S), _p(P), _p(Q), _p(Z)) == 0
    _check(lapack, H, T, S, P, Q, Z)


@pytest.mark.parametrize("n,seed,kind", [(30, 1, "r"), (48, 2, "z"), (64, 3, "g"), (80, 4, "r"), (80, 5, "c"),
                                         (160, 6, "r")])
def test_host_window_qz_multishift(pkg, lapack, host, n, seed, kind):
    """Window QZ by small-bulge multishift sweeps (lockstep chains, shifts
    from the trailing block's eigenvalues): generalized Schur form, backward
    errors within 50 n eps and the eigenvalues of LAPACK DHGEQZ."""
    P_ = pkg.pencils
    H, T = {"r": lambda: P_.random_ht(n, seed), "z": lambda: P_.random_ht(n, seed, 0.05),
            "g": lambda: P_.graded_ht(n, seed), "c": lambda: P_.clustered_ht(n, seed, every=11, scale=1e-9)}[kind]()
    S, P, Q, Z = (np.array(M, order="F", copy=True) for M in (H, T, np.eye(n), np.eye(n)))
    assert host.host_small_qz_ms(n, _p(S), _p(P), _p(Q), _p(Z)) == 0
    assert lapack.schur_structure_ok(S, P)
    _check(lapack, H, T, S, P, Q, Z)


@pytest.mark.parametrize("nskip", [0, 4])
def test_host_aed_window(pkg, lapack, host, nskip):
    """AED on a window whose spike is small near the bottom: the deflated
    part is decoupled, the whole window stays an orthogonal equivalence."""
    n = 48
    H, T = pkg.pencils.clustered_ht(n, 7, every=11, scale=1e-9)
    s = 1e-7
    S, P, Q, Z = (np.array(M, order="F", copy=True) for M in (H, T, np.eye(n), np.eye(n)))
    shifts = np.zeros(3 * n)
    out3 = np.zeros(3, dtype=np.int32)
    host.host_aed(n, _p(S), _p(P), _p(Q), _p(Z), s, nskip, _p(shifts), out3.ctypes.data_as(_pi))
    m, st, tr = (int(v) for v in out3)
    assert st == 0 and 0 <= m <= n
    eps = np.finfo(float).eps
    assert np.linalg.norm(Q @ S @ Z.T - H) <= 50 * n * eps * np.linalg.norm(H)
    assert np.linalg.norm(Q @ P @ Z.T - T) <= 50 * n * eps * np.linalg.norm(T)
    assert np.linalg.norm(Q.T @ Q - np.eye(n)) <= 50 * n * eps
    # spike s * Q(0, :) is negligible over the deflated positions
    assert np.all(np.abs(s * Q[0, m:]) <= 1e-12 * max(1.0, np.abs(s)))
    assert np.all(np.tril(P, -1) == 0.0)


@pytest.mark.parametrize("n,seed,kind", [(150, 1, "r"), (230, 2, "z"), (260, 3, "g"), (200, 4, "c")])
def test_host_full_solve(pkg, lapack, host, n, seed, kind):
    """The iteration driver with AED windows of 32, chase windows of 40 and
    an endgame below 40, so that every phase runs: AED, multishift sweeps
    in waves of chains, zero chasing, the endgame and the finalisation."""
    P_ = pkg.pencils
    H, T = {"r": lambda: P_.random_ht(n, seed), "z": lambda: P_.random_ht(n, seed, 0.05),
            "g": lambda: P_.graded_ht(n, seed), "c": lambda: P_.clustered_ht(n, seed, every=30, scale=1e-8)}[kind]()
    S, P, Q, Z = (np.array(M, order="F", copy=True) for M in (H, T, np.zeros((n, n)), np.zeros((n, n))))
    ar, ai, be = np.zeros(n), np.zeros(n), np.zeros(n)
    st = np.zeros(5, dtype=np.int32)
    info = host.host_solve(n, _p(S), _p(P), _p(Q), _p(Z), 32, 40, 40, 4, _p(ar), _p(ai), _p(be),
                           st.ctypes.data_as(_pi))
    assert info == 0
    assert st[1] > 0 and st[2] > 0 and st[3] > 0  # AEDs, sweeps and chase windows ran
    assert lapack.schur_structure_ok(S, P)
    assert np.all(be >= 0)
    _check(lapack, H, T, S, P, Q, Z, eig=(ar, ai, be))


def _shift_set(rng, nb, cplx):
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


@pytest.mark.parametrize("n,nb,cplx", [(12, 1, False), (30, 3, False), (50, 5, True), (80, 12, True)])
def test_host_chase_matches_restatement(pkg, host, n, nb, cplx):
    """Lockstep chase of an introduced chain (the library's chase routine on
    the host) against the oracle's bulge-by-bulge PDHGEQZB/DHGEQZ5
    restatement from the same state (after the oracle's PDHGEQZA
    introduction): the same reflectors in exact arithmetic, so H, T, U, V
    agree to rounding (1e-9 relative)."""
    from oracle import qzref as R
    H, T = pkg.pencils.random_ht(n, 20 + n)
    rng = np.random.default_rng(n)
    sr, si, sb, coef = _shift_set(rng, nb, cplx)
    H1, T1, _, _ = R.sweep(H, T, sr, si, sb, phase=1)
    S_ref, P_ref, Q_ref, Z_ref = R.sweep(H1, T1, sr, si, sb, phase=2)
    bul, tmax = [], 0
    for k in range(nb):
        base = 3 * (nb - 1 - k) + 1
        thi = (n - 1) - base
        bul += [base, 0, thi, 0]
        tmax = max(tmax, thi)
    bul = np.array(bul, dtype=np.int32)
    S, P = np.array(H1, order="F", copy=True), np.array(T1, order="F", copy=True)
    U, V = np.eye(n, order="F"), np.eye(n, order="F")
    host.host_chase(n, _p(S), _p(P), _p(U), _p(V), bul.ctypes.data_as(_pi), _p(np.ascontiguousarray(coef)), nb,
                    tmax, n - 1)
    for a, b in ((S, S_ref), (P, P_ref), (U, Q_ref), (V, Z_ref)):
        assert np.linalg.norm(a - b) <= 1e-9 * max(1.0, np.linalg.norm(b)), np.linalg.norm(a - b)


def _edge_pencil(pkg, kind):
    P_ = pkg.pencils
    if kind == "n1":
        return P_.random_ht(1, 1)
    if kind == "n2":
        return P_.random_ht(2, 2)
    if kind == "zeros30":
        return P_.random_ht(200, 3, 0.3)
    if kind == "splits":
        H, T = P_.random_ht(240, 4)
        for k in (30, 31, 100, 180):
            H[k, k - 1] = 0.0
        return H, T
    if kind == "tinyT":
        H, T = P_.random_ht(200, 5)
        return H, T * 1e-200
    if kind == "hugeT":
        H, T = P_.random_ht(180, 6)
        return H, T * 1e150
    if kind == "Tdiag0":
        H, T = P_.random_ht(150, 7)
        T[np.arange(150), np.arange(150)] = 0.0
        return H, T
    if kind == "triH":
        H, T = P_.random_ht(150, 8)
        return np.triu(H), T
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["n1", "n2", "zeros30", "splits", "tinyT", "hugeT", "Tdiag0", "triH"])
def test_host_solve_edge_cases(pkg, lapack, host, kind):
    """Edge cases of the driver: orders 1 and 2, 30 % zero T diagonal,
    exact splits of H, T scaled by 1e-200 and 1e150 against H (T is balanced
    by a power of two for the iteration), an all-zero T diagonal and an
    already triangular H."""
    H, T = _edge_pencil(pkg, kind)
    n = H.shape[0]
    S, P, Q, Z = (np.array(M, order="F", copy=True) for M in (H, T, np.zeros((n, n)), np.zeros((n, n))))
    ar, ai, be = np.zeros(n), np.zeros(n), np.zeros(n)
    st = np.zeros(5, dtype=np.int32)
    info = host.host_solve(n, _p(S), _p(P), _p(Q), _p(Z), 32, 40, 40, 4, _p(ar), _p(ai), _p(be),
                           st.ctypes.data_as(_pi))
    assert info == 0
    assert lapack.schur_structure_ok(S, P)
    assert np.all(be >= 0)
    # the (alpha, beta) convention of the Schur form's blocks, also for
    # eigenvalues far from 1 in magnitude
    e = lapack.eig_from_schur(S, P)
    assert np.allclose(e[2], be, rtol=1e-12, atol=1e-300)
    # alpha as a complex number, relative to its modulus (the imaginary part
    # of a nearly real pair is ill-conditioned on its own)
    a_ref, a = e[0] + 1j * e[1], ar + 1j * ai
    assert np.all(np.abs(a - a_ref) <= 1e-12 * np.maximum(np.abs(a_ref), 1e-300))
    _check(lapack, H, T, S, P, Q, Z, eig=(ar, ai, be))


def test_host_solve_default_windows(pkg, lapack, host):
    """The library's default window sizes (AED 48, chase 80, endgame 80) on
    an N(0,1) pencil of order 500."""
    n = 500
    H, T = pkg.pencils.random_ht(n, 41)
    S, P, Q, Z = (np.array(M, order="F", copy=True) for M in (H, T, np.zeros((n, n)), np.zeros((n, n))))
    ar, ai, be = np.zeros(n), np.zeros(n), np.zeros(n)
    st = np.zeros(5, dtype=np.int32)
    info = host.host_solve(n, _p(S), _p(P), _p(Q), _p(Z), 48, 80, 80, 4, _p(ar), _p(ai), _p(be),
                           st.ctypes.data_as(_pi))
    assert info == 0 and st[2] > 0
    assert lapack.schur_structure_ok(S, P)
    _check(lapack, H, T, S, P, Q, Z, eig=(ar, ai, be))


def _solve_p(host, H, T, nw=32, wc=40, nmin=40, nskip=4, stall=300, swapfail=0, schur=1, ms=1):
    n = H.shape[0]
    S, P, Q, Z = (np.array(M, order="F", copy=True) for M in (H, T, np.zeros((n, n)), np.zeros((n, n))))
    ar, ai, be = np.zeros(n), np.zeros(n), np.zeros(n)
    st = np.zeros(5, dtype=np.int32)
    ip = np.array([nw, wc, nmin, nskip, stall, swapfail, schur, ms], dtype=np.int32)
    info = host.host_solve_p(n, _p(S), _p(P), _p(Q), _p(Z), ip.ctypes.data_as(_pi), _p(ar), _p(ai), _p(be),
                             st.ctypes.data_as(_pi))
    return info, (S, P, Q, Z), (ar, ai, be), st


def test_host_swap_failure_branch(pkg, lapack, host):
    """Every AED block swap reports failure: each AED keeps the deflations
    found before its first undeflatable block and re-reduces the window
    (the reference's branch at qzearly.f:321-326); the solve converges."""
    H, T = pkg.pencils.random_ht(220, 51)
    info, (S, P, Q, Z), eig, st = _solve_p(host, H, T, swapfail=1)
    assert info == 0 and st[1] > 0
    assert lapack.schur_structure_ok(S, P)
    _check(lapack, H, T, S, P, Q, Z, eig=eig)


def test_host_no_convergence_info(pkg, lapack, host):
    """Cyclic pencil (H a cyclic shift, T = I) with a stall limit of two
    iterations: INFO is the 1-based row where the iteration stopped
    (PDHGEQZ0.f:1207) and the pencil is still an orthogonal equivalence of
    the input."""
    n = 120
    H = np.zeros((n, n), order="F")
    H[np.arange(1, n), np.arange(n - 1)] = 1.0
    H[0, n - 1] = 1.0
    T = np.eye(n, order="F")
    info, (S, P, Q, Z), _, st = _solve_p(host, H, T, nw=48, wc=80, nmin=4, stall=2)
    assert 0 < info <= n, info
    r = lapack.residuals(H, T, S, P, Q, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])


@pytest.mark.parametrize("kind", ["r", "z"])
def test_host_job_e(pkg, lapack, host, kind):
    """JOB='E': far updates of H and T stop at the active block; the
    eigenvalues read from the diagonal blocks still match LAPACK, and Q, Z
    stay orthogonal."""
    n = 260
    H, T = pkg.pencils.random_ht(n, 52, 0.05 if kind == "z" else 0.0)
    info, (S, P, Q, Z), (ar, ai, be), st = _solve_p(host, H, T, schur=0)
    assert info == 0 and st[2] > 0
    So, Po, lar, lai, lbe, _, _, _ = lapack.dhgeqz(H, T)
    ok, ratio, _ = lapack.match_eigenvalues((lar, lai, lbe), (ar, ai, be), lapack.eig_tolerance(So, Po, H, T))
    assert ok, ratio
    eps = np.finfo(float).eps
    assert np.linalg.norm(Q.T @ Q - np.eye(n)) <= 50 * n * eps
    assert np.linalg.norm(Z.T @ Z - np.eye(n)) <= 50 * n * eps


def test_host_aed_barrier_budget(pkg, lapack, host):
    """The AED kernel's latency model: barriers per AED-routine call on a
    graded pencil with the default window 48 and the whole-window spike test.
    The multishift window QZ needs fewer barriers than double-shift sweeps;
    the total stays under the budget the kernel was designed to (a
    regression guard for the dependent-step count)."""
    H, T = pkg.pencils.graded_ht(900, 2)
    per = {}
    for ms in (0, 1):
        b = (ctypes.c_long * 6)()
        host.host_barriers(b, 1)
        info, (S, P, Q, Z), eig, st = _solve_p(host, H, T, nw=48, wc=80, nmin=80, nskip=0, ms=ms)
        assert info == 0
        host.host_barriers(b, 1)
        calls = max(1, b[5])
        per[ms] = [b[i] / calls for i in range(5)]
        _check(lapack, H, T, S, P, Q, Z, eig=eig)
    print("barriers per AED call (double shift / multishift):", per)
    assert per[1][1] < 0.8 * per[0][1]
    assert sum(per[1][1:]) < 6000


@pytest.mark.parametrize("n,seed,zf", [(3, 2, 0.0), (4, 1, 0.0), (17, 3, 0.0), (48, 7, 0.0), (60, 4, 0.05),
                                       (120, 6, 0.02)])
def test_host_pipelined_sweep_is_the_barrier_sweep(pkg, host, n, seed, zf):
    """The pipelined double-shift sweep (core step, then far step, per step
    on the host) splits the work between the core and the far threads so
    that every element sees the same operations in the same order: the
    window QZ gives bit-identical H, T, Q, Z to the two-barrier sweep."""
    H, T = pkg.pencils.random_ht(n, seed, zf)
    out = []
    try:
        for pipe in (0, 1):
            host.host_set_pipe(pipe)
            S, P, Q, Z = (np.array(M, order="F", copy=True) for M in (H, T, np.eye(n), np.eye(n)))
            info = host.host_small_qz(n, _p(S), _p(P), _p(Q), _p(Z))
            out.append((info, S, P, Q, Z))
            if pipe and n >= 3:
                assert host.host_pipe_far_done() > 0  # the pipelined sweep ran
    finally:
        host.host_set_pipe(0)
    assert out[0][0] == out[1][0] == 0
    for a, b in zip(out[0][1:], out[1][1:]):
        assert np.array_equal(a, b)


def test_host_pipelined_solve(pkg, lapack, host):
    """A whole host solve with pipelined window sweeps: Schur form, backward
    errors and LAPACK's eigenvalues."""
    n = 300
    H, T = pkg.pencils.random_ht(n, 11, 0.02)
    S, P, Q, Z = (np.array(M, order="F", copy=True) for M in (H, T, np.eye(n), np.eye(n)))
    ar, ai, be = np.zeros(n), np.zeros(n), np.zeros(n)
    st = np.zeros(8, dtype=np.int32)
    try:
        host.host_set_pipe(1)
        info = host.host_solve(n, _p(S), _p(P), _p(Q), _p(Z), 48, 80, 75, 0, _p(ar), _p(ai), _p(be),
                               st.ctypes.data_as(_pi))
    finally:
        host.host_set_pipe(0)
    assert info == 0
    assert lapack.schur_structure_ok(S, P)
    _check(lapack, H, T, S, P, Q, Z, (ar, ai, be))


def _swap11_cases():
    rng = np.random.default_rng(5)
    cases = [rng.standard_normal(6) for _ in range(200)]
    cases += [np.array([1.0, 2.0, 1.0, 1.0, 3.0, 1.0]),      # equal eigenvalues
              np.array([1.0, 2.0, 3.0, 1.0, 0.5, 0.0]),      # infinite eigenvalue last
              np.array([1.0, 2.0, 3.0, 0.0, 0.5, 2.0]),      # infinite eigenvalue first
              np.array([0.0, 2.0, 3.0, 1.0, 0.5, 2.0]),      # zero eigenvalue first
              np.array([1e-200, 1.0, 1e200, 1.0, 1e-150, 1.0]),
              np.array([2.0, 0.0, 3.0, 1.0, 0.0, 1.0])]      # already diagonal
    return cases


def test_host_swap11_two_rotations(host):
    """The two-rotation swap of 1x1 blocks: orthogonal factors, upper
    triangular result with the eigenvalues exchanged, Q^T (S,T) Z = (S2,T2)
    to rounding, and the same acceptance as the generalized Sylvester
    path."""
    eps = np.finfo(float).eps
    for a, b, c, d, e, f in _swap11_cases():
        S = np.array([[a, b], [0.0, c]], order="F")
        T = np.array([[d, e], [0.0, f]], order="F")
        out = np.zeros(17)
        host.host_swap11(_p(S), _p(T), 0, _p(out))
        ref = np.zeros(17)
        host.host_swap11(_p(S), _p(T), 1, _p(ref))
        # the two-rotation path may reject a swap of close eigenvalues that
        # the Sylvester path accepts (the library then falls back to it);
        # it never accepts one the Sylvester path rejects
        assert out[0] <= ref[0] or max(abs(S).max(), abs(T).max()) > 1e100
        if out[0] == 0:
            continue
        S2, T2 = out[1:5].reshape(2, 2, order="F"), out[5:9].reshape(2, 2, order="F")
        Q, Z = out[9:13].reshape(2, 2, order="F"), out[13:17].reshape(2, 2, order="F")
        assert np.allclose(Q.T @ Q, np.eye(2), atol=4 * eps) and np.allclose(Z.T @ Z, np.eye(2), atol=4 * eps)
        fn = np.hypot(np.linalg.norm(S), np.linalg.norm(T))
        assert np.linalg.norm(Q.T @ S @ Z - S2) <= 50 * eps * fn
        assert np.linalg.norm(Q.T @ T @ Z - T2) <= 50 * eps * fn
        assert S2[1, 0] == 0.0 and T2[1, 0] == 0.0
        # eigenvalue (c, f) now leads: chordal distance of (S2[0,0], T2[0,0]) to (c, f)
        u, v = np.array([S2[0, 0], T2[0, 0]]), np.array([c, f])
        chord = abs(u[0] * v[1] - u[1] * v[0]) / max(np.linalg.norm(u) * np.linalg.norm(v), 1e-300)
        assert chord <= 1e-10 or np.linalg.norm(v) == 0.0


# ---------------------------------------------------------------------------
# Hessenberg-triangular reduction: the device's launch sequence on the host
# ---------------------------------------------------------------------------
def _host_gghrd(host, A, B, ilo, ihi, W, order, cq=2, cz=2, qrows=0, Q=None, Z=None):
    n = A.shape[0]
    H, T = np.array(A, order="F", copy=True), np.array(B, order="F", copy=True)
    Q = np.array(Q if Q is not None else np.zeros((n, n)), order="F", copy=True)
    Z = np.array(Z if Z is not None else np.zeros((n, n)), order="F", copy=True)
    host.host_gghrd(n, ilo, ihi, _p(H), _p(T), _p(Q), _p(Z), W, cq, cz, qrows, order)
    return H, T, Q, Z


@pytest.mark.parametrize("n,W", [(2, 4), (5, 2), (12, 3), (40, 7), (40, 128), (150, 16), (260, 64)])
def test_host_gghrd_matches_dgghrd(host, lapack, n, W):
    """Windows of W pairs, with each launch's parts run in three orders:
    identical bits (the parts touch disjoint entries), and LAPACK DGGHRD's
    H, T, Q, Z to rounding (same rotations in the same order), exact
    Hessenberg-triangular structure, backward errors within 50 n eps."""
    rng = np.random.default_rng(100 + n + W)
    A = rng.standard_normal((n, n))
    B = np.triu(rng.standard_normal((n, n)))
    outs = [_host_gghrd(host, A, B, 0, n - 1, W, o) for o in (0, 1, 2)]
    for o in (1, 2):
        for k in range(4):
            assert np.array_equal(outs[0][k], outs[o][k])
    H, T, Q, Z = outs[0]
    H0, T0, Q0, Z0, info = lapack.dgghrd(A, B)
    assert info == 0
    assert not np.any(np.tril(H, -2)) and not np.any(np.tril(T, -1))
    tol = 1e-12 * max(1, n)
    assert np.abs(H - H0).max() <= tol * np.abs(H0).max()
    assert np.abs(T - T0).max() <= tol * np.abs(T0).max()
    assert np.abs(Q - Q0).max() <= tol and np.abs(Z - Z0).max() <= tol
    r = lapack.residuals(A, B, H, T, Q, Z)
    for key in ("h", "t", "q", "z"):
        assert r[key] <= 50 * r["neps"], (key, r[key] / r["neps"])


def test_host_gghrd_ilo_ihi_and_modes(host, lapack):
    """ILO/IHI sub-block, COMPQ/COMPZ in {N, V, I}, and the transposed Q
    the reference's PDGGHRD returns (Q <- G Q)."""
    rng = np.random.default_rng(7)
    n, ilo, ihi = 60, 10, 49  # 0-based block rows/columns 10..49
    A = np.triu(rng.standard_normal((n, n)))
    A[ilo:ihi + 1, ilo:ihi + 1] = rng.standard_normal((ihi - ilo + 1,) * 2)
    B = np.triu(rng.standard_normal((n, n)))
    Qi, _ = np.linalg.qr(rng.standard_normal((n, n)))
    Zi, _ = np.linalg.qr(rng.standard_normal((n, n)))
    codes = {0: "N", 1: "V", 2: "I"}
    for cq, cz in ((1, 1), (0, 2), (2, 0)):
        H, T, Q, Z = _host_gghrd(host, A, B, ilo, ihi, 9, 0, cq, cz, 0, Qi, Zi)
        Hl, Tl, Ql, Zl, info = lapack.dgghrd(A, B, codes[cq], codes[cz], ilo + 1, ihi + 1, Qi, Zi)
        assert info == 0
        assert np.abs(H - Hl).max() <= 1e-11 and np.abs(T - Tl).max() <= 1e-11
        if cq:
            assert np.abs(Q - Ql).max() <= 1e-12
        if cz:
            assert np.abs(Z - Zl).max() <= 1e-12
    Qt = _host_gghrd(host, A, B, ilo, ihi, 9, 0, 1, 1, 1, Qi.T.copy(), Zi)[2]
    Qn = _host_gghrd(host, A, B, ilo, ihi, 9, 0, 1, 1, 0, Qi, Zi)[2]
    assert np.array_equal(Qt.T, Qn)


def test_host_hr_lartg_matches_dlartg(host):
    """The reduction's rotation against LAPACK's DLARTG (the convention its
    H, T, Q, Z inherit): c >= 0, r with the sign of f, exact results for a
    zero f or g, rescaling far outside the unit range."""
    from scipy.linalg import lapack as sl
    vals = [0.0, 1.0, -1.0, 3.0, -4.0, 1e-200, -1e-200, 1e200, -1e200, 1e-310, 2.5e-150, 7e149]
    out = np.zeros(3)
    for f in vals:
        for g in vals:
            host.host_hr_lartg(f, g, _p(out))
            c, s, r = sl.dlartg(f, g)
            assert np.allclose(out, [c, s, r], rtol=4e-16, atol=0.0), (f, g, out, (c, s, r))
            if f == 0.0 or g == 0.0:
                assert tuple(out) == (c, s, r), (f, g, out, (c, s, r))


def _dlacn2_estimate(lapack, M):
    """LAPACK DLACN2 by reverse communication on an explicit matrix."""
    n = M.shape[0]
    v = np.zeros(n)
    x = np.zeros(n)
    isgn = np.zeros(n, dtype=np.int32)
    isave = np.zeros(3, dtype=np.int32)
    est = ctypes.c_double(0.0)
    kase = ctypes.c_int(0)
    nn = ctypes.c_int(n)
    f = lapack.lib().scipy_dlacn2_
    while True:
        f(ctypes.byref(nn), _p(v), _p(x), isgn.ctypes.data_as(_pi), ctypes.byref(est), ctypes.byref(kase),
          isave.ctypes.data_as(_pi))
        if kase.value == 0:
            return est.value
        x[:] = M @ x if kase.value == 1 else M.T @ x


@pytest.mark.parametrize("n,seed", [(1, 1), (2, 2), (7, 3), (40, 4), (120, 5)])
def test_host_onenorm_estimator_matches_dlacn2(host, lapack, n, seed):
    """The host restatement of the 1-norm estimator behind DTGSEN's Dif
    (onenorm.h) takes LAPACK DLACN2's steps: the same estimate on explicit
    matrices, random and with a dominant column, a lower bound of the true
    1-norm."""
    rng = np.random.default_rng(seed)
    for M in (rng.standard_normal((n, n)), np.linalg.inv(np.triu(rng.standard_normal((n, n))) + 3 * np.eye(n))):
        M = np.array(M, order="F")
        mine = host.host_onenorm_est(n, _p(M))
        ref = _dlacn2_estimate(lapack, M)
        assert abs(mine - ref) <= 1e-12 * ref, (mine, ref)
        assert mine <= np.abs(M).sum(axis=0).max() * (1 + 1e-12)


@pytest.mark.parametrize("n,ilo,ihi,W", [(2, 0, 1, 2), (3, 0, 2, 160), (9, 0, 8, 160), (9, 3, 3, 4), (9, 3, 4, 4),
                                          (9, 2, 5, 2), (33, 0, 32, 31), (33, 0, 32, 32)])
def test_host_gghrd_edge_cases(host, lapack, n, ilo, ihi, W):
    """Windows longer than a column, windows of two pairs, a column that
    exactly fills or just overflows a window, and ILO/IHI ranges with no
    column or one column to reduce: the same H, T, Q, Z as DGGHRD."""
    rng = np.random.default_rng(1000 + n + ilo + ihi + W)
    A = np.triu(rng.standard_normal((n, n)))
    A[ilo:ihi + 1, ilo:ihi + 1] = rng.standard_normal((ihi - ilo + 1,) * 2)
    B = np.triu(rng.standard_normal((n, n)))
    H, T, Q, Z = _host_gghrd(host, A, B, ilo, ihi, W, 0)
    H0, T0, Q0, Z0, info = lapack.dgghrd(A, B, "I", "I", ilo + 1, ihi + 1)
    assert info == 0
    for X, X0 in ((H, H0), (T, T0), (Q, Q0), (Z, Z0)):
        assert np.abs(X - X0).max() <= 1e-12 * max(1.0, np.abs(X0).max())
    assert not np.any(np.tril(H, -2)) and not np.any(np.tril(T, -1))
