"""ctypes wrapper of the oracle's C restatement (oracle/qzref.c).

Test infrastructure: an oracle for the tests and the CPU baseline, never the product."""
import ctypes
import os

import numpy as np

from . import build as _build
from . import lapack as _lapack

_lib = None
_pd = ctypes.POINTER(ctypes.c_double)


def lib():
    global _lib
    if _lib is None:
        _lapack.lib()  # load scipy's OpenBLAS globally first
        path = _build.build()
        L = ctypes.CDLL(path)
        L.qzref_pdhgeqz.restype = ctypes.c_int
        L.qzref_pdhgeqz.argtypes = [ctypes.c_char, ctypes.c_char, ctypes.c_char, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, _pd, _pd, _pd, _pd, ctypes.c_int, ctypes.c_int, _pd, _pd, _pd, _pd]
        L.qzref_pdhgeqz_ex.restype = ctypes.c_int
        L.qzref_pdhgeqz_ex.argtypes = L.qzref_pdhgeqz.argtypes + [ctypes.c_long, _pd, ctypes.c_long]
        L.qzref_dhgeqz5.restype = None
        L.qzref_dhgeqz5.argtypes = [ctypes.c_int, _pd, ctypes.c_int, _pd, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, _pd, _pd, _pd, _pd, _pd, ctypes.c_int]
        L.qzref_qzfcol2.restype = None
        L.qzref_qzfcol2.argtypes = [_pd, _pd, _pd, _pd, ctypes.c_int, _pd, ctypes.c_int, _pd]
        L.qzref_invhse3.restype = None
        L.qzref_invhse3.argtypes = [_pd, ctypes.c_int, _pd, _pd]
        L.qzref_sweep.restype = None
        L.qzref_sweep.argtypes = [ctypes.c_int, _pd, _pd, _pd, _pd, ctypes.c_int, ctypes.c_int, _pd, _pd, _pd,
                                  ctypes.c_int]
        L.qzref_pushoff.restype = None
        L.qzref_pushoff.argtypes = [_pd, ctypes.c_int, _pd, ctypes.c_int, ctypes.c_int, _pd, _pd, ctypes.c_int]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_pd)


STAT_NAMES = ("iters", "aeds", "sweeps", "small_subproblems", "infinite", "update_flops")


def pdhgeqz(H, T, job="S", compq="I", compz="I", ilo=1, ihi=None, nb=130, Q=None, Z=None, aed_limit=-1,
            aed_clock=None):
    """Run the restatement.  Returns (S, P, Q, Z, alphar, alphai, beta, info, stats).

    aed_limit >= 0 stops the run before that AED (info -2, for bounded
    CPU-baseline samples); aed_clock (float64 array) receives the seconds
    since the start at which each AED began."""
    n = H.shape[0]
    if ihi is None:
        ihi = n
    S = np.array(H, dtype=np.float64, order="F", copy=True)
    P = np.array(T, dtype=np.float64, order="F", copy=True)
    Qm = np.array(Q if Q is not None else np.eye(n), dtype=np.float64, order="F", copy=True)
    Zm = np.array(Z if Z is not None else np.eye(n), dtype=np.float64, order="F", copy=True)
    ar, ai, be = np.zeros(n), np.zeros(n), np.zeros(n)
    st = np.zeros(8)
    clk = aed_clock if aed_clock is not None else np.zeros(1)
    info = lib().qzref_pdhgeqz_ex(job.encode(), compq.encode(), compz.encode(), n, ilo, ihi, _p(S), _p(P), _p(Qm),
                                  _p(Zm), max(1, n), nb, _p(ar), _p(ai), _p(be), _p(st), int(aed_limit),
                                  _p(clk) if aed_clock is not None else None,
                                  len(clk) if aed_clock is not None else 0)
    return S, P, Qm, Zm, ar, ai, be, info, dict(zip(STAT_NAMES, st[:6].tolist()))


def sweep(H, T, sr, si, sb, phase=0):
    """One sweep with len(sr)//2 bulges (phase 0 full, 1 introduction only,
    2 chase of an introduced chain).  Returns (H', T', Q, Z)."""
    n = H.shape[0]
    S = np.array(H, dtype=np.float64, order="F", copy=True)
    P = np.array(T, dtype=np.float64, order="F", copy=True)
    Q = np.eye(n, order="F")
    Z = np.eye(n, order="F")
    sr = np.ascontiguousarray(sr, dtype=np.float64)
    si = np.ascontiguousarray(si, dtype=np.float64)
    sb = np.ascontiguousarray(sb, dtype=np.float64)
    lib().qzref_sweep(n, _p(S), _p(P), _p(Q), _p(Z), n, len(sr) // 2, _p(sr), _p(si), _p(sb), phase)
    return S, P, Q, Z
