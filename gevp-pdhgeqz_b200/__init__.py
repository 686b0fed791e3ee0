"""B200-native multishift QZ behind the PDHGEQZ interface.

Host-side mirror of the reference's operator interface
(``src/pdhgeqz/PDHGEQZ.f:15-31``).  All numerical work runs in the CUDA
library ``libb200qz.so`` built next to this file (``build.py``); importing
this module does not need a GPU, but every solve does and fails loudly
without the library or a device.

Entry points
------------
``pdhgeqz(job, compq, compz, H, T, Q, Z, ilo=1, ihi=None, nb=64)``
    Same argument meaning and INFO codes as the Fortran routine on a 1x1
    grid; arrays are Fortran-ordered numpy float64 and are overwritten in
    place.  Goes through the exported ``pdhgeqz_`` symbol (the drop-in).
``Solver`` (device context)
    ``solve_device`` works on CUDA buffers that already live in HBM
    (column-major, one leading dimension), ``solve_host`` copies numpy
    arrays in and out.
"""
from __future__ import annotations

import ctypes
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libb200qz.so")

_lib = None


def _submodule(base):
    name = "gevp_pdhgeqz_b200_" + base
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(HERE, base + ".py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


pencils = _submodule("pencils")
shard = _submodule("shard")
learned = _submodule("learned")

_i = ctypes.c_int
_d = ctypes.c_double
_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_c = ctypes.c_char

EXPORTS = (
    "pdhgeqz_", "kkqzconf_", "b200qz_create", "b200qz_destroy", "b200qz_solve_dev",
    "b200qz_solve_host", "b200qz_get_stats", "b200qz_set_params", "b200qz_aed_window",
    "b200qz_chase_window", "b200qz_update", "b200qz_set_param", "b200qz_solve_batched_dev",
    "b200qz_batched_seconds", "b200qz_batched_autotune", "b200qz_batched_config",
    "b200qz_solve_batched_noalloc", "b200qz_policy_nparams", "b200qz_set_policy", "b200qz_policy_features",
    "b200qz_mlp_forward", "b200qz_mlp_backward", "b200qz_mlp_train", "b200qz_update_split",
    "b200qz_gghrd_dev", "b200qz_gghrd_host", "pdgghrd_",
)

STAT_NAMES = ("seconds", "iters", "aeds", "aed_deflations", "sweeps", "chains", "windows",
              "endgames", "inf_steps", "shifts", "update_flops", "window_bytes",
              "ms_scan", "ms_aed", "ms_aed_update", "ms_chase", "ms_chase_update", "ms_inf", "ms_final",
              "ms_aed_smallqz", "ms_aed_reorder", "ms_aed_spike", "ms_aed_hessred", "launches",
              "aed_failures", "exceptional_sweeps", "remaining", "stop_ktop", "stop_kbot", "last_aed_fraction",
              "policy_calls", "aed_bytes", "aed_launches", "chase_bytes", "chase_launches",
              "aed_qz_steps", "aed_swaps", "aed_rotations", "aed_ms_sweeps")


def lib() -> ctypes.CDLL:
    """Load libb200qz.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            "libb200qz.so is missing: run `python gevp-pdhgeqz_b200/build.py` "
            "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    L.pdhgeqz_.restype = None
    L.pdhgeqz_.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _pi, _pi, _pi,
                           _pd, _pi, _pd, _pi, _pd, _pd, _pd, _pd, _pi, _pd, _pi, _pd, _pi, _pi, _pi,
                           _pi, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t]
    L.kkqzconf_.restype = None
    L.kkqzconf_.argtypes = [_pd]
    L.b200qz_create.restype = _i
    L.b200qz_create.argtypes = [ctypes.POINTER(_vp), _i]
    L.b200qz_destroy.restype = None
    L.b200qz_destroy.argtypes = [_vp]
    L.b200qz_solve_dev.restype = _i
    L.b200qz_solve_dev.argtypes = [_vp, _c, _c, _c, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _vp, _vp, _vp]
    L.b200qz_solve_host.restype = _i
    L.b200qz_solve_host.argtypes = [_vp, _c, _c, _c, _i, _i, _i, _pd, _i, _pd, _i, _pd, _i, _pd, _i,
                                    _pd, _pd, _pd]
    L.b200qz_get_stats.restype = _i
    L.b200qz_get_stats.argtypes = [_vp, _pd, _i]
    L.b200qz_set_params.restype = _i
    L.b200qz_set_params.argtypes = [_vp, _i, _i, _i, _i, _i, _i]
    L.b200qz_aed_window.restype = _i
    L.b200qz_aed_window.argtypes = [_vp, _vp, _vp, _i, _i, _i, _i, _vp, _vp, _vp, _pi]
    L.b200qz_chase_window.restype = _i
    L.b200qz_chase_window.argtypes = [_vp, _vp, _vp, _i, _i, _i, _i, _pi, _pd, _i, _i, _vp, _vp]
    L.b200qz_set_param.restype = _i
    L.b200qz_set_param.argtypes = [_vp, ctypes.c_char_p, _d]
    L.b200qz_update.restype = _i
    L.b200qz_update.argtypes = [_vp, _c, _vp, _i, _i, _i, _i, _vp, _i, _i]
    L.b200qz_update_split.argtypes = [_vp, _c, _vp, _i, _i, _i, _i, _vp, _i, _i, _i]
    L.b200qz_update_split.restype = _i
    _pl = ctypes.POINTER(ctypes.c_longlong)
    L.b200qz_solve_batched_dev.argtypes = [_vp, _i, _pi, _pl, _pl] + [_vp] * 8
    L.b200qz_solve_batched_dev.restype = _i
    L.b200qz_batched_seconds.argtypes = [_vp]
    L.b200qz_batched_seconds.restype = _d
    L.b200qz_batched_autotune.argtypes = [_vp, _i, _pi, _pl, _vp, _vp, _i, _pd]
    L.b200qz_batched_autotune.restype = _i
    L.b200qz_batched_config.argtypes = [_vp, _pi, _pi, _pi]
    L.b200qz_batched_config.restype = _i
    L.b200qz_solve_batched_noalloc.argtypes = [_i, _pi, _pl, _pl] + [_vp] * 9
    L.b200qz_solve_batched_noalloc.restype = _i
    _pf = ctypes.POINTER(ctypes.c_float)
    L.b200qz_policy_nparams.argtypes = []
    L.b200qz_policy_nparams.restype = _i
    L.b200qz_set_policy.argtypes = [_vp, _pf, _i]
    L.b200qz_set_policy.restype = _i
    L.b200qz_policy_features.argtypes = [_vp, _vp, _i, _i, _i, _d, _pf]
    L.b200qz_policy_features.restype = _i
    L.b200qz_mlp_forward.argtypes = [_vp, _vp, _i, _vp, _vp, _vp, _vp]
    L.b200qz_mlp_forward.restype = _i
    L.b200qz_mlp_backward.argtypes = [_vp, _vp, _vp, _i] + [_vp] * 8
    L.b200qz_mlp_backward.restype = _i
    L.b200qz_mlp_train.argtypes = [_vp, _vp, _vp, _i, _i, ctypes.c_float, _pf]
    L.b200qz_mlp_train.restype = _i
    for f in ("b200qz_ggbal_dev", "b200qz_ggbal_host"):
        getattr(L, f).argtypes = [_vp, _c, _i, _vp, _i, _vp, _i, _pi, _pi, _pd, _pd]
        getattr(L, f).restype = _i
    L.b200qz_tgsen_host.argtypes = [_vp, _i, _i, _i, _pi, _i] + [_vp, _i] * 4 + [_pd] * 3 + [_pi, _pd, _pd, _pd, _pi]
    L.b200qz_tgsen_host.restype = _i
    L.b200qz_tgsen_dev.argtypes = [_vp, _i, _i, _i, _pi, _i] + [_vp, _i] * 4 + [_vp] * 3 + [_pi, _pd, _pd, _pd, _pi, _pi]
    L.b200qz_tgsen_dev.restype = _i
    for f in ("b200qz_ggbak_dev", "b200qz_ggbak_host"):
        getattr(L, f).argtypes = [_vp, _c, _c, _i, _i, _i, _pd, _pd, _i, _vp, _i]
        getattr(L, f).restype = _i
    for f in ("b200qz_gghrd_dev", "b200qz_gghrd_host"):
        getattr(L, f).argtypes = [_vp, _c, _c, _i, _i, _i] + [_vp, _i] * 4
        getattr(L, f).restype = _i
    L.pdgghrd_.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _pi, _pi, _pi, _vp, _pi, _vp, _pi, _vp, _pi, _vp, _pi,
                           _pd, _pi, _pi, ctypes.c_size_t, ctypes.c_size_t]
    L.pdgghrd_.restype = None
    _lib = L
    return L


def _p(a: np.ndarray):
    return a.ctypes.data_as(_pd)


def _ip(v: int):
    return ctypes.byref(ctypes.c_int(int(v)))


def descriptor(n: int, nb: int, lld: int, ctxt: int = 0) -> np.ndarray:
    """ScaLAPACK array descriptor of a full n x n matrix on a 1x1 grid:
    [DTYPE=1, CTXT, M, N, MB, NB, RSRC=0, CSRC=0, LLD]."""
    return np.array([1, ctxt, n, n, nb, nb, 0, 0, max(1, lld)], dtype=np.int32)


def kkqzconf(eps: float = np.finfo(np.float64).eps) -> None:
    """Accepted no-op (see include/b200qz.h)."""
    lib().kkqzconf_(ctypes.byref(ctypes.c_double(eps)))


def pdhgeqz(job, compq, compz, H, T, Q=None, Z=None, ilo=1, ihi=None, nb=64,
            ldwork=None, liwork=None, descs=None):
    """Call the ``pdhgeqz_`` drop-in exactly as a Fortran caller would.

    H, T (and Q, Z when COMPQ/COMPZ are not 'N') are Fortran-ordered float64
    numpy arrays, overwritten in place.  Returns (alphar, alphai, beta, info);
    with ldwork == -1 or liwork == -1 the workspace sizes come back in
    place of alphar/alphai as (dwork[0], iwork[0])."""
    L = lib()
    n = H.shape[0]
    if ihi is None:
        ihi = n
    for nm, a in (("H", H), ("T", T), ("Q", Q), ("Z", Z)):
        if a is not None and not (a.dtype == np.float64 and a.flags.f_contiguous):
            raise ValueError("%s must be a Fortran-ordered float64 array" % nm)
    Qa = Q if Q is not None else np.zeros((1, 1), order="F")
    Za = Z if Z is not None else np.zeros((1, 1), order="F")
    if descs is None:
        descs = [descriptor(n, nb, a.shape[0]) for a in (H, T, Qa, Za)]
    ar = np.zeros(max(1, n))
    ai = np.zeros(max(1, n))
    be = np.zeros(max(1, n))
    if ldwork is None:
        ldwork = max(1, n * nb)
    if liwork is None:
        liwork = max(1, 2 * n)
    dwork = np.zeros(max(1, ldwork if ldwork > 0 else 1))
    iwork = np.zeros(max(1, liwork if liwork > 0 else 1), dtype=np.int32)
    info = ctypes.c_int(0)
    dp = [d.ctypes.data_as(_pi) for d in descs]
    L.pdhgeqz_(job.encode(), compq.encode(), compz.encode(), _ip(n), _ip(ilo), _ip(ihi),
               _p(H), dp[0], _p(T), dp[1], _p(ar), _p(ai), _p(be), _p(Qa), dp[2], _p(Za), dp[3],
               _p(dwork), _ip(ldwork), iwork.ctypes.data_as(_pi), _ip(liwork), ctypes.byref(info),
               1, 1, 1)
    if ldwork == -1 or liwork == -1:
        return dwork[0], iwork[0], None, info.value
    return ar[:n], ai[:n], be[:n], info.value


class Solver:
    """A device context (stream + workspace) of the CUDA solver."""

    def __init__(self, device: int = 0):
        L = lib()
        h = _vp()
        rc = L.b200qz_create(ctypes.byref(h), int(device))
        if rc != 0:
            raise RuntimeError("b200qz_create failed with CUDA error %d" % rc)
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            lib().b200qz_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_params(self, nw_max=-1, w_chase=-1, nmin=-1, nibble=-1, ns_max=-1, maxit_factor=-1):
        rc = lib().b200qz_set_params(self._h, nw_max, w_chase, nmin, nibble, ns_max, maxit_factor)
        if rc != 0:
            raise ValueError("b200qz_set_params: bad argument %d" % -rc)

    def set_param(self, name: str, value) -> None:
        rc = lib().b200qz_set_param(self._h, name.encode(), float(value))
        if rc != 0:
            raise ValueError("b200qz_set_param(%s=%r) failed: %d" % (name, value, rc))

    def set_policy(self, params) -> None:
        """Load learned (nw, ns) MLP parameters (float32 array of
        b200qz_policy_nparams() values); None switches back to the table."""
        if params is None:
            rc = lib().b200qz_set_policy(self._h, None, 0)
        else:
            p = np.ascontiguousarray(params, dtype=np.float32)
            rc = lib().b200qz_set_policy(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), p.size)
        if rc != 0:
            raise ValueError("b200qz_set_policy failed: %d" % rc)

    def policy_features(self, h_ptr, ld, ktop, kbot, lastfrac=0.0) -> np.ndarray:
        out = np.zeros(64, dtype=np.float32)
        rc = lib().b200qz_policy_features(self._h, _vp(h_ptr), ld, ktop, kbot, float(lastfrac),
                                          out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        if rc != 0:
            raise RuntimeError("b200qz_policy_features failed: %d" % rc)
        return out

    def stats(self) -> dict:
        out = np.zeros(len(STAT_NAMES))
        k = lib().b200qz_get_stats(self._h, _p(out), len(STAT_NAMES))
        return dict(zip(STAT_NAMES[:k], out[:k].tolist()))

    def solve_device(self, h_ptr, t_ptr, q_ptr, z_ptr, ld, n, ar_ptr, ai_ptr, be_ptr,
                     job="S", compq="I", compz="I", ilo=1, ihi=None) -> int:
        """Solve on column-major device buffers given as integer pointers
        (e.g. ``tensor.data_ptr()``).  Returns INFO."""
        if ihi is None:
            ihi = n
        return lib().b200qz_solve_dev(self._h, job.encode(), compq.encode(), compz.encode(), n, ilo, ihi,
                                      _vp(h_ptr), _vp(t_ptr), _vp(q_ptr), _vp(z_ptr), ld,
                                      _vp(ar_ptr), _vp(ai_ptr), _vp(be_ptr))

    def solve_host(self, H, T, Q=None, Z=None, job="S", compq="I", compz="I", ilo=1, ihi=None):
        """Host-array solve (copies in and out).  Returns (alphar, alphai, beta, info)."""
        n = H.shape[0]
        if ihi is None:
            ihi = n
        Qa = Q if Q is not None else np.zeros((max(1, n), 1), order="F")
        Za = Z if Z is not None else np.zeros((max(1, n), 1), order="F")
        ar = np.zeros(n)
        ai = np.zeros(n)
        be = np.zeros(n)
        info = lib().b200qz_solve_host(self._h, job.encode(), compq.encode(), compz.encode(), n, ilo, ihi,
                                       _p(H), H.shape[0], _p(T), T.shape[0], _p(Qa), Qa.shape[0], _p(Za),
                                       Za.shape[0], _p(ar), _p(ai), _p(be))
        return ar, ai, be, info


    def ggbal(self, A, B, job="B"):
        """Balance the host pencil (A, B) in place on the GPU (DGGBAL
        semantics).  Returns (ilo, ihi, lscale, rscale, info); ilo/ihi are
        1-based."""
        n = A.shape[0]
        ls = np.zeros(max(1, n))
        rs = np.zeros(max(1, n))
        ilo = ctypes.c_int(0)
        ihi = ctypes.c_int(0)
        info = lib().b200qz_ggbal_host(self._h, job.encode(), n, _vp(A.ctypes.data), max(1, A.shape[0]),
                                       _vp(B.ctypes.data), max(1, B.shape[0]), ctypes.byref(ilo), ctypes.byref(ihi),
                                       _p(ls), _p(rs))
        return ilo.value, ihi.value, ls[:n], rs[:n], info

    def ggbal_device(self, a_ptr, b_ptr, n, ld, job="B"):
        """Balance device arrays (column-major, leading dimension ld) in
        place.  Returns (ilo, ihi, lscale, rscale, info)."""
        ls = np.zeros(max(1, n))
        rs = np.zeros(max(1, n))
        ilo = ctypes.c_int(0)
        ihi = ctypes.c_int(0)
        info = lib().b200qz_ggbal_dev(self._h, job.encode(), n, _vp(a_ptr), ld, _vp(b_ptr), ld, ctypes.byref(ilo),
                                      ctypes.byref(ihi), _p(ls), _p(rs))
        return ilo.value, ihi.value, ls[:n], rs[:n], info

    def tgsen(self, S, T, Q, Z, select, ijob=0, wantq=True, wantz=True, dif=None):
        """Reorder the host generalized Schur form (S, T) and Q, Z in place
        on the GPU so that the selected eigenvalues lead (DTGSEN
        semantics, ijob 0, 1, 3 or 5).  Returns (alphar, alphai, beta, m,
        pl, pr, info, ret) with ret the C return code; for ijob 3 and 5 the
        Difu, Difl estimates go to ``dif`` (a float64 array of 2) when
        given."""
        n = S.shape[0]
        sel = np.ascontiguousarray(np.asarray(select, dtype=np.int32).reshape(-1))
        ar, ai, be = np.zeros(max(1, n)), np.zeros(max(1, n)), np.zeros(max(1, n))
        m, info = ctypes.c_int(0), ctypes.c_int(0)
        pl, pr = ctypes.c_double(0), ctypes.c_double(0)
        d = dif if dif is not None else np.zeros(2)
        Qa = Q if Q is not None else np.zeros((1, 1), order="F")
        Za = Z if Z is not None else np.zeros((1, 1), order="F")
        ret = lib().b200qz_tgsen_host(self._h, ijob, int(wantq), int(wantz),
                                      sel.ctypes.data_as(_pi), n, _vp(S.ctypes.data), max(1, n), _vp(T.ctypes.data),
                                      max(1, n), _vp(Qa.ctypes.data), max(1, Qa.shape[0]), _vp(Za.ctypes.data),
                                      max(1, Za.shape[0]), _p(ar), _p(ai), _p(be), ctypes.byref(m),
                                      ctypes.byref(pl), ctypes.byref(pr), _p(d), ctypes.byref(info))
        return ar[:n], ai[:n], be[:n], m.value, pl.value, pr.value, info.value, ret

    def gghrd(self, A, B, Q=None, Z=None, compq="I", compz="I", ilo=1, ihi=None):
        """Reduce the host pencil (A, B), B upper triangular, to
        Hessenberg-triangular form in place on the GPU (DGGHRD semantics):
        Q^T A Z = H, Q^T B Z = T.  compq/compz 'N', 'I' or 'V' (Q, Z
        updated in place; with 'I' they need not be set).  Returns the C
        return code (0, -i for an illegal argument, 10001)."""
        n = A.shape[0]
        ihi = n if ihi is None else ihi
        dummy = np.zeros((1, 1), order="F")
        Qa = Q if Q is not None else dummy
        Za = Z if Z is not None else dummy
        return lib().b200qz_gghrd_host(self._h, compq.encode(), compz.encode(), n, ilo, ihi, _vp(A.ctypes.data),
                                       max(1, A.shape[0]), _vp(B.ctypes.data), max(1, B.shape[0]),
                                       _vp(Qa.ctypes.data), max(1, Qa.shape[0]), _vp(Za.ctypes.data),
                                       max(1, Za.shape[0]))

    def gghrd_device(self, a_ptr, b_ptr, q_ptr, z_ptr, n, ld, compq="I", compz="I", ilo=1, ihi=None):
        """The same on device arrays (column-major, leading dimension ld)."""
        ihi = n if ihi is None else ihi
        return lib().b200qz_gghrd_dev(self._h, compq.encode(), compz.encode(), n, ilo, ihi, _vp(a_ptr), ld,
                                      _vp(b_ptr), ld, _vp(q_ptr), ld, _vp(z_ptr), ld)

    def ggbak(self, V, ilo, ihi, lscale, rscale, side="R", job="B"):
        """Back-transform the host matrix V (n x m) in place (DGGBAK
        semantics).  Returns info."""
        n = V.shape[0]
        m = V.shape[1] if V.ndim == 2 else 1
        ls = np.ascontiguousarray(lscale, dtype=np.float64)
        rs = np.ascontiguousarray(rscale, dtype=np.float64)
        return lib().b200qz_ggbak_host(self._h, job.encode(), side.encode(), n, ilo, ihi, _p(ls), _p(rs), m,
                                       _vp(V.ctypes.data), max(1, n))


class Batch:
    """Layout of a batch of independent pencils of uneven sizes packed in
    one device buffer: pencil ``p`` (order ``n[p]``, column-major, leading
    dimension ``n[p]``) starts at double offset ``moff[p]``; its eigenvalues
    start at ``eoff[p]``."""

    def __init__(self, sizes):
        self.n = np.ascontiguousarray(sizes, dtype=np.int32)
        sq = self.n.astype(np.int64) ** 2
        self.moff = np.zeros(len(self.n), dtype=np.int64)
        self.eoff = np.zeros(len(self.n), dtype=np.int64)
        if len(self.n):
            self.moff[1:] = np.cumsum(sq)[:-1]
            self.eoff[1:] = np.cumsum(self.n.astype(np.int64))[:-1]
        self.count = len(self.n)
        self.elems = int(sq.sum())
        self.neig = int(self.n.sum())

    def pack(self, mats):
        out = np.empty(self.elems)
        for p, M in enumerate(mats):
            out[self.moff[p]:self.moff[p] + M.size] = np.asarray(M, dtype=np.float64).ravel(order="F")
        return out

    def unpack(self, flat, p):
        n = int(self.n[p])
        return flat[self.moff[p]:self.moff[p] + n * n].reshape((n, n), order="F")


def _batch_args(b: "Batch"):
    _pl = ctypes.POINTER(ctypes.c_longlong)
    return (b.n.ctypes.data_as(_pi), b.moff.ctypes.data_as(_pl), b.eoff.ctypes.data_as(_pl))


def solve_batched_device(solver: "Solver", b: "Batch", h_ptr, t_ptr, q_ptr, z_ptr, ar_ptr, ai_ptr, be_ptr,
                         info_ptr) -> float:
    """Reduce every pencil of the batch to generalized Schur form with Q, Z
    (device buffers given as integer pointers).  Returns device seconds;
    per-pencil INFO goes to ``info_ptr`` (int32, device)."""
    n, mo, eo = _batch_args(b)
    rc = lib().b200qz_solve_batched_dev(solver.handle, b.count, n, mo, eo, _vp(h_ptr), _vp(t_ptr), _vp(q_ptr),
                                        _vp(z_ptr), _vp(ar_ptr), _vp(ai_ptr), _vp(be_ptr), _vp(info_ptr))
    if rc != 0:
        raise RuntimeError("b200qz_solve_batched_dev failed: %d" % rc)
    return lib().b200qz_batched_seconds(solver.handle)


def autotune_batched(solver: "Solver", b: "Batch", h_ptr, t_ptr, sample=256):
    """Pick threads per CTA, shared-memory cutoff and CTAs per SM for this
    batch on a copy of ``sample`` of its pencils.  Returns
    (threads, smem_max, ctas_per_sm, best_seconds)."""
    n, mo, _ = _batch_args(b)
    best = ctypes.c_double(0.0)
    rc = lib().b200qz_batched_autotune(solver.handle, b.count, n, mo, _vp(h_ptr), _vp(t_ptr), sample,
                                       ctypes.byref(best))
    if rc != 0:
        raise RuntimeError("b200qz_batched_autotune failed: %d" % rc)
    th, sm, cps = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lib().b200qz_batched_config(solver.handle, ctypes.byref(th), ctypes.byref(sm), ctypes.byref(cps))
    return th.value, sm.value, cps.value, best.value


def solve(H, T, job="S", compq="I", compz="I", device=0):
    """Convenience: copy, solve on the GPU, return (S, P, Q, Z, alphar, alphai, beta, info)."""
    n = H.shape[0]
    S = np.array(H, dtype=np.float64, order="F", copy=True)
    P = np.array(T, dtype=np.float64, order="F", copy=True)
    Q = np.eye(n, order="F")
    Z = np.eye(n, order="F")
    s = Solver(device)
    try:
        ar, ai, be, info = s.solve_host(S, P, Q, Z, job=job, compq=compq, compz=compz)
    finally:
        s.close()
    return S, P, Q, Z, ar, ai, be, info
