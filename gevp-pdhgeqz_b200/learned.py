"""Learned choice of the AED window size nw and the shift count ns.

The reference takes nw and ns from a fixed table (PIPARMQ / PILAENVX,
``src/pdhgeqz/piparmq.f:438-535``, NS(NH) and NW(NS) with NIBBLE).  Here a
64-128-128-2 FP32 MLP makes that choice at every AED decision from a
profile of the active block's subdiagonal (the features are computed on the
device, ``b200qz_policy_features``); the table stays the fallback.

Training data are traces the method generates itself:

* seeded pencils (n ~ U{2000..8000}, N(0,1), every 50th subdiagonal scaled
  by 1e-8 so that deflation clusters) are run with the table up to a
  decision point (the solver stops before its j-th AED, ``aed_limit``);
* from that state every candidate (nw, ns) of a small grid runs three AEDs
  and the sweeps between them; it is scored by deflations per flop (counted
  off-diagonal update flops plus 10 nw^3 per AED window) and by deflations
  per device second (its solve time minus that of a run that stops before
  the first AED, i.e. without the restart's own cost).  The AED and chase
  kernels are latency-bound on the GPU, so the label uses the per-second
  score, the cost that time-to-Schur actually pays;
* the label is the best candidate, encoded as y0 = (nw - 16) / 64 and
  y1 = ns / nw.

Training runs on the GPU with the library's own forward, backward and Adam
kernels (``b200qz_mlp_train``).  A numpy restatement of the same network
(``forward_np``, ``backward_np``) checks their outputs and gradients.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
POLICY_DIR = os.path.join(HERE, "policy")
WEIGHTS = os.path.join(POLICY_DIR, "weights.npz")
TRACES = os.path.join(POLICY_DIR, "traces.npz")

NIN, NHID, NOUT = 64, 128, 2
NW_MIN, NW_SPAN, NW_MAX = 16, 64, 80
TABLE_NW = 48  # the solver's fixed AED window (SolveParams::nw_max)
GRID_NW = (24, 32, 40, 48, 56, 64, 80)
GRID_NSF = (0.5, 1.0)
DECISIONS = (0, 5, 20, 60, 150)  # AED indices at which a trace samples the choice
AED_FLOP_FACTOR = 10.0  # window QZ + reordering cost per AED, in units of nw^3


def _pkg():
    mod = sys.modules.get("gevp_pdhgeqz_b200")
    if mod is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location("gevp_pdhgeqz_b200", os.path.join(HERE, "__init__.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules["gevp_pdhgeqz_b200"] = mod
        spec.loader.exec_module(mod)
    return mod


# ---------------------------------------------------------------------------
# parameters and the numpy restatement
# ---------------------------------------------------------------------------
def nparams() -> int:
    return NHID * NIN + NHID + NHID * NHID + NHID + NOUT * NHID + NOUT


def unpack(P):
    o = 0
    out = []
    for shape in ((NHID, NIN), (NHID,), (NHID, NHID), (NHID,), (NOUT, NHID), (NOUT,)):
        k = int(np.prod(shape))
        out.append(P[o:o + k].reshape(shape))
        o += k
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases (float32)."""
    rng = np.random.Generator(np.random.Philox(seed))
    parts = []
    for fan_in, shape in ((NIN, (NHID, NIN)), (None, (NHID,)), (NHID, (NHID, NHID)), (None, (NHID,)),
                          (NHID, (NOUT, NHID)), (None, (NOUT,))):
        if fan_in is None:
            parts.append(np.zeros(shape))
        else:
            parts.append(rng.standard_normal(shape) * np.sqrt(2.0 / fan_in))
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)


def forward_np(P, X):
    """Returns (A1, A2, Y) in float64 (reference for the CUDA kernels)."""
    W1, b1, W2, b2, W3, b3 = (np.asarray(a, dtype=np.float64) for a in unpack(np.asarray(P)))
    X = np.asarray(X, dtype=np.float64)
    A1 = np.maximum(X @ W1.T + b1, 0.0)
    A2 = np.maximum(A1 @ W2.T + b2, 0.0)
    Y = A2 @ W3.T + b3
    return A1, A2, Y


def loss_np(P, X, T):
    _, _, Y = forward_np(P, X)
    return float(np.mean((Y - np.asarray(T, dtype=np.float64)) ** 2))


def backward_np(P, X, T):
    """Gradient of mean((Y - T)^2) with respect to the flat parameters."""
    W1, b1, W2, b2, W3, b3 = (np.asarray(a, dtype=np.float64) for a in unpack(np.asarray(P)))
    X = np.asarray(X, dtype=np.float64)
    A1, A2, Y = forward_np(P, X)
    DY = 2.0 * (Y - np.asarray(T, dtype=np.float64)) / Y.size
    D2 = (DY @ W3) * (A2 > 0)
    D1 = (D2 @ W2) * (A1 > 0)
    g = [D1.T @ X, D1.sum(0), D2.T @ A1, D2.sum(0), DY.T @ A2, DY.sum(0)]
    return np.concatenate([a.ravel() for a in g])


def features_np(H, ktop, kbot, lastfrac=0.0):
    """The 64 policy features of the active block [ktop, kbot] of H (numpy
    restatement of the device kernel k_features)."""
    nh = kbot - ktop + 1
    k = np.arange(ktop, kbot)
    hs = np.abs(H[k + 1, k])
    den = np.abs(H[k, k]) + np.abs(H[k + 1, k + 1])
    with np.errstate(divide="ignore", invalid="ignore"):
        r = -np.log10(hs / den)
    x = np.clip(r, 0.0, 16.0) / 16.0
    x = np.where(hs == 0.0, 1.0, np.where(den == 0.0, 0.0, x))
    d = kbot - 1 - k
    b = np.clip((62.0 * np.log1p(d) / np.log(max(nh, 2))).astype(np.int64), 0, 61)
    out = np.zeros(NIN, dtype=np.float64)
    prev = 0.0
    for i in range(62):
        sel = b == i
        v = float(np.mean(x[sel])) if sel.any() else prev
        out[i] = v
        prev = v
    out[62] = np.log2(nh) / 14.0
    out[63] = lastfrac
    return out


def decode(y, nh: int):
    """(nw, ns) from the two outputs, as the solver decodes them."""
    y0 = float(np.clip(y[0], 0.0, 1.0))
    y1 = float(np.clip(y[1], 0.0, 1.0))
    nw = min(int(round(NW_MIN + y0 * NW_SPAN)), NW_MAX)
    ns = int(round(y1 * nw))
    ns = max(2, ns - ns % 2)
    return min(nw, nh), ns


def encode(nw: int, nsf: float):
    return np.array([(nw - NW_MIN) / NW_SPAN, nsf], dtype=np.float32)


def table_choice(nh: int, table_nw: int = TABLE_NW):
    """(nw, ns/nw) the fixed table gives (nw_max and NS(NH), piparmq.f:504-533)."""
    ns = 2
    if nh >= 30:
        ns = 4
    if nh >= 60:
        ns = 10
    if nh >= 150:
        ns = max(10, int(nh / round(np.log(nh) / np.log(2.0))))
    if nh >= 590:
        ns = 64
    if nh >= 3000:
        ns = 128
    ns = max(2, ns - ns % 2)
    nw = min(table_nw, nh)
    return nw, min(1.0, ns / nw)


def nearest_candidate(nw, nsf, grid_nw=GRID_NW, grid_nsf=GRID_NSF):
    i = int(np.argmin([abs(nw - g) for g in grid_nw]))
    j = int(np.argmin([abs(nsf - g) for g in grid_nsf]))
    return i, j


# ---------------------------------------------------------------------------
# device training through the C-ABI
# ---------------------------------------------------------------------------
def train_device(P0, X, T, epochs=3000, lr=1e-3):
    """Full-batch Adam on the GPU with the library's kernels.  Returns
    (params, final mse)."""
    import torch
    L = _pkg().lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    p = torch.from_numpy(np.ascontiguousarray(P0, dtype=np.float32)).to(dev)
    x = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(dev)
    t = torch.from_numpy(np.ascontiguousarray(T, dtype=np.float32)).to(dev)
    torch.cuda.synchronize()
    loss = ctypes.c_float(0.0)
    rc = L.b200qz_mlp_train(ctypes.c_void_p(p.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                            ctypes.c_void_p(t.data_ptr()), x.shape[0], epochs, lr, ctypes.byref(loss))
    if rc != 0:
        raise RuntimeError("b200qz_mlp_train failed: %d" % rc)
    return p.cpu().numpy(), float(loss.value)


def load_weights(path: str = WEIGHTS):
    if not os.path.exists(path):
        return None
    return np.load(path)["params"].astype(np.float32)


# ---------------------------------------------------------------------------
# trace generation (GPU)
# ---------------------------------------------------------------------------
def training_pencils(count: int = 200, seed: int = 300, lo: int = 2000, hi: int = 8000):
    """(index, n, pencil seed) of the training pencils."""
    rng = np.random.Generator(np.random.Philox(seed))
    sizes = rng.integers(lo, hi + 1, size=count)
    return [(i, int(n), 3_000_000 + i) for i, n in enumerate(sizes)]


def _solve(solver, bufs, n):
    dH, dT, dQ, dZ, de = bufs
    return solver.solve_device(dH.data_ptr(), dT.data_ptr(), dQ.data_ptr(), dZ.data_ptr(), n, n, de.data_ptr(),
                               de.data_ptr() + 8 * n, de.data_ptr() + 16 * n)


def _set(solver, nw_max, ns_max, aed_limit):
    """ns_max 0: the table's NS(NH); aed_limit -1: no limit."""
    solver.set_param("nw_max", nw_max)
    solver.set_param("ns_max", ns_max)
    solver.set_param("aed_limit", aed_limit)


def trace_pencil(solver, H, T, decisions=DECISIONS, horizon=3):
    """Samples (features, scores_per_second, scores_per_flop, nh) of one
    pencil at the given AED decision points; scores are arrays
    [len(GRID_NW), len(GRID_NSF)]."""
    import torch
    n = H.shape[0]
    dev = torch.device("cuda", torch.cuda.current_device())
    dH0 = torch.from_numpy(np.ascontiguousarray(H.T)).to(dev)
    dT0 = torch.from_numpy(np.ascontiguousarray(T.T)).to(dev)
    bufs = [torch.empty_like(dH0), torch.empty_like(dT0), torch.empty_like(dH0), torch.empty_like(dH0),
            torch.empty(3 * n, dtype=torch.float64, device=dev)]
    snapH, snapT = torch.empty_like(dH0), torch.empty_like(dT0)
    out = []
    for j in decisions:
        bufs[0].copy_(dH0)
        bufs[1].copy_(dT0)
        _set(solver, TABLE_NW, 0, j)
        info = _solve(solver, bufs, n)
        st = solver.stats()
        if info != 10003:
            break  # converged (or failed) before reaching the decision point
        ktop, kbot = int(st["stop_ktop"]), int(st["stop_kbot"])
        rem0 = int(st["remaining"])
        frac = float(st["last_aed_fraction"])
        snapH.copy_(bufs[0])
        snapT.copy_(bufs[1])
        feat = solver.policy_features(snapH.data_ptr(), n, ktop, kbot, frac)
        # cost of restarting from the snapshot alone (scans down to kbot)
        bufs[0].copy_(snapH)
        bufs[1].copy_(snapT)
        _set(solver, TABLE_NW, 0, 0)
        _solve(solver, bufs, n)
        t0 = solver.stats()["seconds"]
        s_time = np.zeros((len(GRID_NW), len(GRID_NSF)))
        s_flop = np.zeros_like(s_time)
        for a, nw in enumerate(GRID_NW):
            for b, nsf in enumerate(GRID_NSF):
                bufs[0].copy_(snapH)
                bufs[1].copy_(snapT)
                ns = max(2, int(round(nsf * nw)) // 2 * 2)
                _set(solver, nw, ns, horizon)
                info = _solve(solver, bufs, n)
                st = solver.stats()
                if info not in (0, 10003):
                    continue
                defl = rem0 - int(st["remaining"])
                cost = st["update_flops"] + AED_FLOP_FACTOR * st["aeds"] * min(nw, kbot - ktop + 1) ** 3
                s_flop[a, b] = defl / max(cost, 1.0)
                s_time[a, b] = defl / max(st["seconds"] - t0, 1e-6)
        out.append((feat, s_time, s_flop, kbot - ktop + 1))
    _set(solver, TABLE_NW, 0, -1)
    return out


def labels_from_scores(scores, grid_nw=GRID_NW, grid_nsf=GRID_NSF):
    """Best candidate of each sample as the regression target."""
    T = []
    for sc in scores:
        a, b = np.unravel_index(int(np.argmax(sc)), sc.shape)
        T.append(encode(grid_nw[a], grid_nsf[b]))
    return np.stack(T)


def score_of_choice(score, nw, nsf, grid_nw=GRID_NW, grid_nsf=GRID_NSF):
    i, j = nearest_candidate(nw, nsf, grid_nw, grid_nsf)
    return float(score[i, j])


def trace_grid(tr):
    """(grid_nw, grid_nsf, table_nw) a trace file was recorded with (files
    without them predate the current grid)."""
    if "grid_nw" in tr:
        return tuple(int(v) for v in tr["grid_nw"]), tuple(float(v) for v in tr["grid_nsf"]), int(tr["table_nw"])
    return (24, 40, 56, 80), (0.5, 1.0), 80


def offline_gain(P, X, scores, nh, grid=None):
    """Geometric mean over samples of score(network's choice) /
    score(table's choice), both taken at the nearest grid candidate (ratios
    floored at 1e-3 so that a zero score counts as a large loss, not -inf).
    grid: (grid_nw, grid_nsf, table_nw) of the traces (trace_grid)."""
    gnw, gnsf, tnw_fixed = grid if grid is not None else (GRID_NW, GRID_NSF, TABLE_NW)
    _, _, Y = forward_np(P, X)
    logs = []
    for y, sc, h in zip(Y, scores, nh):
        nw, ns = decode(y, int(h))
        tnw, tnsf = table_choice(int(h), tnw_fixed)
        s_net = score_of_choice(sc, nw, ns / max(nw, 1), gnw, gnsf)
        s_tab = score_of_choice(sc, tnw, tnsf, gnw, gnsf)
        if s_tab > 0:
            logs.append(np.log(max(s_net / s_tab, 1e-3)))
    return float(np.exp(np.mean(logs))) if logs else 1.0


def generate_traces(count=200, decisions=DECISIONS, device=0, log=None):
    """Trace all training pencils on the GPU.  Returns dict of arrays."""
    import torch
    pkg = _pkg()
    torch.cuda.set_device(device)
    solver = pkg.Solver(device)
    feats, scores, sflop, nhs, ids = [], [], [], [], []
    try:
        for i, n, seed in training_pencils(count):
            H, T = pkg.pencils.clustered_ht(n, seed, every=50, scale=1e-8)
            for f, st, sf, nh in trace_pencil(solver, H, T, decisions):
                feats.append(f)
                scores.append(st)
                sflop.append(sf)
                nhs.append(nh)
                ids.append(i)
            if log:
                log("pencil %d n=%d samples=%d" % (i, n, len(feats)))
    finally:
        solver.close()
    return {"features": np.stack(feats).astype(np.float32), "scores": np.stack(scores),
            "scores_per_flop": np.stack(sflop), "nh": np.array(nhs), "pencil": np.array(ids),
            "grid_nw": np.array(GRID_NW), "grid_nsf": np.array(GRID_NSF), "table_nw": TABLE_NW,
            "decisions": np.array(decisions)}
