"""Generate tuning traces, train the (nw, ns) MLP on the GPU, evaluate it.

    python gevp-pdhgeqz_b200/train_policy.py traces  --out DIR [--count 200]
    python gevp-pdhgeqz_b200/train_policy.py train   --traces F --out DIR [--epochs 4000]
    python gevp-pdhgeqz_b200/train_policy.py evaluate --weights F [--n 16000]

traces    runs the seeded training pencils (n ~ U{2000..8000}, every 50th
          subdiagonal scaled by 1e-8) and scores every candidate (nw, ns)
          at the decision points (learned.trace_pencil); writes traces.npz
train     trains the MLP with the library's CUDA kernels on the decision
          points of 4 out of every 5 pencils, reports the held-out gain in
          deflations per flop over the fixed table; writes weights.npz
evaluate  solves the seed-3 N(0,1) pencil with the fixed table and with the
          network; prints one JSON line (seconds, sweeps, AEDs, backward
          errors of both)
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _pkg():
    name = "gevp_pdhgeqz_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(HERE, "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


DECISIONS_DEFAULT = (0, 5, 20, 60, 150)


def cmd_traces(a):
    pkg = _pkg()
    t0 = time.time()
    tr = pkg.learned.generate_traces(a.count, tuple(a.decisions), log=lambda m: print(m, flush=True))
    os.makedirs(a.out, exist_ok=True)
    np.savez_compressed(os.path.join(a.out, "traces.npz"), **tr)
    print("samples %d in %.1f s" % (len(tr["nh"]), time.time() - t0), flush=True)


def cmd_train(a):
    pkg = _pkg()
    lrn = pkg.learned
    tr = np.load(a.traces)
    X, scores, nh, pid = tr["features"], tr["scores"], tr["nh"], tr["pencil"]
    grid = lrn.trace_grid(tr)
    T = lrn.labels_from_scores(scores, grid[0], grid[1])
    hold = pid % 5 == 0
    P0 = lrn.init_params(a.seed)
    t0 = time.time()
    P, mse = lrn.train_device(P0, X[~hold], T[~hold], epochs=a.epochs, lr=a.lr)
    dt = time.time() - t0
    res = {"samples_train": int((~hold).sum()), "samples_holdout": int(hold.sum()), "mse_train": mse,
           "label": "argmax deflations per device second",
           "mse_holdout": lrn.loss_np(P, X[hold], T[hold]), "train_seconds": dt,
           "gain_train": lrn.offline_gain(P, X[~hold], scores[~hold], nh[~hold], grid),
           "gain_holdout": lrn.offline_gain(P, X[hold], scores[hold], nh[hold], grid)}
    os.makedirs(a.out, exist_ok=True)
    np.savez_compressed(os.path.join(a.out, "weights.npz"), params=P, epochs=a.epochs, lr=a.lr, seed=a.seed)
    print(json.dumps(res), flush=True)


def _solve_timed(pkg, solver, H, T, n):
    import torch
    dH = torch.from_numpy(np.ascontiguousarray(H.T)).cuda()
    dT = torch.from_numpy(np.ascontiguousarray(T.T)).cuda()
    H0, T0 = dH.clone(), dT.clone()
    dQ, dZ = torch.empty_like(dH), torch.empty_like(dH)
    de = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    info = solver.solve_device(dH.data_ptr(), dT.data_ptr(), dQ.data_ptr(), dZ.data_ptr(), n, n, de.data_ptr(),
                               de.data_ptr() + 8 * n, de.data_ptr() + 16 * n)
    st = solver.stats()
    eps = np.finfo(np.float64).eps
    # device tensors hold the transposes of the column-major matrices:
    # (Q^T H Z - S)^T = Z^T H^T Q - S^T
    res_h = float(torch.linalg.norm(dZ @ H0 @ dQ.T - dH) / torch.linalg.norm(H0)) / (n * eps)
    res_t = float(torch.linalg.norm(dZ @ T0 @ dQ.T - dT) / torch.linalg.norm(T0)) / (n * eps)
    return {"info": info, "seconds": st["seconds"], "sweeps": st["sweeps"], "aeds": st["aeds"],
            "iters": st["iters"], "policy_calls": st["policy_calls"], "backward_error_neps": [res_h, res_t]}


def cmd_evaluate(a):
    import torch
    pkg = _pkg()
    torch.cuda.set_device(0)
    n = a.n
    H, T = pkg.pencils.random_ht(n, 3)
    P = np.load(a.weights)["params"]
    s = pkg.Solver(0)
    try:
        table = _solve_timed(pkg, s, H, T, n)
        s.set_policy(P)
        learned = _solve_timed(pkg, s, H, T, n)
    finally:
        s.close()
    print(json.dumps({"n": n, "pencil": "N(0,1) seed 3", "table": table, "learned": learned,
                      "speedup": table["seconds"] / learned["seconds"]}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    p = sub.add_parser("traces")
    p.add_argument("--out", required=True)
    p.add_argument("--count", type=int, default=200)
    p.add_argument("--decisions", type=int, nargs="+", default=list(DECISIONS_DEFAULT))
    p = sub.add_parser("train")
    p.add_argument("--traces", required=True)
    p.add_argument("--out", required=True)
    p.add_argument("--epochs", type=int, default=300)
    p.add_argument("--lr", type=float, default=1e-3)
    p.add_argument("--seed", type=int, default=0)
    p = sub.add_parser("evaluate")
    p.add_argument("--weights", required=True)
    p.add_argument("--n", type=int, default=16000)
    a = ap.parse_args()
    {"traces": cmd_traces, "train": cmd_train, "evaluate": cmd_evaluate}[a.cmd](a)


if __name__ == "__main__":
    main()
