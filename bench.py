"""Benchmark: time-to-Schur of the multishift QZ path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 10000] [--workload c3] [--mode plain|split|learned|split+learned]
       python bench.py --workload ggbal|tgsen|gghrd   (balancing / reordering / HT reduction,
                                                    LAPACK timed beside)

One step = one complete reduction of a Hessenberg-triangular pencil to
generalized real Schur form with Q and Z (JOB='S', COMPQ=COMPZ='I').
Default workload: the graded n=10000 pencil from seed 2 (H = D1 X_H D2,
T = D1 X_T D2, diag(D1), diag(D2) = 10^U(-3,3)); inputs are 4 x 800 MB,
larger than L2, so no flush is needed between steps.

value      mean device seconds per solve (CUDA events on the solver stream),
           inputs restored from a device-resident copy before each step
           outside the timed events, in --mode (default plain: FP64 DMMA
           updates, (nw, ns) from the fixed table)
forms      the other three forms (split: INT8 Ozaki updates; learned: (nw, ns)
           from the trained MLP; split+learned: both) timed on the same
           pencil, each with its AED and sweep counts and backward errors;
           "comparison" keeps the split+learned speed-up over plain
eigen      the eigenvalues of the timed solve matched as a set against the
           oracle port's solve of the same pencil (tests/golden fixture),
           chordal distance in units of 50 n eps ||(H,T)||_F / s_j
e2e        the same solve through the public C-ABI entry b200qz_solve_host
           with pinned host buffers: H, T copied in, S, P, Q, Z and the
           eigenvalues copied out inside the timed region
roofline   the kernel with the largest device-time share in a profiled
           solve: achieved GB/s from the algorithmic bytes of the windows it
           actually processed; the updates' FP64 TFLOP/s against a cuBLAS
           DGEMM measured in the same process
cpu_baseline
           the oracle's C restatement of the reference path (oracle/qzref.c,
           OpenBLAS on all host threads) run on the same pencil for its first
           AEDs only, scaled by the share of the whole solve those AEDs took
           in the committed full-size profile (bounded to about 20 s)
--impl reference
           the same restatement solving the full pencil, as many whole solves
           as fit the --ref-budget seconds (the true count is reported)

Multi-GPU: a single pencil does not shard; every rank solves its own
replica, value = max over ranks.  Without torchrun, --gpus N > 1 starts N
ranks itself (torch.distributed.run on 127.0.0.1).

--workload c5 (batched): 2048 pencils per GPU (seed 4, n ~ U{32..512}, N(0,1),
2% zero T diagonal) solved in one persistent graph-captured launch after an
autotuning pass; value = pencils/s over all ranks (each rank solves its
size-balanced shard of a global batch of 2048 x N pencils), plus the worst
backward error over the batch.  --check-ranks joins the ranks on gloo and
checks the shard partition without solving (launcher test on CPU hosts).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import socket
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_pkg():
    name = "gevp_pdhgeqz_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "gevp-pdhgeqz_b200", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


METRIC = "time-to-Schur (s) at n=10k, backward err<=50*n*eps; split+learned vs plain FP64 GPU"
EPS = np.finfo(np.float64).eps
GOLDEN = os.path.join(ROOT, "tests", "golden")
FORMS = ("plain", "split", "learned", "split+learned")


def make_pencil(pkg, workload, n):
    P = pkg.pencils
    if workload == "c3":
        return P.graded_ht(n, 2), "graded (D1 X D2, 10^U(-3,3)) seed 2"
    if workload == "c2":
        return P.random_ht(n, 1, 0.05), "N(0,1) seed 1, 5% zero T diagonal"
    if workload == "c1":
        return P.random_ht(n, 0), "N(0,1) seed 0"
    if workload == "c4":
        return P.random_ht(n, 3), "N(0,1) seed 3"
    raise ValueError(workload)


def workload_config(pkg, workload, n, desc):
    """The config block both arms print for a single-pencil workload."""
    return {"workload": "%s: %s n=%d" % (workload, desc, n), "n": n, "job": "S", "compq": "I", "compz": "I",
            "generator": pkg.pencils.GENERATOR}


def port_fixture(workload, n):
    """The oracle port's eigenvalues of this pencil (tests/golden), or None."""
    p = os.path.join(GOLDEN, "port_%s_n%d.npz" % (workload, n))
    if not os.path.exists(p):
        return None
    return dict(np.load(p))


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def fp64_gemm_peak(torch, dev, n=8192, reps=3):
    """FP64 TFLOP/s of a cuBLAS DGEMM (n^3, best of reps) on this GPU: the
    denominator of the updates' roofline (no FP64 figure is in the measured
    peaks)."""
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    c = a @ b
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


# ---------------------------------------------------------------------------
# CPU: the oracle port (reference arm and cpu_baseline)
# ---------------------------------------------------------------------------
def _port():
    from oracle import lapack as L
    from oracle import qzref as R
    threads = os.cpu_count() or 1
    L.set_threads(threads)
    R.lib()
    return R, threads


def port_nb(n):
    return 130 if n > 6000 else 60


def cpu_baseline_sample(pkg, workload, n, budget_s=20.0):
    """The port on the benchmarked pencil itself, stopped after its first K
    AEDs; the seconds are divided by the share of the whole solve those K
    AEDs took in the committed full-size profile (``aed_clock``,
    ``seconds`` of tests/golden/port_<workload>_n<n>.npz).  K is the largest
    count whose profiled share stays within budget_s of the profiled solve.
    Returns the baseline dict, or None without a profile."""
    fx = port_fixture(workload, n)
    if fx is None or "aed_clock" not in fx:
        return None
    clock, total = np.asarray(fx["aed_clock"]), float(fx["seconds"])
    scale = float(fx["threads"]) / float(os.cpu_count() or 1)
    k = int(np.searchsorted(clock, budget_s / max(scale, 1e-3), side="right"))
    k = max(1, min(k, len(clock) - 1))
    frac = float(clock[k]) / total
    R, threads = _port()
    (H, T), desc = make_pencil(pkg, workload, n)
    t0 = time.perf_counter()
    out = R.pdhgeqz(H, T, nb=port_nb(n), aed_limit=k)
    dt = time.perf_counter() - t0
    if out[7] != -2:
        raise RuntimeError("bounded port run did not stop at its AED limit (info=%d)" % out[7])
    return {"value": dt / frac, "unit": "s", "cores": threads, "kind": "port",
            "sample": "oracle/qzref.c (OpenBLAS, %d threads) on this %s pencil for its first %d AEDs: %.2f s, "
                      "divided by the %.3f share of the whole solve those AEDs took in the full-size profile "
                      "(%s, %.1f s on %d threads)" % (threads, desc, k, dt, frac,
                                                      "tests/golden/port_%s_n%d.npz" % (workload, n), total,
                                                      int(fx["threads"]))}


def run_reference(args, pkg, rank):
    """Whole solves of the benchmarked pencil by the oracle port, as many as
    fit the budget (at least one)."""
    if rank != 0:
        return
    R, threads = _port()
    (H, T), desc = make_pencil(pkg, args.workload, args.n)
    # warm-up: one small solve (OpenBLAS thread pool, page-in of the library)
    Hs, Ts = pkg.pencils.random_ht(300, 0)
    R.pdhgeqz(Hs, Ts, nb=60)
    times = []
    t_all = time.perf_counter()
    while len(times) < max(1, args.steps):
        t0 = time.perf_counter()
        out = R.pdhgeqz(H, T, nb=port_nb(args.n))
        dt = time.perf_counter() - t0
        if out[7] != 0:
            raise RuntimeError("oracle port did not converge (info=%d)" % out[7])
        times.append(dt)
        if time.perf_counter() - t_all + dt > args.ref_budget:
            break
    v = float(np.mean(times))
    sample = ("oracle/qzref.c (C restatement of PDHGEQZ on a 1x1 grid, PDHGEQZ0 regime above n=6000, OpenBLAS "
              "%d threads): %d whole solve(s) of the %s pencil at n=%d; warm-up: one n=300 solve" %
              (threads, len(times), desc, args.n))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus,
            "steps": len(times), "warmup": 1, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(pkg, args.workload, args.n, desc),
            "steps_note": "whole solves within --ref-budget %.0f s (requested %d)" % (args.ref_budget, args.steps),
            "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def configure(pkg, solver, mode):
    """Set the solver up for a form: 'split' routes the off-diagonal updates
    through 8 INT8 Ozaki slices on the tensor cores, 'learned' loads the
    trained (nw, ns) network (policy/weights.npz).  Returns a note."""
    solver.set_param("split", 8 if "split" in mode else 0)
    note = "split: 8 INT8 slices" if "split" in mode else "updates: FP64 DMMA"
    if "learned" in mode:
        P = pkg.learned.load_weights()
        if P is None:
            raise RuntimeError("mode %s needs gevp-pdhgeqz_b200/policy/weights.npz" % mode)
        solver.set_policy(P)
        note += "; (nw, ns): learned MLP"
    else:
        solver.set_policy(None)
        note += "; (nw, ns): fixed table"
    return note


def errors(torch, dH0, dT0, dH, dT, dQ, dZ, n, dev):
    """Backward errors and orthogonality (units of n*eps), FP64 on the GPU;
    the tensors hold the transposes of the column-major matrices."""
    Ht, Tt, S, P, Q, Z = dH0.t(), dT0.t(), dH.t(), dT.t(), dQ.t(), dZ.t()
    res_h = (torch.linalg.norm(Q.T @ Ht @ Z - S).item() / torch.linalg.norm(Ht).item()) / (n * EPS)
    res_t = (torch.linalg.norm(Q.T @ Tt @ Z - P).item() / torch.linalg.norm(Tt).item()) / (n * EPS)
    I = torch.eye(n, dtype=torch.float64, device=dev)
    orth_q = torch.linalg.norm(Q.T @ Q - I).item() / (n * EPS)
    orth_z = torch.linalg.norm(Z.T @ Z - I).item() / (n * EPS)
    return res_h, res_t, orth_q, orth_z


def eigen_match(fx, de, n):
    """Chordal match of the solve's eigenvalues against the port's, in units
    of 50 n eps ||(H,T)||_F / s_j (s_j: DTGSNA reciprocal condition numbers
    in the port's Schur form).  <= 1 everywhere is a match."""
    from oracle import lapack as L
    e = de.cpu().numpy()
    ar, ai, be = e[:n], e[n:2 * n], e[2 * n:]
    tol = np.clip(50.0 * n * EPS * float(fx["norm"]) / np.maximum(fx["rcond"], 1e-300), 50.0 * n * EPS, 2.0)
    ok, ratio, _ = L.match_eigenvalues((fx["alphar"], fx["alphai"], fx["beta"]), (ar, ai, be), tol)
    return {"against": "oracle port (oracle/qzref.c) solve of the same pencil", "max_ratio": ratio, "match": ok,
            "infinite": int(np.sum(be == 0.0)), "infinite_port": int(np.sum(fx["beta"] == 0.0))}


def roofline_of(pst, phases, peaks, peak_kind, fp64_peak, split):
    """Roofline of the dominant kernel of a profiled solve, plus the update
    kernels' FP64 rate.  Window kernels: achieved = algorithmic bytes of the
    windows they processed (6*8*w^2 per window of order w) / their device
    time; launches = windows launched (AED and endgame windows; chase waves)."""
    dom = max(phases, key=phases.get)
    upd_ms = phases.get("aed_update", 0.0) + phases.get("chase_update", 0.0)
    upd = {"kernel": "k_ozaki_update (INT8 tcgen05, 8 slices)" if split else "k_update_persist (DMMA FP64)",
           "fp64_equivalent_flops": pst["update_flops"], "ms": upd_ms,
           "achieved_tflops": pst["update_flops"] / max(upd_ms * 1e-3, 1e-12) / 1e12,
           "peak_tflops": fp64_peak, "peak_source": "cuBLAS DGEMM 8192^3 measured in this process",
           "frac": pst["update_flops"] / max(upd_ms * 1e-3, 1e-12) / 1e12 / fp64_peak}
    win = {"aed": ("k_aed_win", pst["aed_bytes"], pst["aed_launches"]),
           "chase": ("k_chase_win", pst["chase_bytes"], pst["chase_launches"])}
    if dom in win:
        kname, byts, launches = win[dom]
        dur = phases[dom] * 1e-3 / max(1.0, launches)
        ach = byts / max(launches, 1.0) / dur / 1e9
        roof = {"kernel": kname, "bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": ach / peaks["hbm_gbs"], "traffic": None, "launches": int(launches),
                "avg_launch_ms": dur * 1e3, "bytes_per_launch": byts / max(launches, 1.0),
                "peak_source": "%s HBM copy bandwidth (of %s)" % (peak_kind, peak_kind),
                "traffic_note": "ncu DRAM bytes per launch: profiles/ncu_%s_c1_n2000.md" % kname}
    elif dom in ("aed_update", "chase_update"):
        roof = {"kernel": upd["kernel"], "bound": "tensor", "achieved": upd["achieved_tflops"],
                "peak": fp64_peak, "unit": "TFLOP/s", "frac": upd["frac"], "traffic": None,
                "peak_source": upd["peak_source"]}
    else:
        roof = {"kernel": dom, "bound": "hbm", "achieved": None, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": None, "traffic": None}
    roof["updates"] = upd
    return roof


def maybe_launch_ranks(args):
    """python bench.py --gpus N (N > 1) outside torchrun: start N ranks with
    torch.distributed.run on 127.0.0.1 and exit with their status."""
    if args.gpus <= 1 or "WORLD_SIZE" in os.environ:
        return
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=%d" % args.gpus,
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    sys.exit(subprocess.call(cmd))


def init_dist(torch, world, local, backend="nccl"):
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return dist


C5_METRIC = ("batched pencils/s: 2048 pencils per GPU, n~U{32..512}, seed 4, 2% zero T diagonal, "
             "one persistent graph-captured launch; worst backward error reported")


def c5_cpu_pencils_per_s(pkg, sizes_all, idx, sample_every):
    """The oracle port (oracle/qzref.c) on every sample_every-th pencil of
    the shard, one pencil per host thread.  Returns (pencils/s, threads,
    sample count, seconds)."""
    import concurrent.futures as cf
    from oracle import lapack as L
    from oracle import qzref as R
    L.set_threads(1)
    R.lib()
    threads = os.cpu_count() or 1
    pick = idx[::sample_every]
    mats = [pkg.pencils.batched_pencil(i, int(sizes_all[i])) for i in pick]

    def one(m):
        out = R.pdhgeqz(m[0], m[1], nb=60)
        if out[7] != 0:
            raise RuntimeError("oracle port did not converge (info=%d)" % out[7])

    with cf.ThreadPoolExecutor(threads) as ex:
        list(ex.map(one, mats[:threads]))  # warm-up
        t0 = time.perf_counter()
        list(ex.map(one, mats))
        dt = time.perf_counter() - t0
    return len(mats) / dt, threads, len(mats), dt


def check_ranks(args, pkg, rank, world):
    """Join the ranks on gloo, take this rank's shard of the batch and
    gather every rank's shard on rank 0, which checks that the shards
    partition the batch.  No solve (a launcher test for CPU-only hosts)."""
    import torch
    dist = init_dist(torch, world, 0, backend="gloo")
    sizes_all = pkg.pencils.batch_sizes(args.batch * world, 4)
    mine = pkg.shard.shard(sizes_all, rank, world)
    parts = [mine]
    if dist is not None:
        parts = [None] * world
        dist.all_gather_object(parts, mine)
    if rank == 0:
        flat = sorted(i for p in parts for i in p)
        print(json.dumps({"check_ranks": True, "n_ranks": world, "pencils": len(sizes_all),
                          "partition_ok": flat == list(range(len(sizes_all))),
                          "per_rank": [len(p) for p in parts]}), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_batched(args, pkg, rank, world, local):
    per_rank = args.batch
    sizes_all = pkg.pencils.batch_sizes(per_rank * world, 4)
    idx = pkg.shard.shard(sizes_all, rank, world)
    wl = "c5: %d pencils per GPU (global %d), seed 4, n~U{32..512}, 2%% zero T diagonal" % (per_rank,
                                                                                         per_rank * world)
    config = {"workload": wl, "job": "S", "compq": "I", "compz": "I", "generator": pkg.pencils.GENERATOR}
    if args.impl == "reference":
        if rank != 0:
            return
        vals = []
        for _ in range(max(1, args.steps)):
            v, threads, cnt, dt = c5_cpu_pencils_per_s(pkg, sizes_all, idx, 4)
            vals.append(v)
        v = float(np.mean(vals))
        sample = ("oracle/qzref.c (C restatement of PDHGEQZ, the KKQZ/DHGEQZ regime below n=201) on every "
                  "4th pencil of the batch (%d pencils, %.2f s), one pencil per host thread" % (cnt, dt))
        line = {"impl": "reference", "metric": C5_METRIC, "value": v, "unit": "pencils/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * per_rank / v,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": v, "unit": "pencils/s", "cores": threads, "kind": "port",
                                 "sample": sample},
                "e2e": {"value": v, "unit": "pencils/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    dist = init_dist(torch, world, local)
    if dist is None:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    sizes = [int(sizes_all[i]) for i in idx]
    b = pkg.Batch(sizes)
    hH = np.empty(b.elems)
    hT = np.empty(b.elems)
    for k, i in enumerate(idx):
        Hm, Tm = pkg.pencils.batched_pencil(i, sizes[k])
        o = int(b.moff[k])
        hH[o:o + Hm.size] = Hm.ravel(order="F")
        hT[o:o + Tm.size] = Tm.ravel(order="F")
    dH0 = torch.from_numpy(hH).to(dev)
    dT0 = torch.from_numpy(hT).to(dev)
    dH, dT = torch.empty_like(dH0), torch.empty_like(dT0)
    dQ, dZ = torch.empty_like(dH0), torch.empty_like(dH0)
    de = torch.empty(3 * b.neig, dtype=torch.float64, device=dev)
    dinfo = torch.empty(b.count, dtype=torch.int32, device=dev)
    solver = pkg.Solver(dev)
    th, smx, cps, best = pkg.autotune_batched(solver, b, dH0.data_ptr(), dT0.data_ptr(), sample=256)
    ptrs = (dH.data_ptr(), dT.data_ptr(), dQ.data_ptr(), dZ.data_ptr(), de.data_ptr(), de.data_ptr() + 8 * b.neig,
            de.data_ptr() + 16 * b.neig, dinfo.data_ptr())

    def one_step():
        dH.copy_(dH0)
        dT.copy_(dT0)
        torch.cuda.synchronize()
        return pkg.solve_batched_device(solver, b, *ptrs)

    for _ in range(args.warmup):
        one_step()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    times = [one_step() for _ in range(args.steps)]
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist is not None:
        dist.barrier()
    t_mean = float(np.mean(times))
    if int((dinfo != 0).sum().item()) != 0:
        raise RuntimeError("batched solve: %d pencils did not converge" % int((dinfo != 0).sum().item()))

    # worst backward error / orthogonality over the batch (FP64 on the GPU)
    worst = {"h": 0.0, "t": 0.0, "q": 0.0, "z": 0.0}
    for k, n in enumerate(sizes):
        o = int(b.moff[k])
        v = lambda x: x[o:o + n * n].view(n, n).t()
        H0, T0, S, P, Q, Z = v(dH0), v(dT0), v(dH), v(dT), v(dQ), v(dZ)
        I = torch.eye(n, dtype=torch.float64, device=dev)
        nh = max(float(torch.linalg.norm(H0)), 1e-300)
        nt = max(float(torch.linalg.norm(T0)), 1e-300)
        worst["h"] = max(worst["h"], float(torch.linalg.norm(Q.T @ H0 @ Z - S)) / nh / (n * EPS))
        worst["t"] = max(worst["t"], float(torch.linalg.norm(Q.T @ T0 @ Z - P)) / nt / (n * EPS))
        worst["q"] = max(worst["q"], float(torch.linalg.norm(Q.T @ Q - I)) / (n * EPS))
        worst["z"] = max(worst["z"], float(torch.linalg.norm(Z.T @ Z - I)) / (n * EPS))

    # end to end: pinned host inputs in, Schur forms, factors and eigenvalues out
    pin = lambda m: torch.empty(m, dtype=torch.float64, pin_memory=True)
    pH, pT = pin(b.elems), pin(b.elems)
    pH.copy_(torch.from_numpy(hH))
    pT.copy_(torch.from_numpy(hT))
    oS, oP, oQ, oZ, oE = pin(b.elems), pin(b.elems), pin(b.elems), pin(b.elems), pin(3 * b.neig)
    oI = torch.empty(b.count, dtype=torch.int32, pin_memory=True)
    e2e_times = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dH.copy_(pH, non_blocking=True)
        dT.copy_(pT, non_blocking=True)
        torch.cuda.synchronize()
        pkg.solve_batched_device(solver, b, *ptrs)
        for dst, src in ((oS, dH), (oP, dT), (oQ, dQ), (oZ, dZ), (oE, de), (oI, dinfo)):
            dst.copy_(src, non_blocking=True)
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
    e2e = float(np.mean(e2e_times))
    if dist is not None:
        tt = torch.tensor([t_mean, e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_mean, e2e = float(tt[0]), float(tt[1])
        wv = torch.tensor([worst[k] for k in "htqz"], dtype=torch.float64, device=dev)
        dist.all_reduce(wv, op=dist.ReduceOp.MAX)
        worst = dict(zip("htqz", wv.tolist()))
    total = per_rank * world

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, threads, cnt, dt = c5_cpu_pencils_per_s(pkg, sizes_all, idx, 4)
        cpu = {"value": v, "unit": "pencils/s", "cores": threads, "kind": "port",
               "sample": "oracle/qzref.c on every 4th pencil of the batch (%d pencils, %.2f s), one pencil "
                         "per host thread" % (cnt, dt)}
    if rank == 0:
        alg_bytes = 6.0 * 8.0 * b.elems  # H, T in; H, T, Q, Z out
        peaks, peak_kind = read_peaks()
        ach = alg_bytes / t_mean / 1e9
        config.update({
            "parallelism": "size-balanced shards, no collective" if world > 1 else "single-gpu",
            "l2": "inputs 2 x %.0f MB per GPU > L2; restored from device copy outside timed events"
                  % (8 * b.elems / 1e6),
            "autotuned": {"threads": th, "smem_max": smx, "ctas_per_sm": cps, "sample_seconds": best},
            "worst_backward_error_neps": {"h": worst["h"], "t": worst["t"]},
            "worst_orthogonality_neps": {"q": worst["q"], "z": worst["z"]}})
        line = {
            "metric": C5_METRIC, "value": total / t_mean, "unit": "pencils/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_mean * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
            "e2e": {"value": total / e2e, "unit": "pencils/s", "h2d_bytes_per_step": 2 * 8 * b.elems,
                    "d2h_bytes_per_step": 4 * 8 * b.elems + 8 * 3 * b.neig + 4 * b.count},
            "gpu_launches": args.steps,
            "clocks": clk,
            "roofline": {"kernel": "k_batch_qz", "bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": ach / peaks["hbm_gbs"], "traffic": None,
                         "bytes_per_launch": alg_bytes,
                         "peak_source": "%s HBM copy bandwidth (of %s)" % (peak_kind, peak_kind)},
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if dist is not None:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# The steps either side of the solve: balancing (DGGBAL semantics) and
# reordering of the Schur form (DTGSEN semantics), each timed on the GPU
# with LAPACK's routine timed beside it on the same input.
# ---------------------------------------------------------------------------
def post_pencil(n, seed, k1, k2, decades):
    """Dense pencil with k1 + k2 eigenvalues that permutations isolate
    (block triangular under hidden row/column permutations) and rows and
    columns graded over ``decades`` decades."""
    rng = np.random.default_rng(seed)

    def one():
        M = rng.standard_normal((n, n))
        M[k1:, :k1] = 0.0
        M[n - k2:, :n - k2] = 0.0
        M[:k1, :k1] = np.triu(M[:k1, :k1])
        M[n - k2:, n - k2:] = np.triu(M[n - k2:, n - k2:])
        return M

    A, B = one(), one()
    pr, pc = rng.permutation(n), rng.permutation(n)
    d = np.logspace(-decades / 2, decades / 2, n)
    return np.asfortranarray(A[pr][:, pc] * d[:, None]), np.asfortranarray(B[pr][:, pc] * d[None, ::-1])


def run_post(args, pkg):
    import time
    import torch
    from oracle import lapack as L
    torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    solver = pkg.Solver(dev)
    peaks, peak_kind = read_peaks()
    clocks = ClockSampler(dev)
    if args.workload == "ggbal":
        n = args.n
        A, B = post_pencil(n, 5, 64, 64, 8)
        dA0 = torch.from_numpy(np.ascontiguousarray(A.T)).to(dev)
        dB0 = torch.from_numpy(np.ascontiguousarray(B.T)).to(dev)
        dA, dB = torch.empty_like(dA0), torch.empty_like(dB0)

        def step():
            dA.copy_(dA0)
            dB.copy_(dB0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ilo, ihi, ls, rs, info = solver.ggbal_device(dA.data_ptr(), dB.data_ptr(), n, n, "B")
            t = time.perf_counter() - t0
            if info != 0:
                raise RuntimeError("ggbal returned %d" % info)
            return t, (ilo, ihi, ls, rs)

        for _ in range(args.warmup):
            step()
        clocks.start()
        ts = [step() for _ in range(args.steps)]
        clk = clocks.stop()
        t = float(np.mean([x[0] for x in ts]))
        ilo, ihi, ls, rs = ts[-1][1]
        # end to end: host arrays in, balanced host arrays out
        te = []
        for _ in range(args.steps):
            Ah, Bh = np.array(A, order="F"), np.array(B, order="F")
            t0 = time.perf_counter()
            solver.ggbal(Ah, Bh, "B")
            te.append(time.perf_counter() - t0)
        cpu = None
        if not args.no_cpu_baseline:
            t0 = time.perf_counter()
            La, Lb, lilo, lihi, lls, lrs, _ = L.dggbal(A, B, "B")
            cpu_t = time.perf_counter() - t0
            same = (lilo, lihi) == (ilo, ihi) and np.array_equal(lls, ls) and np.array_equal(lrs, rs)
            cpu = {"value": cpu_t, "unit": "s", "cores": 1, "kind": "reference",
                   "sample": "LAPACK DGGBAL (scipy's OpenBLAS) on the same pencil, one call",
                   "identical_output": bool(same)}
        nr = ihi - ilo + 1
        # algorithmic bytes: counts (read A, B), logs (two reads of the
        # active block), maxima (read), apply (read + write), nonzero byte
        # matrix and its reads by the CG iterations (at most nr + 2)
        alg = 16.0 * n * n * 4 + 32.0 * nr * nr + 1.0 * nr * nr
        peak = peaks.get("hbm_gbs")
        ach = alg / t / 1e9
        line = {"metric": "balance_seconds", "value": t, "unit": "s", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "ggbal: DGGBAL job B, n=%d, 128 isolatable eigenvalues under hidden "
                                       "permutations, rows/columns graded over 8 decades (seed 5)" % n,
                           "n": n, "ilo": ilo, "ihi": ihi, "inputs": "device-resident copies, 2 x %.2f GB" %
                           (8e-9 * n * n)},
                "e2e": {"value": float(np.mean(te)), "unit": "s", "h2d_bytes_per_step": 16 * n * n,
                        "d2h_bytes_per_step": 16 * n * n},
                "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                             "frac": (ach / peak) if peak else None, "traffic": None,
                             "peak_source": "%s HBM copy bandwidth" % peak_kind,
                             "note": "whole call (host isolation/CG control included) against the copy "
                                     "bandwidth; algorithmic bytes %.3g" % alg},
                "cpu_baseline": cpu, "clocks": clk, "gpu_launches": None}
        print(json.dumps(line), flush=True)
        solver.close()
        return
    if args.workload == "gghrd":
        run_gghrd(args, pkg, solver, peaks, peak_kind, clocks)
        solver.close()
        return
    # tgsen: reorder the GPU's Schur form of a random pencil so that the
    # eigenvalues of modulus below the median lead (n = 2000 unless --n
    # is given: LAPACK's DTGSEN beside it takes minutes above that)
    n = args.n if args.n != 10000 else 2000
    H, T = pkg.pencils.random_ht(n, 6, 0.0)
    S, P, Q, Z, ar, ai, be, info = pkg.solve(H, T)
    if info != 0:
        raise RuntimeError("solve returned %d" % info)
    lam = np.abs(ar + 1j * ai) / np.maximum(np.abs(be), 1e-300)
    sel = (lam < np.median(lam)).astype(np.int32)
    d0 = [torch.from_numpy(np.ascontiguousarray(M.T)).to(dev) for M in (S, P, Q, Z)]
    dw = [torch.empty_like(x) for x in d0]
    de = torch.empty(3 * n, dtype=torch.float64, device=dev)
    lib = pkg.lib()

    def step():
        for a, b in zip(dw, d0):
            a.copy_(b)
        torch.cuda.synchronize()
        m, inf = pkg.ctypes.c_int(0), pkg.ctypes.c_int(0)
        pl, pr = pkg.ctypes.c_double(0), pkg.ctypes.c_double(0)
        cnt = np.zeros(2, dtype=np.int32)
        t0 = time.perf_counter()
        rc = lib.b200qz_tgsen_dev(solver.handle, 0, 1, 1, sel.ctypes.data_as(pkg._pi), n,
                                  pkg._vp(dw[0].data_ptr()), n, pkg._vp(dw[1].data_ptr()), n,
                                  pkg._vp(dw[2].data_ptr()), n, pkg._vp(dw[3].data_ptr()), n,
                                  pkg._vp(de.data_ptr()), pkg._vp(de.data_ptr() + 8 * n),
                                  pkg._vp(de.data_ptr() + 16 * n), pkg.ctypes.byref(m), pkg.ctypes.byref(pl),
                                  pkg.ctypes.byref(pr), None, pkg.ctypes.byref(inf), cnt.ctypes.data_as(pkg._pi))
        t = time.perf_counter() - t0
        if rc != 0 or inf.value != 0:
            raise RuntimeError("tgsen returned %d / info %d" % (rc, inf.value))
        return t, m.value, cnt

    for _ in range(args.warmup):
        step()
    clocks.start()
    ts = [step() for _ in range(args.steps)]
    clk = clocks.stop()
    t = float(np.mean([x[0] for x in ts]))
    m, cnt = ts[-1][1], ts[-1][2]
    te = []
    for _ in range(args.steps):
        Sh, Ph, Qh, Zh = (np.array(M, order="F") for M in (S, P, Q, Z))
        t0 = time.perf_counter()
        solver.tgsen(Sh, Ph, Qh, Zh, sel, ijob=0)
        te.append(time.perf_counter() - t0)
    cpu = None
    if not args.no_cpu_baseline:
        t0 = time.perf_counter()
        out = L.dtgsen(S, P, Q, Z, sel, ijob=0)
        cpu_t = time.perf_counter() - t0
        cpu = {"value": cpu_t, "unit": "s", "cores": 1, "kind": "reference",
               "sample": "LAPACK DTGSEN (IJOB 0, scipy's OpenBLAS) on the same Schur form, one call",
               "m": int(out[7])}
    # the windows' factor updates: each window of k rows updates k rows of
    # S, T to its right, k columns of S, T above it and k columns of Q, Z
    # (read + write, 16 bytes per element); at most 80 rows per window
    upd_bytes = 16.0 * int(cnt[1]) * 80 * (2 * n + 2 * n)
    peak = peaks.get("hbm_gbs")
    line = {"metric": "reorder_seconds", "value": t, "unit": "s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "tgsen: DTGSEN IJOB 0, Schur form of random_ht(n=%d, seed 6), eigenvalues "
                                   "of modulus below the median selected" % n, "n": n, "m": m,
                       "swaps": int(cnt[0]), "windows": int(cnt[1])},
            "e2e": {"value": float(np.mean(te)), "unit": "s", "h2d_bytes_per_step": 32 * n * n,
                    "d2h_bytes_per_step": 32 * n * n + 24 * n},
            "roofline": {"bound": "hbm", "achieved": upd_bytes / t / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": (upd_bytes / t / 1e9 / peak) if peak else None, "traffic": None,
                         "peak_source": "%s HBM copy bandwidth" % peak_kind,
                         "note": "factor-update bytes of the windows over the whole call; the swap chains "
                                 "inside each window are latency-bound on one CTA"},
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": 3 * int(cnt[1]) + 2}
    print(json.dumps(line), flush=True)
    solver.close()


def run_gghrd(args, pkg, solver, peaks, peak_kind, clocks):
    """Hessenberg-triangular reduction of a dense A with upper triangular B
    (n = 2000 unless --n is given; the reference's own example pair is of
    order 4800): device time, end-to-end time through the host entry, and
    LAPACK DGGHD3 (the blocked reduction) on one host core beside it."""
    import time
    import torch
    from oracle import lapack as L
    n = args.n if args.n != 10000 else 2000
    dev = torch.cuda.current_device()
    rng = np.random.default_rng(7)
    A = rng.standard_normal((n, n))
    B = np.triu(rng.standard_normal((n, n)))
    dA0 = torch.from_numpy(np.ascontiguousarray(A.T)).to(dev)
    dB0 = torch.from_numpy(np.ascontiguousarray(B.T)).to(dev)
    dA, dB = torch.empty_like(dA0), torch.empty_like(dB0)
    dQ, dZ = torch.empty_like(dA0), torch.empty_like(dA0)
    win = 128
    for p in args.param:
        k, v = p.split("=")
        if k == "hr_win":
            win = int(float(v))
            solver.set_param("hr_win", win)

    def step():
        dA.copy_(dA0)
        dB.copy_(dB0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rc = solver.gghrd_device(dA.data_ptr(), dB.data_ptr(), dQ.data_ptr(), dZ.data_ptr(), n, n)
        e1.record()
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError("gghrd returned %d" % rc)
        return e0.elapsed_time(e1) / 1e3

    for _ in range(args.warmup):
        step()
    clocks.start()
    ts = [step() for _ in range(args.steps)]
    clk = clocks.stop()
    t = float(np.mean(ts))
    # backward errors of the last reduction (FP64 products on the GPU)
    Hm, Tm, Qm, Zm, A0m, B0m = dA.T, dB.T, dQ.T, dZ.T, dA0.T, dB0.T
    eps = np.finfo(np.float64).eps
    res = {"a": float(torch.linalg.norm(Qm @ Hm @ Zm.T - A0m) / torch.linalg.norm(A0m)) / (n * eps),
           "b": float(torch.linalg.norm(Qm @ Tm @ Zm.T - B0m) / torch.linalg.norm(B0m)) / (n * eps)}
    # end to end: host arrays in, the reduced pencil and Q, Z out
    te = []
    for _ in range(args.steps):
        Ah, Bh = np.array(A, order="F"), np.array(B, order="F")
        Qh, Zh = np.empty((n, n), order="F"), np.empty((n, n), order="F")
        t0 = time.perf_counter()
        if solver.gghrd(Ah, Bh, Qh, Zh) != 0:
            raise RuntimeError("gghrd (host) failed")
        te.append(time.perf_counter() - t0)
    cpu = None
    if not args.no_cpu_baseline:
        L.set_threads(1)
        t0 = time.perf_counter()
        _, _, _, _, linfo = L.dgghd3(A, B)
        cpu_t = time.perf_counter() - t0
        cpu = {"value": cpu_t, "unit": "s", "cores": 1, "kind": "reference",
               "sample": "LAPACK DGGHD3 (blocked Hessenberg-triangular reduction, scipy's OpenBLAS, one "
                         "thread) on the same pencil, one call", "info": int(linfo)}
    pairs = (n - 1) * (n - 2) // 2
    windows = sum(-(-(n - 2 - jc) // win) for jc in range(n - 2))
    # algorithmic bytes of the rotation walks: per column jc every touched
    # entry of A, B, Q, Z is read and written once (about
    # 2 (n-jc)^2 + 3 n (n-jc) entries, 16 bytes each)
    alg = 16.0 * sum(2.0 * (n - jc) ** 2 + 3.0 * n * (n - jc) for jc in range(n - 2))
    peak = peaks.get("hbm_gbs")
    ach = alg / t / 1e9
    line = {"metric": "ht_reduction_seconds", "value": t, "unit": "s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "gghrd: DGGHRD COMPQ=COMPZ=I, A dense N(0,1), B upper triangular N(0,1), "
                                   "n=%d (seed 7)" % n, "n": n, "pairs": pairs, "windows": windows,
                       "hr_win": win, "backward_error_n_eps": res,
                       "inputs": "device-resident copies, 2 x %.2f GB" % (8e-9 * n * n)},
            "e2e": {"value": float(np.mean(te)), "unit": "s", "h2d_bytes_per_step": 16 * n * n,
                    "d2h_bytes_per_step": 32 * n * n},
            "roofline": {"bound": "latency", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": (ach / peak) if peak else None, "traffic": None,
                         "peak_source": "%s HBM copy bandwidth" % peak_kind,
                         "note": "the walks' algorithmic bytes over the whole call; the bound is the chain "
                                 "of %d dependent rotation pairs on one SM (FP64 latency)" % pairs},
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": windows + 2 * (n - 2) + 4}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=10000)
    ap.add_argument("--workload", default="c3")
    ap.add_argument("--ref-budget", type=float, default=900.0,
                    help="seconds of whole reference solves (--impl reference)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--param", action="append", default=[], help="solver tunable name=value")
    ap.add_argument("--batch", type=int, default=2048, help="pencils per GPU for --workload c5")
    ap.add_argument("--mode", default="plain", choices=list(FORMS), help="form of the timed solves")
    ap.add_argument("--form-steps", type=int, default=2, help="timed solves of each other form (0: skip them)")
    ap.add_argument("--check-ranks", action="store_true", help="join the ranks and check the c5 shards only")
    args = ap.parse_args()
    maybe_launch_ranks(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pkg = load_pkg()

    if args.check_ranks:
        check_ranks(args, pkg, rank, world)
        return
    if args.workload == "c5":
        run_batched(args, pkg, rank, world, local)
        return
    if args.workload in ("ggbal", "tgsen", "gghrd"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the ggbal/tgsen/gghrd workloads time LAPACK "
                              "beside the GPU call in their own line (cpu_baseline)"}))
        elif rank == 0:
            run_post(args, pkg)
        return
    if args.impl == "reference":
        run_reference(args, pkg, rank)
        return

    import torch
    dist = init_dist(torch, world, local)
    if dist is None:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    n = args.n
    (H, T), desc = make_pencil(pkg, args.workload, n)
    ld = n
    # device-resident pristine copies (column-major storage = transposed torch tensors)
    dH0 = torch.from_numpy(np.ascontiguousarray(H.T)).to(dev)
    dT0 = torch.from_numpy(np.ascontiguousarray(T.T)).to(dev)
    dH = torch.empty_like(dH0)
    dT = torch.empty_like(dT0)
    dQ = torch.empty_like(dH0)
    dZ = torch.empty_like(dH0)
    de = torch.empty(3 * n, dtype=torch.float64, device=dev)
    solver = pkg.Solver(dev)
    mode_note = configure(pkg, solver, args.mode)
    for kv in args.param:
        k, v = kv.split("=")
        solver.set_param(k, float(v))

    def one_solve():
        dH.copy_(dH0)
        dT.copy_(dT0)
        torch.cuda.synchronize()
        info = solver.solve_device(dH.data_ptr(), dT.data_ptr(), dQ.data_ptr(), dZ.data_ptr(), ld, n,
                                   de.data_ptr(), de.data_ptr() + 8 * n, de.data_ptr() + 16 * n)
        if info != 0:
            raise RuntimeError("solver returned INFO=%d" % info)
        st = solver.stats()
        return st["seconds"], st

    for _ in range(args.warmup):
        one_solve()
    clocks = ClockSampler(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    times, launches = [], 0
    last_stats = None
    for _ in range(args.steps):
        t, st = one_solve()
        times.append(t)
        launches += int(st.get("launches", 0))
        last_stats = st
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist is not None:
        dist.barrier()
    t_mean = float(np.mean(times))
    if dist is not None:
        tt = torch.tensor([t_mean], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_mean = float(tt.item())

    # ---- accuracy of the last timed solve: backward errors (FP64 on the
    # GPU) and the eigenvalue set against the port's solve of this pencil ----
    res_h, res_t, orth_q, orth_z = errors(torch, dH0, dT0, dH, dT, dQ, dZ, n, dev)
    fx = port_fixture(args.workload, n)
    eigen = eigen_match(fx, de, n) if fx is not None else None

    # ---- the other forms on the same pencil ----
    forms = {args.mode: {"value": t_mean, "aeds": last_stats["aeds"], "sweeps": last_stats["sweeps"],
                         "note": mode_note, "backward_error_neps": {"h": res_h, "t": res_t},
                         "orthogonality_neps": {"q": orth_q, "z": orth_z}}}
    if args.form_steps > 0:
        for fm in FORMS:
            if fm == args.mode:
                continue
            note = configure(pkg, solver, fm)
            one_solve()
            ts, st = [], None
            for _ in range(args.form_steps):
                t, st = one_solve()
                ts.append(t)
            t_f = float(np.mean(ts))
            if dist is not None:
                tt = torch.tensor([t_f], dtype=torch.float64, device=dev)
                dist.all_reduce(tt, op=dist.ReduceOp.MAX)
                t_f = float(tt.item())
            ce = errors(torch, dH0, dT0, dH, dT, dQ, dZ, n, dev)
            forms[fm] = {"value": t_f, "aeds": st["aeds"], "sweeps": st["sweeps"], "note": note,
                         "backward_error_neps": {"h": ce[0], "t": ce[1]},
                         "orthogonality_neps": {"q": ce[2], "z": ce[3]}}
        configure(pkg, solver, args.mode)
    comparison = None
    if "plain" in forms and "split+learned" in forms:
        comparison = {"split_learned_speedup_over_plain": forms["plain"]["value"] / forms["split+learned"]["value"],
                      "split_speedup_over_plain": forms["plain"]["value"] / forms["split"]["value"]
                      if "split" in forms else None,
                      "learned_speedup_over_plain": forms["plain"]["value"] / forms["learned"]["value"]
                      if "learned" in forms else None}

    # ---- profiled solve (untimed, in the benchmarked form) for the phase
    # breakdown and the roofline ----
    os.environ["B200QZ_PROFILE"] = "1"
    _, pst = one_solve()
    os.environ.pop("B200QZ_PROFILE", None)
    peaks, peak_kind = read_peaks()
    sub = ("ms_aed_smallqz", "ms_aed_reorder", "ms_aed_spike", "ms_aed_hessred")
    phases = {k[3:]: v for k, v in pst.items() if k.startswith("ms_") and k not in sub}
    fp64_peak = fp64_gemm_peak(torch, dev)
    roof = roofline_of(pst, phases, peaks, peak_kind, fp64_peak, "split" in args.mode)
    share = {k: round(v / max(1e-9, sum(phases.values())), 4) for k, v in phases.items()}
    aed_split = {k[7:]: round(pst[k], 1) for k in sub}

    # ---- end to end through the C-ABI with pinned host buffers ----
    e2e_times = []
    pin = lambda a: torch.empty(a.shape[::-1], dtype=torch.float64, pin_memory=True).numpy().T
    Hp, Tp, Qp, Zp = pin(H), pin(T), pin(H), pin(H)
    for _ in range(max(1, min(args.steps, 5))):
        np.copyto(Hp, H)
        np.copyto(Tp, T)
        t0 = time.perf_counter()
        ar, ai, be, info = solver.solve_host(Hp, Tp, Qp, Zp)
        e2e_times.append(time.perf_counter() - t0)
        if info != 0:
            raise RuntimeError("e2e solve INFO=%d" % info)
    e2e = float(np.mean(e2e_times))
    if dist is not None:
        tt = torch.tensor([e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e = float(tt.item())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(pkg, args.workload, n)

    if rank == 0:
        config = workload_config(pkg, args.workload, n, desc)
        config.update({"parallelism": "replicas" if world > 1 else "single-gpu",
                       "l2": "inputs 4 x %.0f MB > L2; restored from device copy outside timed events"
                             % (8 * n * n / 1e6),
                       "params": args.param,
                       "backward_error_neps": {"h": res_h, "t": res_t},
                       "orthogonality_neps": {"q": orth_q, "z": orth_z},
                       "eigenvalues": eigen,
                       "stats": {k: v for k, v in last_stats.items() if not k.startswith("ms_")}})
        line = {
            "metric": METRIC, "value": t_mean, "unit": "s", "n_gpus": world, "steps": args.steps,
            "mode": args.mode, "mode_note": mode_note, "forms": forms, "comparison": comparison,
            "warmup": args.warmup, "ms_per_step": t_mean * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": 2 * 8 * n * n,
                    "d2h_bytes_per_step": 4 * 8 * n * n + 3 * 8 * n},
            "gpu_launches": launches,
            "clocks": clk,
            "roofline": roof,
            "phase_share": share,
            "aed_ms": aed_split,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
