"""Generate the eigenvalue fixtures of the oracle port at the benchmark sizes.

    python tests/golden/make_port_fixtures.py c3      # n=10000 graded, seed 2
    python tests/golden/make_port_fixtures.py c2      # n=4000, 5% zero T diagonal, seed 1
    python tests/golden/make_port_fixtures.py c4      # n=16000, seed 3 (about 75 min, mostly DTGSNA)

Test infrastructure.  For each workload the oracle's C restatement of the
reference path (oracle/qzref.c, the PDHGEQZ0 regime above n=6000, PDHGEQZ1
below) solves the seeded pencil once with OpenBLAS on all host threads.  The
fixture ``port_<workload>_n<n>.npz`` keeps

* ``alphar``, ``alphai``, ``beta``: the port's eigenvalues;
* ``rcond``: DTGSNA reciprocal condition numbers s_j of those eigenvalues in
  the port's Schur form (DTGEVC eigenvectors), which scale the chordal
  matching tolerance 50 n eps ||(H,T)||_F / s_j;
* ``norm``: ||(H, T)||_F of the input pencil;
* ``seconds``, ``threads``, ``info`` and the port's backward errors;
* ``aed_clock``: the seconds since the start of the solve at which each AED
  began (the profile that scales bench.py's bounded CPU-baseline sample,
  which runs the port on the same pencil for its first AEDs only).

The GPU parity test of the full-size pencils and bench.py's eigenvalue check
compare against these arrays, so the n=10000 comparison needs no CPU solve
on the GPU machine.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def _pencils():
    import importlib.util
    spec = importlib.util.spec_from_file_location("pencils", os.path.join(ROOT, "gevp-pdhgeqz_b200", "pencils.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def make(workload: str) -> str:
    from oracle import lapack as L
    from oracle import qzref as R

    P = _pencils()
    n = P.WORKLOADS[workload]["n"]
    H, T = P.workload(workload)
    threads = os.cpu_count() or 1
    L.set_threads(threads)
    R.lib()
    clock = np.zeros(100000)
    t0 = time.perf_counter()
    S, Pm, Q, Z, ar, ai, be, info, st = R.pdhgeqz(H, T, nb=130 if n > 6000 else 60, aed_clock=clock)
    secs = time.perf_counter() - t0
    clock = clock[:int(st["aeds"])]
    print("%s: port n=%d info=%d %.1f s on %d threads %s" % (workload, n, info, secs, threads, st), flush=True)
    r = L.residuals(H, T, S, Pm, Q, Z)
    print("  residuals (n eps): %s" % {k: r[k] / r["neps"] for k in "htqz"}, flush=True)
    del Q, Z
    t1 = time.perf_counter()
    s = L.eig_condition(S, Pm)
    print("  DTGEVC + DTGSNA %.1f s" % (time.perf_counter() - t1), flush=True)
    out = os.path.join(HERE, "port_%s_n%d.npz" % (workload, n))
    np.savez_compressed(out, alphar=ar, alphai=ai, beta=be, rcond=s,
                        norm=np.hypot(np.linalg.norm(H), np.linalg.norm(T)), seconds=secs, threads=threads,
                        info=info, res=np.array([r[k] / r["neps"] for k in "htqz"]), aed_clock=clock)
    return out


if __name__ == "__main__":
    for w in sys.argv[1:] or ["c3"]:
        print(make(w))
