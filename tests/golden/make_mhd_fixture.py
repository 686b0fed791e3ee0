"""Generate the real-data fixture of the reference's own example pencil.

    python tests/golden/make_mhd_fixture.py [/root/reference/examples]

Test infrastructure.  The reference's example EXRAND3 (examples/EXRAND3.f:
297-316) reads the 4800 x 4800 MatrixMarket pair examples/sparseA.mtx
(general, 102252 entries) and examples/sparseB.mtx (symmetric, 16160
entries of the lower triangle), factors B = Q_B R by QR, applies Q_B^T to
A, reduces (Q_B^T A, R) to Hessenberg-triangular form with PDGGHRD and
solves it with PDHGEQZ.  This script reads the two files, and with numpy's
QR and LAPACK on one thread (DGGHD3, DHGEQZ, DTGEVC + DTGSNA) computes the
eigenvalues of the pencil and their reciprocal condition numbers.  The
fixture ``mhd4800.npz`` keeps

* ``a_i``, ``a_j``, ``a_v``: the entries of A (0-based row, column);
* ``b_i``, ``b_j``, ``b_v``: the stored entries of B (one triangle; the
  matrix is symmetric);
* ``alphar``, ``alphai``, ``beta``, ``rcond``, ``norm``: LAPACK's
  eigenvalues of (Q_B^T A, R), their DTGSNA condition numbers in LAPACK's
  Schur form, and ||(Q_B^T A, R)||_F, for the condition-scaled match.

The GPU test rebuilds the dense pencil from the entries, so the reference
tree is needed only to regenerate the fixture.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def read_mtx(path):
    """MatrixMarket coordinate real file -> (n, rows, cols, vals, symmetric)."""
    with open(path) as f:
        header = f.readline().lower()
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        nr, nc, nnz = (int(v) for v in line.split())
        data = np.loadtxt(f, dtype=np.float64, ndmin=2)
    assert nr == nc and data.shape[0] == nnz
    return nr, data[:, 0].astype(np.int32) - 1, data[:, 1].astype(np.int32) - 1, data[:, 2], "symmetric" in header


def dense(n, i, j, v, symmetric):
    M = np.zeros((n, n))
    np.add.at(M, (i, j), v)
    if symmetric:
        off = i != j
        np.add.at(M, (j[off], i[off]), v[off])
    return M


def make(src: str) -> str:
    from oracle import lapack as L
    n, ai, aj, av, asym = read_mtx(os.path.join(src, "sparseA.mtx"))
    nb, bi, bj, bv, bsym = read_mtx(os.path.join(src, "sparseB.mtx"))
    assert n == nb and not asym and bsym
    A = dense(n, ai, aj, av, False)
    B = dense(n, bi, bj, bv, True)
    L.set_threads(1)
    t0 = time.perf_counter()
    qb, rb = np.linalg.qr(B)
    A1 = qb.T @ A
    B1 = np.triu(rb)
    H, T, _, _, info = L.dgghd3(A1, B1, "N", "N")
    assert info == 0
    S, P, ar, ai_, be, _, _, info = L.dhgeqz(H, T, job="S", compq="N", compz="N")
    assert info == 0
    print("LAPACK QR + DGGHD3 + DHGEQZ: %.1f s" % (time.perf_counter() - t0), flush=True)
    t1 = time.perf_counter()
    s = L.eig_condition(S, P)
    print("DTGEVC + DTGSNA: %.1f s" % (time.perf_counter() - t1), flush=True)
    out = os.path.join(HERE, "mhd4800.npz")
    np.savez_compressed(out, a_i=ai, a_j=aj, a_v=av, b_i=bi, b_j=bj, b_v=bv, alphar=ar, alphai=ai_, beta=be,
                        rcond=s, norm=np.hypot(np.linalg.norm(A1), np.linalg.norm(B1)))
    return out


if __name__ == "__main__":
    print(make(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/examples"))
