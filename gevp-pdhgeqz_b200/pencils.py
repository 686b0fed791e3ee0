"""Seeded Hessenberg-triangular pencil generators for the five benchmark
workloads of the multishift QZ path.

Every generator uses numpy's Philox counter-based bit generator
(``numpy.random.Generator(numpy.random.Philox(seed))``) and returns
Fortran-ordered (column-major) float64 arrays, the storage the PDHGEQZ
interface expects (``src/pdhgeqz/PDHGEQZ.f:15-31``: H, T, Q, Z are local
column-major arrays with leading dimension ``DESC(9)``).

The reference's own drivers draw H and T uniformly from (-1, 1] with
chi-like subdiagonals (``testing/EXRAND1.f:243-279``) from a
non-reproducible seed; the workloads here use the normal distributions the
benchmark configurations name instead, with fixed seeds.

Workloads
---------
* ``c1``  n=1000, seed 0: H upper Hessenberg and T upper triangular, N(0,1).
* ``c2``  n=4000, seed 1: as c1 plus 5% of T's diagonal set to exactly 0 at
  seeded positions (infinite eigenvalues).
* ``c3``  n=10000, seed 2: graded, H = D1 X_H D2, T = D1 X_T D2 with
  diag(D1), diag(D2) = 10**u, u ~ U(-3, 3).
* ``c4``  training pencils with every 50th subdiagonal scaled by 1e-8, and
  the n=16000 seed-3 evaluation pencil.
* ``c5``  2048 pencils, seed 4, n ~ U{32..512}, N(0,1), 2% zero T-diagonal.
"""
from __future__ import annotations

import numpy as np

GENERATOR = "numpy.random.Philox(seed) standard_normal, column-major"


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(int(seed)))


def _ht_from_rng(rng: np.random.Generator, n: int):
    """Draw H (Hessenberg) and T (triangular) column by column.

    Column j of H holds rows 0..min(j+1, n-1); column j of T rows 0..j.  The
    draws are taken in that order so the bytes do not depend on memory
    layout.
    """
    H = np.zeros((n, n), dtype=np.float64, order="F")
    T = np.zeros((n, n), dtype=np.float64, order="F")
    # one bulk draw, then scatter: count of entries in each column
    hcnt = np.minimum(np.arange(n) + 2, n)
    tcnt = np.arange(n) + 1
    hv = rng.standard_normal(int(hcnt.sum()))
    tv = rng.standard_normal(int(tcnt.sum()))
    hoff = 0
    toff = 0
    for j in range(n):
        H[: hcnt[j], j] = hv[hoff:hoff + hcnt[j]]
        hoff += hcnt[j]
        T[: tcnt[j], j] = tv[toff:toff + tcnt[j]]
        toff += tcnt[j]
    return H, T


def random_ht(n: int, seed: int, zero_frac: float = 0.0):
    """N(0,1) Hessenberg-triangular pencil; optionally a fraction of T's
    diagonal entries set to exactly zero at seeded positions."""
    rng = _rng(seed)
    H, T = _ht_from_rng(rng, n)
    if zero_frac > 0.0 and n > 0:
        nz = int(round(zero_frac * n))
        pos = rng.choice(n, size=nz, replace=False)
        T[pos, pos] = 0.0
    return H, T


def graded_ht(n: int, seed: int, decades: float = 3.0):
    """Graded pencil H = D1 X_H D2, T = D1 X_T D2, diag entries 10**U(-d, d)."""
    rng = _rng(seed)
    H, T = _ht_from_rng(rng, n)
    d1 = 10.0 ** rng.uniform(-decades, decades, n)
    d2 = 10.0 ** rng.uniform(-decades, decades, n)
    H *= d1[:, None]
    H *= d2[None, :]
    T *= d1[:, None]
    T *= d2[None, :]
    return H, T


def clustered_ht(n: int, seed: int, every: int = 50, scale: float = 1e-8):
    """N(0,1) pencil with every ``every``-th subdiagonal entry scaled."""
    H, T = random_ht(n, seed)
    idx = np.arange(every, n, every)
    H[idx, idx - 1] *= scale
    return H, T


def batch_sizes(count: int, seed: int, lo: int = 32, hi: int = 512):
    return _rng(seed).integers(lo, hi + 1, size=count)


def batched_ht(count: int = 2048, seed: int = 4, lo: int = 32, hi: int = 512,
               zero_frac: float = 0.02):
    """List of (H, T) for the batched workload: sizes from ``seed``, pencil
    i drawn from seed ``seed * 1_000_003 + i``."""
    sizes = batch_sizes(count, seed, lo, hi)
    out = []
    for i, n in enumerate(sizes):
        out.append(random_ht(int(n), seed * 1_000_003 + i, zero_frac))
    return out


def batched_pencil(index: int, n: int, seed: int = 4, zero_frac: float = 0.02):
    """Pencil ``index`` of the batched workload (same draw as batched_ht)."""
    return random_ht(int(n), seed * 1_000_003 + int(index), zero_frac)


WORKLOADS = {
    "c1": dict(n=1000, seed=0, kind="random", zero_frac=0.0),
    "c2": dict(n=4000, seed=1, kind="random", zero_frac=0.05),
    "c3": dict(n=10000, seed=2, kind="graded"),
    "c4": dict(n=16000, seed=3, kind="random", zero_frac=0.0),
}


def workload(name: str, n: int | None = None):
    """Return (H, T) for a named workload, optionally at a smaller n with
    the same distribution (used by parity tests)."""
    w = WORKLOADS[name]
    n = int(n if n is not None else w["n"])
    if w["kind"] == "graded":
        return graded_ht(n, w["seed"])
    return random_ht(n, w["seed"], w.get("zero_frac", 0.0))
