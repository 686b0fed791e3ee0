// Reordering of a generalized real Schur form (S, T) with Q, Z on the
// device, so that the selected eigenvalues lead: the semantics of LAPACK
// DTGSEN for IJOB 0 and 1, in the role of the reference's PDTGSEN and its
// windowed reordering PDTGORD (src/reorder/PDTGSEN.f:1, PDTGORD.f:1;
// used after the solve at examples/EXRAND3.f:473).
//
// Moves.  The selected blocks are taken in order from the top; each moves
// up to the next free position through windows of at most 80 rows.  One
// CTA holds a window's S and T in shared memory, swaps the block up to the
// window's top by adjacent block swaps (the generalized Sylvester swap of
// the AED, cta_swap, standardising the 2x2 blocks it moves) and
// accumulates the window's orthogonal factors U, V; the DMMA update
// kernels then apply U, V to the rest of S, T and to Q, Z.  The host keeps
// the block structure (sizes in order), so windows start at block
// boundaries without reading the matrices back.  A rejected swap sets a
// device flag: later windows leave their pencil unchanged (identity
// factors) and the call returns info = 1 with the partly reordered form,
// as DTGSEN does.
//
// Normalisation.  A 1x1 block whose T entry is negative has its rows of S
// and T and its column of Q negated (DTGSEN's convention); the eigenvalues
// are read from the diagonal blocks.
//
// Projections (IJOB 1).  With m selected eigenvalues, R and L (m x (n-m))
// solve the generalized Sylvester equation
//     S11 R - L S22 = S12,   T11 R - L T22 = T12,
// and PL = 1 / sqrt(1 + |R|_F^2), PR = 1 / sqrt(1 + |L|_F^2) (Kagstrom and
// Poromaa, "Computing eigenspaces with specified eigenvalues of a regular
// matrix pair (A,B) and condition estimation", Numer. Algorithms 12
// (1996)).  The solve runs on anti-diagonal waves of diagonal-block pairs
// (block rows from the bottom, block columns from the left): a warp per
// pair gathers its right-hand side from the already solved blocks,
//     S11(i,i) R(i,j) - L(i,j) S22(j,j)
//        = S12(i,j) - sum_{k>i} S11(i,k) R(k,j) + sum_{k<j} L(i,k) S22(k,j),
// and the same with T, and solves the Kronecker system of order <= 8 by
// Gaussian elimination with complete pivoting.
#include "reorder.h"

#include <cfloat>
#include <cmath>
#include <vector>

#include "kernels.h"
#include "onenorm.h"

namespace qz {
namespace {

constexpr int kReoWin = 80;  // window rows (shared memory)
constexpr int kReoThreads = 128;

struct ReoExec {
  int tid, nt;
  int* si;
  double* sd;
  __device__ void sync() { __syncthreads(); }
  __device__ void stamp(int) {}
  __device__ void count(int) {}
};

size_t reo_smem(int wk) { return ((size_t)4 * wk * smem_ld(wk) + 256) * sizeof(double) + 64 * sizeof(int); }

// Move the block at window row ifst (size bs) up to window row 0 of the
// window S(w0:w0+wk, w0:w0+wk); U, V receive the window's factors.
// status = {failed, global row where the block stopped}.
__global__ void __launch_bounds__(kReoThreads) k_reorder_win(double* S, int64_t lds, double* T, int64_t ldt, int w0,
                                                             int wk, int ifst, int bs, Tol tol, double* U, double* V,
                                                             int* status) {
  extern __shared__ double smem[];
  const int lw = smem_ld(wk);
  double* Hs = smem;
  double* Ts = Hs + wk * lw;
  double* Us = Ts + wk * lw;
  double* Vs = Us + wk * lw;
  double* sd = Vs + wk * lw;
  int* si = (int*)(sd + 256);
  const bool skip = *(volatile int*)status != 0;  // an earlier window was rejected
  for (int idx = threadIdx.x; idx < wk * wk; idx += blockDim.x) {
    const int i = idx % wk, j = idx / wk;
    if (!skip) {
      Hs[i + j * lw] = S[(w0 + i) + (int64_t)(w0 + j) * lds];
      Ts[i + j * lw] = T[(w0 + i) + (int64_t)(w0 + j) * ldt];
    }
    Us[i + j * lw] = (i == j) ? 1.0 : 0.0;
    Vs[i + j * lw] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  if (!skip) {
    ReoExec x{(int)threadIdx.x, (int)blockDim.x, si, sd};
    WinState w;
    w.n = wk;
    w.H = MatV{Hs, lw};
    w.T = MatV{Ts, lw};
    w.Q = MatV{Us, lw};
    w.Z = MatV{Vs, lw};
    w.wantq = true;
    w.wantz = true;
    w.tol = tol;
    int here = ifst;
    bool ok = true;
    while (here > 0) {
      int nbn = 1;
      if (here >= 2 && w.H(here - 1, here - 2) != 0.0) nbn = 2;
      if (!cta_swap(x, w, here - nbn, nbn, bs, true)) { ok = false; break; }
      here -= nbn;
      const int nbnow = (bs == 2 && w.H(here + 1, here) != 0.0) ? 2 : 1;
      if (nbnow != bs) { ok = false; break; }
    }
    __syncthreads();
    if (!ok && threadIdx.x == 0) {
      status[0] = 1;
      status[1] = w0 + here;
    }
    for (int idx = threadIdx.x; idx < wk * wk; idx += blockDim.x) {
      const int i = idx % wk, j = idx / wk;
      S[(w0 + i) + (int64_t)(w0 + j) * lds] = Hs[i + j * lw];
      T[(w0 + i) + (int64_t)(w0 + j) * ldt] = Ts[i + j * lw];
    }
  }
  for (int idx = threadIdx.x; idx < wk * wk; idx += blockDim.x) {
    const int i = idx % wk, j = idx / wk;
    U[idx] = Us[i + j * lw];
    V[idx] = Vs[i + j * lw];
  }
}

// 1x1 blocks with a negative T entry: rows of S and T and column of Q negated
__global__ void k_tgsen_signs(double* S, int64_t lds, double* T, int64_t ldt, double* Q, int64_t ldq, int n,
                              int wantq) {
  const int k = blockIdx.x;
  const bool below = (k + 1 < n) && S[(k + 1) + (int64_t)k * lds] != 0.0;
  const bool above = (k > 0) && S[k + (int64_t)(k - 1) * lds] != 0.0;
  if (below || above || !signbit(T[k + (int64_t)k * ldt])) return;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    S[k + (int64_t)j * lds] = -S[k + (int64_t)j * lds];
    T[k + (int64_t)j * ldt] = -T[k + (int64_t)j * ldt];
    if (wantq) Q[j + (int64_t)k * ldq] = -Q[j + (int64_t)k * ldq];
  }
}

__global__ void k_tgsen_eigs(const double* S, int64_t lds, const double* T, int64_t ldt, int n, double* ar, double* ai,
                             double* be) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const bool below = (j + 1 < n) && S[(j + 1) + (int64_t)j * lds] != 0.0;
  const bool above = (j > 0) && S[j + (int64_t)(j - 1) * lds] != 0.0;
  if (!below && !above) {
    ar[j] = S[j + (int64_t)j * lds];
    ai[j] = 0.0;
    be[j] = T[j + (int64_t)j * ldt];
    return;
  }
  const int f = below ? j : j - 1;
  const double a[4] = {S[f + (int64_t)f * lds], S[(f + 1) + (int64_t)f * lds], S[f + (int64_t)(f + 1) * lds],
                       S[(f + 1) + (int64_t)(f + 1) * lds]};
  double o_ar[2], o_ai[2], o_be[2];
  eig2_complex(a, T[f + (int64_t)f * ldt], T[(f + 1) + (int64_t)(f + 1) * ldt], o_ar, o_ai, o_be);
  const int e = j - f;
  ar[j] = e ? o_ar[1] : o_ar[0];
  ai[j] = e ? o_ai[1] : o_ai[0];
  be[j] = e ? o_be[1] : o_be[0];
}

// transposed copy of the leading m x m block: D(j, i) = A(i, j)
__global__ void k_transpose_lead(const double* A, int64_t lda, int m, double* D) {
  __shared__ double tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int i = bx + threadIdx.x, j = by + k;
    if (i < m && j < m) tile[k][threadIdx.x] = A[i + (int64_t)j * lda];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int j = by + threadIdx.x, i = bx + k;
    if (i < m && j < m) D[j + (int64_t)i * m] = tile[threadIdx.x][k];
  }
}

struct SylvArgs {
  const double* S;  // pencil (S, T), leading dimensions lds, ldt
  const double* T;
  int64_t lds, ldt;
  int m1, m2;            // S11 is m1 x m1, S22 is m2 x m2 (at (m1, m1))
  const double* S11t;    // S11^T, T11^T (m1 x m1)
  const double* T11t;
  double* R;             // m1 x m2 (ld m1)
  double* Lt;            // L^T, m2 x m1 (ld m2)
  const int* b1s;        // diagonal blocks of S11: starts, sizes
  const int* b1z;
  const int* b2s;        // of S22 (relative to m1)
  const int* b2z;
  int nb1, nb2;
};

template <int P, int Q>
__device__ void sylv_block_solve(const SylvArgs& a, int i0, int j0, const double* ce, const double* fe) {
  constexpr int NQ = P * Q, NS = 2 * NQ;
  double A[NS * NS], rhs[NS];
#pragma unroll
  for (int k = 0; k < NS * NS; ++k) A[k] = 0.0;
  const int m1 = a.m1;
#pragma unroll
  for (int j = 0; j < Q; ++j)
#pragma unroll
    for (int i = 0; i < P; ++i) {
      const int row = i + P * j;
#pragma unroll
      for (int k = 0; k < P; ++k) {
        A[row + NS * (k + P * j)] += a.S[(i0 + i) + (int64_t)(i0 + k) * a.lds];
        A[(row + NQ) + NS * (k + P * j)] += a.T[(i0 + i) + (int64_t)(i0 + k) * a.ldt];
      }
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        A[row + NS * (NQ + i + P * k)] -= a.S[(m1 + j0 + k) + (int64_t)(m1 + j0 + j) * a.lds];
        A[(row + NQ) + NS * (NQ + i + P * k)] -= a.T[(m1 + j0 + k) + (int64_t)(m1 + j0 + j) * a.ldt];
      }
      rhs[row] = ce[i + 2 * j];
      rhs[row + NQ] = fe[i + 2 * j];
    }
  small_solve_cp<NS>(A, rhs, DBL_MIN);
#pragma unroll
  for (int j = 0; j < Q; ++j)
#pragma unroll
    for (int i = 0; i < P; ++i) {
      a.R[(i0 + i) + (int64_t)(j0 + j) * m1] = rhs[i + P * j];
      a.Lt[(j0 + j) + (int64_t)(i0 + i) * a.m2] = rhs[NQ + i + P * j];
    }
}

// one anti-diagonal wave d of block pairs, a warp per pair
__global__ void k_sylv_wave(SylvArgs a, int d) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int jlo = d - (a.nb1 - 1) > 0 ? d - (a.nb1 - 1) : 0;
  const int jhi = d < a.nb2 - 1 ? d : a.nb2 - 1;
  const int bj = jlo + warp;
  if (bj > jhi) return;
  const int bi = a.nb1 - 1 - (d - bj);
  const int i0 = a.b1s[bi], p = a.b1z[bi], j0 = a.b2s[bj], q = a.b2z[bj];
  const int m1 = a.m1, m2 = a.m2;
  // acc[a + 2b]: S- and T-parts of the rows below (R) and the columns to the left (L)
  double sr[4] = {0, 0, 0, 0}, tr[4] = {0, 0, 0, 0}, sl[4] = {0, 0, 0, 0}, tl[4] = {0, 0, 0, 0};
  for (int k = i0 + p + lane; k < m1; k += 32) {
    const double s0 = a.S11t[k + (int64_t)i0 * m1], t0 = a.T11t[k + (int64_t)i0 * m1];
    const double s1 = (p > 1) ? a.S11t[k + (int64_t)(i0 + 1) * m1] : 0.0;
    const double t1 = (p > 1) ? a.T11t[k + (int64_t)(i0 + 1) * m1] : 0.0;
    const double r0 = a.R[k + (int64_t)j0 * m1];
    const double r1 = (q > 1) ? a.R[k + (int64_t)(j0 + 1) * m1] : 0.0;
    sr[0] += s0 * r0; sr[1] += s1 * r0; sr[2] += s0 * r1; sr[3] += s1 * r1;
    tr[0] += t0 * r0; tr[1] += t1 * r0; tr[2] += t0 * r1; tr[3] += t1 * r1;
  }
  for (int k = lane; k < j0; k += 32) {
    const double l0 = a.Lt[k + (int64_t)i0 * m2];
    const double l1 = (p > 1) ? a.Lt[k + (int64_t)(i0 + 1) * m2] : 0.0;
    const double s0 = a.S[(m1 + k) + (int64_t)(m1 + j0) * a.lds], t0 = a.T[(m1 + k) + (int64_t)(m1 + j0) * a.ldt];
    const double s1 = (q > 1) ? a.S[(m1 + k) + (int64_t)(m1 + j0 + 1) * a.lds] : 0.0;
    const double t1 = (q > 1) ? a.T[(m1 + k) + (int64_t)(m1 + j0 + 1) * a.ldt] : 0.0;
    sl[0] += l0 * s0; sl[1] += l1 * s0; sl[2] += l0 * s1; sl[3] += l1 * s1;
    tl[0] += l0 * t0; tl[1] += l1 * t0; tl[2] += l0 * t1; tl[3] += l1 * t1;
  }
#pragma unroll
  for (int e = 0; e < 4; ++e)
    for (int o = 16; o; o >>= 1) {
      sr[e] += __shfl_xor_sync(0xffffffffu, sr[e], o);
      tr[e] += __shfl_xor_sync(0xffffffffu, tr[e], o);
      sl[e] += __shfl_xor_sync(0xffffffffu, sl[e], o);
      tl[e] += __shfl_xor_sync(0xffffffffu, tl[e], o);
    }
  if (lane != 0) return;
  double ce[4], fe[4];
  for (int b = 0; b < q; ++b)
    for (int i = 0; i < p; ++i) {
      ce[i + 2 * b] = a.S[(i0 + i) + (int64_t)(m1 + j0 + b) * a.lds] - sr[i + 2 * b] + sl[i + 2 * b];
      fe[i + 2 * b] = a.T[(i0 + i) + (int64_t)(m1 + j0 + b) * a.ldt] - tr[i + 2 * b] + tl[i + 2 * b];
    }
  if (p == 1 && q == 1) sylv_block_solve<1, 1>(a, i0, j0, ce, fe);
  else if (p == 1) sylv_block_solve<1, 2>(a, i0, j0, ce, fe);
  else if (q == 1) sylv_block_solve<2, 1>(a, i0, j0, ce, fe);
  else sylv_block_solve<2, 2>(a, i0, j0, ce, fe);
}

// sums of squares of x[0..len) per block, then one fixed-order total
constexpr int kSsqBlocks = 256;
__global__ void k_ssq_part(const double* x, int64_t len, double* part) {
  __shared__ double red[8];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
    s += x[i] * x[i];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    part[blockIdx.x] = t;
  }
}
__global__ void k_ssq_final(const double* part, int np, double* out) {
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < np; ++i) t += part[i];
    *out = t;
  }
}

// ---------------------------------------------------------------------------
// General generalized Sylvester solve for the Dif estimates (the role of
// LAPACK DTGSYL with IJOB = 0 inside DTGSEN IJOB 3 and 5): (A, D) is an
// m x m and (B, E) an n x n upper quasi-triangular pair, (C, F) an m x n
// right-hand side overwritten by the solution (R, L) of
//   trans 0:  A R - L B = C,        D R - L E = F
//   trans 1:  A^T R + D^T L = C,    R B^T + L E^T = -F
// Block pairs (i, j) of the diagonal blocks are solved on anti-diagonal
// waves, a warp per pair: trans 0 from the bottom-left corner (blocks below
// and to the left first), trans 1 from the top-right corner.
// ---------------------------------------------------------------------------
struct SylvGen {
  const double *A, *D, *B, *E;
  int64_t lda, ldd, ldb, lde;
  double *C, *F;  // m x n, leading dimension m
  int m, n;
  const int *as, *az, *bs, *bz;  // diagonal blocks: starts, sizes
  int na, nb;
  int trans;
};

template <int P, int Q>
__device__ void sylv_gen_solve(const SylvGen& g, int i0, int j0, const double* ce, const double* fe) {
  constexpr int NQ = P * Q, NS = 2 * NQ;
  double M[NS * NS], rhs[NS];
#pragma unroll
  for (int k = 0; k < NS * NS; ++k) M[k] = 0.0;
  auto A = [&](int r, int c) { return g.A[(i0 + r) + (int64_t)(i0 + c) * g.lda]; };
  auto D = [&](int r, int c) { return g.D[(i0 + r) + (int64_t)(i0 + c) * g.ldd]; };
  auto B = [&](int r, int c) { return g.B[(j0 + r) + (int64_t)(j0 + c) * g.ldb]; };
  auto E = [&](int r, int c) { return g.E[(j0 + r) + (int64_t)(j0 + c) * g.lde]; };
#pragma unroll
  for (int b = 0; b < Q; ++b)
#pragma unroll
    for (int a = 0; a < P; ++a) {
      const int r1 = a + P * b, r2 = NQ + a + P * b;
#pragma unroll
      for (int c = 0; c < P; ++c) {
        if (g.trans) {
          M[r1 + NS * (c + P * b)] += A(c, a);
          M[r1 + NS * (NQ + c + P * b)] += D(c, a);
        } else {
          M[r1 + NS * (c + P * b)] += A(a, c);
          M[r2 + NS * (c + P * b)] += D(a, c);
        }
      }
#pragma unroll
      for (int c = 0; c < Q; ++c) {
        if (g.trans) {
          M[r2 + NS * (a + P * c)] += B(b, c);
          M[r2 + NS * (NQ + a + P * c)] += E(b, c);
        } else {
          M[r1 + NS * (NQ + a + P * c)] -= B(c, b);
          M[r2 + NS * (NQ + a + P * c)] -= E(c, b);
        }
      }
      rhs[r1] = ce[a + 2 * b];
      rhs[r2] = fe[a + 2 * b];
    }
  small_solve_cp<NS>(M, rhs, DBL_MIN);
#pragma unroll
  for (int b = 0; b < Q; ++b)
#pragma unroll
    for (int a = 0; a < P; ++a) {
      g.C[(i0 + a) + (int64_t)(j0 + b) * g.m] = rhs[a + P * b];
      g.F[(i0 + a) + (int64_t)(j0 + b) * g.m] = rhs[NQ + a + P * b];
    }
}

__global__ void k_sylv_gen_wave(SylvGen g, int d) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  int bi, bj;
  if (!g.trans) {
    const int jlo = d - (g.na - 1) > 0 ? d - (g.na - 1) : 0;
    const int jhi = d < g.nb - 1 ? d : g.nb - 1;
    bj = jlo + warp;
    if (bj > jhi) return;
    bi = g.na - 1 - (d - bj);
  } else {
    const int ilo = d - (g.nb - 1) > 0 ? d - (g.nb - 1) : 0;
    const int ihi = d < g.na - 1 ? d : g.na - 1;
    bi = ilo + warp;
    if (bi > ihi) return;
    bj = g.nb - 1 - (d - bi);
  }
  const int i0 = g.as[bi], p = g.az[bi], j0 = g.bs[bj], q = g.bz[bj];
  const int m = g.m, n = g.n;
  double s1[4] = {0, 0, 0, 0}, s2[4] = {0, 0, 0, 0};
  if (!g.trans) {
    // rows below (solved R) and columns to the left (solved L)
    for (int k = i0 + p + lane; k < m; k += 32)
      for (int b = 0; b < q; ++b) {
        const double r = g.C[k + (int64_t)(j0 + b) * m];
        for (int a = 0; a < p; ++a) {
          s1[a + 2 * b] -= g.A[(i0 + a) + (int64_t)k * g.lda] * r;
          s2[a + 2 * b] -= g.D[(i0 + a) + (int64_t)k * g.ldd] * r;
        }
      }
    for (int k = lane; k < j0; k += 32)
      for (int a = 0; a < p; ++a) {
        const double l = g.F[(i0 + a) + (int64_t)k * m];
        for (int b = 0; b < q; ++b) {
          s1[a + 2 * b] += l * g.B[k + (int64_t)(j0 + b) * g.ldb];
          s2[a + 2 * b] += l * g.E[k + (int64_t)(j0 + b) * g.lde];
        }
      }
  } else {
    // rows above (solved R, L) and columns to the right (solved R, L)
    for (int k = lane; k < i0; k += 32)
      for (int b = 0; b < q; ++b) {
        const double r = g.C[k + (int64_t)(j0 + b) * m], l = g.F[k + (int64_t)(j0 + b) * m];
        for (int a = 0; a < p; ++a)
          s1[a + 2 * b] -= g.A[k + (int64_t)(i0 + a) * g.lda] * r + g.D[k + (int64_t)(i0 + a) * g.ldd] * l;
      }
    for (int k = j0 + q + lane; k < n; k += 32)
      for (int a = 0; a < p; ++a) {
        const double r = g.C[(i0 + a) + (int64_t)k * m], l = g.F[(i0 + a) + (int64_t)k * m];
        for (int b = 0; b < q; ++b)
          s2[a + 2 * b] -= r * g.B[(j0 + b) + (int64_t)k * g.ldb] + l * g.E[(j0 + b) + (int64_t)k * g.lde];
      }
  }
#pragma unroll
  for (int e = 0; e < 4; ++e)
    for (int o = 16; o; o >>= 1) {
      s1[e] += __shfl_xor_sync(0xffffffffu, s1[e], o);
      s2[e] += __shfl_xor_sync(0xffffffffu, s2[e], o);
    }
  if (lane != 0) return;
  double ce[4], fe[4];
  for (int b = 0; b < q; ++b)
    for (int a = 0; a < p; ++a) {
      const double c0 = g.C[(i0 + a) + (int64_t)(j0 + b) * m], f0 = g.F[(i0 + a) + (int64_t)(j0 + b) * m];
      ce[a + 2 * b] = c0 + s1[a + 2 * b];
      fe[a + 2 * b] = (g.trans ? -f0 : f0) + s2[a + 2 * b];
    }
  if (p == 1 && q == 1) sylv_gen_solve<1, 1>(g, i0, j0, ce, fe);
  else if (p == 1) sylv_gen_solve<1, 2>(g, i0, j0, ce, fe);
  else if (q == 1) sylv_gen_solve<2, 1>(g, i0, j0, ce, fe);
  else sylv_gen_solve<2, 2>(g, i0, j0, ce, fe);
}

struct DevMem {
  void* p = nullptr;
  ~DevMem() {
    if (p) cudaFree(p);
  }
};

void add_job(UpdBatch& B, double* M, int64_t ld, int r0, int c0, int len, const double* W, int k) {
  if (len <= 0 || !M) return;
  UpdJob& j = B.job[B.njobs++];
  j.M = M; j.ld = ld; j.r0 = r0; j.c0 = c0; j.len = len; j.W = W; j.ldw = k; j.k = k;
  j.tiles = (len + update_tile(k) - 1) / update_tile(k);
}

// Difu and Difl of the reordered pencil by the 1-norm estimates of DTGSEN
// IJOB 3/5: Difu = 1 / est(Zu^-1), Zu the Sylvester operator of (S11, T11)
// and (S22, T22); Difl the same with the blocks exchanged.  b1/b2: the
// diagonal blocks of S11 and of S22 (starts relative to their block, then
// sizes).
cudaError_t dif_estimates(cudaStream_t st, const double* S, int64_t lds, const double* T, int64_t ldt, int m1,
                          int m2, const std::vector<int>& b1s, const std::vector<int>& b1z,
                          const std::vector<int>& b2s, const std::vector<int>& b2z, double* dif) {
  const int n1 = (int)b1s.size(), n2 = (int)b2s.size();
  const size_t mn = (size_t)m1 * m2;
  DevMem mem;
  cudaError_t e = cudaMalloc(&mem.p, 2 * mn * sizeof(double) + 2 * (size_t)(n1 + n2) * sizeof(int));
  if (e != cudaSuccess) return e;
  double* X = (double*)mem.p;
  int* dbl = (int*)(X + 2 * mn);
  std::vector<int> hb;
  hb.insert(hb.end(), b1s.begin(), b1s.end());
  hb.insert(hb.end(), b1z.begin(), b1z.end());
  hb.insert(hb.end(), b2s.begin(), b2s.end());
  hb.insert(hb.end(), b2z.begin(), b2z.end());
  e = cudaMemcpyAsync(dbl, hb.data(), hb.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  const double* S22 = S + m1 + (int64_t)m1 * lds;
  const double* T22 = T + m1 + (int64_t)m1 * ldt;
  for (int which = 0; which < 2; ++which) {
    SylvGen g;
    if (which == 0) {
      g.A = S; g.D = T; g.B = S22; g.E = T22; g.m = m1; g.n = m2;
      g.as = dbl; g.az = dbl + n1; g.bs = dbl + 2 * n1; g.bz = dbl + 2 * n1 + n2; g.na = n1; g.nb = n2;
    } else {
      g.A = S22; g.D = T22; g.B = S; g.E = T; g.m = m2; g.n = m1;
      g.as = dbl + 2 * n1; g.az = dbl + 2 * n1 + n2; g.bs = dbl; g.bz = dbl + n1; g.na = n2; g.nb = n1;
    }
    g.lda = g.ldb = lds;
    g.ldd = g.lde = ldt;
    g.C = X;
    g.F = X + mn;
    auto apply = [&](int kind, std::vector<double>& x) {
      g.trans = kind == 2 ? 1 : 0;
      if (cudaMemcpyAsync(X, x.data(), 2 * mn * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return false;
      const int waves = g.na + g.nb - 1, width = g.na < g.nb ? g.na : g.nb;
      for (int d = 0; d < waves; ++d) k_sylv_gen_wave<<<(width + 7) / 8, 256, 0, st>>>(g, d);
      if (cudaGetLastError() != cudaSuccess) return false;
      if (cudaMemcpyAsync(x.data(), X, 2 * mn * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return false;
      return cudaStreamSynchronize(st) == cudaSuccess;
    };
    bool ok = true;
    const double est = onenorm_est((int)(2 * mn), apply, ok);
    if (!ok) return cudaErrorUnknown;
    dif[which] = 1.0 / est;
  }
  return cudaSuccess;
}

}  // namespace

cudaError_t tgsen_device(cudaStream_t st, int ijob, bool wantq, bool wantz, const int* select, int n, double* S,
                         int64_t lds, double* T, int64_t ldt, double* Q, int64_t ldq, double* Z, int64_t ldz,
                         double* alphar, double* alphai, double* beta, ReorderOut* out) {
  *out = ReorderOut{};
  if (n <= 0) return cudaSuccess;
  cudaError_t e;
  // block structure from the subdiagonal of S
  std::vector<double> sub(n > 1 ? n - 1 : 1, 0.0);
  if (n > 1) {
    e = cudaMemcpy2DAsync(sub.data(), sizeof(double), S + 1, (size_t)(lds + 1) * sizeof(double), sizeof(double),
                          n - 1, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
  }
  std::vector<int> sz, sel;
  for (int k = 0; k < n;) {
    const int bs = (k + 1 < n && sub[k] != 0.0) ? 2 : 1;
    sz.push_back(bs);
    sel.push_back((select[k] != 0) || (bs == 2 && select[k + 1] != 0));
    out->m += sel.back() ? bs : 0;
    k += bs;
  }
  const int nb = (int)sz.size();
  Tol tol;
  tol.ulp = DBL_EPSILON;
  tol.safmin = DBL_MIN;
  tol.smlnum = DBL_MIN * ((double)n / DBL_EPSILON);
  tol.ttol = DBL_MIN;
  tol.htol = DBL_MIN;

  DevMem mem;
  e = cudaMalloc(&mem.p, sizeof(double) * 2 * kReoWin * kReoWin + 64);
  if (e != cudaSuccess) return e;
  double* U = (double*)mem.p;
  double* V = U + kReoWin * kReoWin;
  int* status = (int*)(V + kReoWin * kReoWin);
  e = cudaMemsetAsync(status, 0, 2 * sizeof(int), st);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_reorder_win, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)reo_smem(kReoWin));
  if (e != cudaSuccess) return e;

  int ks = 0, bks = 0;  // next free row and block index
  for (int b = 0; b < nb && out->info == 0; ++b) {
    if (!sel[b]) continue;
    int pos = ks;
    for (int k = bks; k < b; ++k) pos += sz[k];
    const int bs = sz[b];
    int ci = b;
    while (ci > bks) {
      // window: from the first block boundary within kReoWin rows of the
      // block's end down to the block's end
      int ti = ci, tpos = pos;
      while (ti > bks && (pos + bs) - (tpos - sz[ti - 1]) <= kReoWin) tpos -= sz[--ti];
      const int wk = pos + bs - tpos;
      k_reorder_win<<<1, kReoThreads, reo_smem(wk), st>>>(S, lds, T, ldt, tpos, wk, pos - tpos, bs, tol, U, V,
                                                          status);
      UpdBatch L, R;
      L.njobs = 0;
      R.njobs = 0;
      add_job(L, S, lds, tpos, tpos + wk, n - (tpos + wk), U, wk);
      add_job(L, T, ldt, tpos, tpos + wk, n - (tpos + wk), U, wk);
      add_job(R, S, lds, 0, tpos, tpos, V, wk);
      add_job(R, T, ldt, 0, tpos, tpos, V, wk);
      if (wantq) add_job(R, Q, ldq, 0, tpos, n, U, wk);
      if (wantz) add_job(R, Z, ldz, 0, tpos, n, V, wk);
      if (L.njobs) launch_update(st, L, 0);
      if (R.njobs) launch_update(st, R, 1);
      e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      out->windows += 1;
      out->swaps += ci - ti;
      // the block now leads the window
      for (int k = ci; k > ti; --k) {
        std::swap(sz[k], sz[k - 1]);
        std::swap(sel[k], sel[k - 1]);
      }
      ci = ti;
      pos = tpos;
    }
    int hs[2] = {0, 0};
    e = cudaMemcpyAsync(hs, status, sizeof(hs), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    if (hs[0]) {
      out->info = 1;
      break;
    }
    ks += bs;
    ++bks;
  }
  k_tgsen_signs<<<n, 256, 0, st>>>(S, lds, T, ldt, Q, ldq, n, wantq ? 1 : 0);
  k_tgsen_eigs<<<(n + 255) / 256, 256, 0, st>>>(S, lds, T, ldt, n, alphar, alphai, beta);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (out->info) {
    out->pl = out->pr = 0.0;
    return cudaStreamSynchronize(st);
  }
  const int m1 = out->m, m2 = n - out->m;
  if ((ijob == 1 || ijob == 5) && m1 > 0 && m2 > 0) {
    // diagonal blocks of S11 and S22 (the selected blocks lead)
    std::vector<int> blk(2 * (size_t)nb);
    int nb1 = 0, nb2 = 0;
    for (int k = 0, p = 0; k < nb; p += sz[k], ++k) {
      if (p < m1) { blk[nb1] = p; blk[nb + nb1] = sz[k]; ++nb1; }
    }
    std::vector<int> b2(2 * (size_t)nb);
    for (int k = 0, p = 0; k < nb; p += sz[k], ++k) {
      if (p >= m1) { b2[nb2] = p - m1; b2[nb + nb2] = sz[k]; ++nb2; }
    }
    DevMem sm;
    const size_t nd = 2 * (size_t)m1 * m1 + 2 * (size_t)m1 * m2 + kSsqBlocks + 2;
    e = cudaMalloc(&sm.p, nd * sizeof(double) + 4 * (size_t)nb * sizeof(int));
    if (e != cudaSuccess) return e;
    double* S11t = (double*)sm.p;
    double* T11t = S11t + (size_t)m1 * m1;
    double* Rm = T11t + (size_t)m1 * m1;
    double* Lt = Rm + (size_t)m1 * m2;
    double* part = Lt + (size_t)m1 * m2;
    double* nrm = part + kSsqBlocks;
    int* dblk = (int*)(nrm + 2);
    std::vector<int> hb(4 * (size_t)nb, 0);
    for (int k = 0; k < nb1; ++k) { hb[k] = blk[k]; hb[nb + k] = blk[nb + k]; }
    for (int k = 0; k < nb2; ++k) { hb[2 * nb + k] = b2[k]; hb[3 * nb + k] = b2[nb + k]; }
    e = cudaMemcpyAsync(dblk, hb.data(), sizeof(int) * 4 * (size_t)nb, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    const dim3 tg((m1 + 31) / 32, (m1 + 31) / 32), tb(32, 8);
    k_transpose_lead<<<tg, tb, 0, st>>>(S, lds, m1, S11t);
    k_transpose_lead<<<tg, tb, 0, st>>>(T, ldt, m1, T11t);
    SylvArgs a{S, T, lds, ldt, m1, m2, S11t, T11t, Rm, Lt, dblk, dblk + nb, dblk + 2 * nb, dblk + 3 * nb, nb1, nb2};
    for (int d = 0; d < nb1 + nb2 - 1; ++d) {
      const int jlo = d - (nb1 - 1) > 0 ? d - (nb1 - 1) : 0;
      const int jhi = d < nb2 - 1 ? d : nb2 - 1;
      const int pairs = jhi - jlo + 1;
      k_sylv_wave<<<(pairs + 7) / 8, 256, 0, st>>>(a, d);
    }
    k_ssq_part<<<kSsqBlocks, 256, 0, st>>>(Rm, (int64_t)m1 * m2, part);
    k_ssq_final<<<1, 32, 0, st>>>(part, kSsqBlocks, nrm);
    k_ssq_part<<<kSsqBlocks, 256, 0, st>>>(Lt, (int64_t)m1 * m2, part);
    k_ssq_final<<<1, 32, 0, st>>>(part, kSsqBlocks, nrm + 1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    double hn[2];
    e = cudaMemcpyAsync(hn, nrm, sizeof(hn), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    out->pl = 1.0 / sqrt(1.0 + hn[0]);
    out->pr = 1.0 / sqrt(1.0 + hn[1]);
  }
  if (ijob == 3 || ijob == 5) {
    if (m1 == 0 || m2 == 0) {
      // nothing to separate: both estimates are ||(S, T)||_F, as DTGSEN sets them
      DevMem nm;
      e = cudaMalloc(&nm.p, (592 + 2) * sizeof(double));
      if (e != cudaSuccess) return e;
      double* part = (double*)nm.p;
      launch_sumsq(st, S, lds, 0, n, part + 592, part);
      launch_sumsq(st, T, ldt, 0, n, part + 593, part);
      double hn[2];
      e = cudaMemcpyAsync(hn, part + 592, sizeof(hn), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return e;
      out->dif[0] = out->dif[1] = sqrt(hn[0] + hn[1]);
    } else {
      std::vector<int> b1s, b1z, b2s, b2z;
      for (int k = 0, p = 0; k < nb; p += sz[k], ++k) {
        if (p < m1) { b1s.push_back(p); b1z.push_back(sz[k]); }
        else { b2s.push_back(p - m1); b2z.push_back(sz[k]); }
      }
      e = dif_estimates(st, S, lds, T, ldt, m1, m2, b1s, b1z, b2s, b2z, out->dif);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaStreamSynchronize(st);
}

}  // namespace qz
