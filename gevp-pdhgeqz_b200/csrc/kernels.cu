// sm_100a kernels of the multishift QZ path.
//
//   k_aed_win     one CTA: window Schur form + spike test + reordering +
//                 re-reduction (AED, PDHGEQZ2/QZEARLY) or a full small
//                 solve (endgame, PDHGEQZ4/KKQZ) with the window in smem
//   k_chase_win   one CTA: a chain of bulges through one window (PDHGEQZ5/
//                 A/B, DHGEQZ5) accumulating U, V in smem
//   k_inf_win     one CTA: zero chasing of an infinite eigenvalue through a
//                 window (PDHGEQZ7/8, DHGEQZ7)
//   k_update_*    in-place off-diagonal updates on DMMA (PDHGEQZ6)
//   k_scan        deflation search (PDLASMSUB) + zero T-diagonal detection
//   k_inf_top     top deflation of an infinite eigenvalue (one rotation)
//   k_signs, k_eigs   sign normalisation (beta >= 0) and alpha/beta output
#include <cuda_runtime.h>
#include <stdint.h>

#define QZ_DEFINE_UPDATE_KERNELS
#include "qz_window.cuh"
#include "update.cuh"
#include "kernels.h"

namespace qz {

// Executor of the CTA-level algorithms.  With kWarp the CTA is one warp and
// the barrier is __syncwarp (also a shared-memory fence for the warp).
template <bool kWarp>
struct DevExecT {
  int tid, nt;
  int* si;
  double* sd;
  unsigned long long* ts = nullptr;  // phase timestamps (ns), thread 0 writes
  PipeBuf* pipe = nullptr;            // pipelined double-shift sweeps (shared memory)
  __device__ void sync() {
    if constexpr (kWarp) __syncwarp();
    else __syncthreads();
  }
  __device__ void stamp(int k) {
    if (ts && tid == 0) {
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      ts[k] = t;
    }
  }
  // event counters (profiling, ts has 16 slots): 0 double-shift steps, 1
  // block swaps, 2 re-reduction rotation pairs, 3 multishift window sweeps
  __device__ void count(int k) {
    if (ts && tid == 0) ts[5 + k] += 1;
  }
};

using DevExec = DevExecT<false>;

// shared-memory scratch carved at the end of the dynamic smem block
constexpr int kSi = 64;

__device__ __forceinline__ double& G(double* p, int64_t ld, int i, int j) { return p[i + (int64_t)j * ld]; }

// ---------------------------------------------------------------------------
// AED / small-solve window kernel
// ---------------------------------------------------------------------------
template <int kThreads>
__global__ void __launch_bounds__(kThreads) k_aed_win(double* H, double* T, int64_t ld, int ktop, int kwtop,
                                                         int nw, Tol tol, double* Qw, double* Zw, double* shifts,
                                                         int* info, double* gscratch, int maxit,
                                                         unsigned long long* ts, int nskip, int swapfail, int ms) {
  extern __shared__ double smem[];
  const int n = nw;
  const bool in_smem = n <= kWinSmemMax;
  // odd leading dimension in shared memory: row accesses hit distinct banks
  const int lw = in_smem ? smem_ld(n) : n;
  double* Hs;
  double* Ts;
  double* Qs;
  double* Zs;
  double* sd;
  if (in_smem) {
    Hs = smem;
    Ts = Hs + n * lw;
    Qs = Ts + n * lw;
    Zs = Qs + n * lw;
    sd = Zs + n * lw;
  } else {
    Hs = gscratch;
    Ts = gscratch + (int64_t)n * n;
    Qs = Qw;
    Zs = Zw;
    sd = smem;
  }
  // sd: 64 doubles of swap/spike scalars, 4n of spike vectors, the
  // multishift window QZ's scratch, then the sweep pipeline's buffer
  int* si = (int*)(sd + 64 + 4 * n + kMsScratch + kPipeDoubles);
  DevExecT<kThreads == 32> x{(int)threadIdx.x, kThreads, si, sd, ts};
  if (kThreads >= 64) x.pipe = (PipeBuf*)(sd + 64 + 4 * n + kMsScratch);
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    int i = idx % n, j = idx / n;
    Hs[i + j * lw] = G(H, ld, kwtop + i, kwtop + j);
    Ts[i + j * lw] = G(T, ld, kwtop + i, kwtop + j);
    Qs[i + j * lw] = (i == j) ? 1.0 : 0.0;
    Zs[i + j * lw] = (i == j) ? 1.0 : 0.0;
  }
  double s = (kwtop > ktop) ? G(H, ld, kwtop, kwtop - 1) : 0.0;
  __syncthreads();
  WinState w;
  w.n = n;
  w.H = MatV{Hs, lw};
  w.T = MatV{Ts, lw};
  w.Q = MatV{Qs, lw};
  w.Z = MatV{Zs, lw};
  w.wantq = true;
  w.wantz = true;
  w.tol = tol;
  cta_aed(x, w, s, shifts, shifts + n, shifts + 2 * n, maxit, nskip, swapfail != 0, ms ? sd + 64 + 4 * n : nullptr);
  __syncthreads();
  const int m = si[8], st = si[9], tr = si[10];
  if (st == 0 && tr) {
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
      int i = idx % n, j = idx / n;
      G(H, ld, kwtop + i, kwtop + j) = Hs[i + j * lw];
      G(T, ld, kwtop + i, kwtop + j) = Ts[i + j * lw];
      if (in_smem) {
        Qw[idx] = Qs[i + j * lw];
        Zw[idx] = Zs[i + j * lw];
      }
    }
    if (threadIdx.x == 0 && kwtop > ktop) G(H, ld, kwtop, kwtop - 1) = s * Qs[0];
  }
  if (threadIdx.x == 0) {
    info[0] = m;
    info[1] = st;
    info[2] = tr;
  }
}

// ---------------------------------------------------------------------------
// chase kernel
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kChaseThreads) k_chase_win(double* H, double* T, int64_t ld, const ChaseWave wave,
                                                             double* Ug, double* Vg, int64_t ustride) {
  extern __shared__ double smem[];
  const ChaseJob& J = wave.job[blockIdx.x];
  const int w0 = J.w0, wk = J.wk, last = J.last, nb = J.nb, tmax = J.tmax;
  double* U = Ug + blockIdx.x * ustride;
  double* V = Vg + blockIdx.x * ustride;
  const int lw = smem_ld(wk);
  double* Hs = smem;
  double* Ts = Hs + wk * lw;
  double* Us = Ts + wk * lw;
  double* Vs = Us + wk * lw;
  Bulge* bl = (Bulge*)(Vs + wk * lw);
  BulgeRec* rec = (BulgeRec*)(bl + kMaxChain);
  int* si = (int*)(rec + kMaxChain);
  DevExec x{(int)threadIdx.x, (int)blockDim.x, si, nullptr};
  for (int idx = threadIdx.x; idx < wk * wk; idx += blockDim.x) {
    int i = idx % wk, j = idx / wk;
    Hs[i + j * lw] = G(H, ld, w0 + i, w0 + j);
    Ts[i + j * lw] = G(T, ld, w0 + i, w0 + j);
    Us[i + j * lw] = (i == j) ? 1.0 : 0.0;
    Vs[i + j * lw] = (i == j) ? 1.0 : 0.0;
  }
  for (int b = threadIdx.x; b < nb; b += blockDim.x) bl[b] = J.bl[b];
  __syncthreads();
  cta_chase_window(x, wk, last, MatV{Hs, lw}, MatV{Ts, lw}, MatV{Us, lw}, MatV{Vs, lw}, bl, nb, tmax, rec);
  __syncthreads();
  for (int idx = threadIdx.x; idx < wk * wk; idx += blockDim.x) {
    int i = idx % wk, j = idx / wk;
    G(H, ld, w0 + i, w0 + j) = Hs[i + j * lw];
    G(T, ld, w0 + i, w0 + j) = Ts[i + j * lw];
    U[idx] = Us[i + j * lw];
    V[idx] = Vs[i + j * lw];
  }
}

// ---------------------------------------------------------------------------
// infinite-eigenvalue zero chase through a window
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kWinThreads) k_inf_win(double* H, double* T, int64_t ld, int w0, int wk, int top,
                                                         int jz, int stop, int deflate, double* U, double* V) {
  extern __shared__ double smem[];
  const int lw = smem_ld(wk);
  double* Hs = smem;
  double* Ts = Hs + wk * lw;
  double* Us = Ts + wk * lw;
  double* Vs = Us + wk * lw;
  int* si = (int*)(Vs + wk * lw);
  DevExec x{(int)threadIdx.x, (int)blockDim.x, si, nullptr};
  for (int idx = threadIdx.x; idx < wk * wk; idx += blockDim.x) {
    int i = idx % wk, j = idx / wk;
    Hs[i + j * lw] = G(H, ld, w0 + i, w0 + j);
    Ts[i + j * lw] = G(T, ld, w0 + i, w0 + j);
    Us[i + j * lw] = (i == j) ? 1.0 : 0.0;
    Vs[i + j * lw] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  cta_inf_window(x, wk, top, jz, stop, deflate != 0, MatV{Hs, lw}, MatV{Ts, lw}, MatV{Us, lw}, MatV{Vs, lw});
  __syncthreads();
  for (int idx = threadIdx.x; idx < wk * wk; idx += blockDim.x) {
    int i = idx % wk, j = idx / wk;
    G(H, ld, w0 + i, w0 + j) = Hs[i + j * lw];
    G(T, ld, w0 + i, w0 + j) = Ts[i + j * lw];
    U[idx] = Us[i + j * lw];
    V[idx] = Vs[i + j * lw];
  }
}

// ---------------------------------------------------------------------------
// deflation scan: ktop = largest k in (ifirst, kbot] with negligible
// H(k,k-1) (zeroed), then zero T-diagonal entries in [ktop, kbot].
// out = {ktop, ninf, jmax, jmin, nonfinite}
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_scan(double* H, double* T, int64_t ld, int ifirst, int kbot, Tol tol,
                                               int* out) {
  __shared__ int s_best;
  __shared__ int s_cnt, s_jmax, s_jmin, s_bad;
  if (threadIdx.x == 0) { s_best = -1; s_cnt = 0; s_jmax = -1; s_jmin = 0x7fffffff; s_bad = 0; }
  __syncthreads();
  // numerical breakdown guard: a non-finite entry on the diagonals of the
  // active block is reported instead of being iterated on
  for (int j = ifirst + (int)threadIdx.x; j <= kbot; j += blockDim.x) {
    double a = G(H, ld, j, j), b = G(T, ld, j, j), c = (j > ifirst) ? G(H, ld, j, j - 1) : 0.0;
    if (!isfinite(a) || !isfinite(b) || !isfinite(c)) s_bad = 1;
  }
  __syncthreads();
  for (int base = kbot; base > ifirst; base -= blockDim.x) {
    int k = base - (int)threadIdx.x;
    if (k > ifirst) {
      if (negligible_sub(G(H, ld, k, k - 1), G(H, ld, k - 1, k - 1), G(H, ld, k, k), tol)) atomicMax(&s_best, k);
    }
    __syncthreads();
    if (s_best >= 0) break;
    __syncthreads();
  }
  int ktop = (s_best >= 0) ? s_best : ifirst;
  __syncthreads();
  if (threadIdx.x == 0 && ktop > ifirst) G(H, ld, ktop, ktop - 1) = 0.0;
  for (int j = ktop + (int)threadIdx.x; j <= kbot; j += blockDim.x) {
    double t = G(T, ld, j, j);
    if (fabs(t) <= tol.ttol) {
      G(T, ld, j, j) = 0.0;
      atomicAdd(&s_cnt, 1);
      atomicMax(&s_jmax, j);
      atomicMin(&s_jmin, j);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    out[0] = ktop;
    out[1] = s_cnt;
    out[2] = s_jmax;
    out[3] = (s_cnt > 0) ? s_jmin : -1;
    out[4] = s_bad;
  }
}

// top deflation: T(f,f) = 0; rotation of rows f, f+1 zeroing H(f+1,f)
__global__ void __launch_bounds__(1024) k_inf_top(double* H, double* T, double* Q, int64_t ld, int n, int f, int wantq) {
  double c, s, r;
  lartg(G(H, ld, f, f), G(H, ld, f + 1, f), c, s, r);
  __syncthreads();
  for (int j = f + 1 + (int)threadIdx.x; j < n; j += blockDim.x) {
    double a = G(H, ld, f, j), b = G(H, ld, f + 1, j);
    G(H, ld, f, j) = c * a + s * b;
    G(H, ld, f + 1, j) = -s * a + c * b;
    a = G(T, ld, f, j); b = G(T, ld, f + 1, j);
    G(T, ld, f, j) = c * a + s * b;
    G(T, ld, f + 1, j) = -s * a + c * b;
  }
  if (wantq)
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double a = G(Q, ld, i, f), b = G(Q, ld, i, f + 1);
      G(Q, ld, i, f) = c * a + s * b;
      G(Q, ld, i, f + 1) = -s * a + c * b;
    }
  if (threadIdx.x == 0) { G(H, ld, f, f) = r; G(H, ld, f + 1, f) = 0.0; }
}

// ---------------------------------------------------------------------------
// finalisation
// ---------------------------------------------------------------------------
// 1x1 blocks with T(j,j) < 0: negate column j of H, T (rows 0..j) and Z
__global__ void k_signs(double* H, double* T, double* Z, int64_t ld, int n, int wantz) {
  int j = blockIdx.x;
  bool below = (j + 1 < n) && G(H, ld, j + 1, j) != 0.0;
  bool above = (j > 0) && G(H, ld, j, j - 1) != 0.0;
  if (below || above) return;
  if (!(G(T, ld, j, j) < 0.0)) return;
  __syncthreads();
  for (int i = threadIdx.x; i <= j; i += blockDim.x) {
    G(H, ld, i, j) = -G(H, ld, i, j);
    G(T, ld, i, j) = -G(T, ld, i, j);
  }
  if (wantz)
    for (int i = threadIdx.x; i < n; i += blockDim.x) G(Z, ld, i, j) = -G(Z, ld, i, j);
}

__global__ void k_eigs(const double* H, const double* T, int64_t ld, int n, double* ar, double* ai, double* be) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  bool below = (j + 1 < n) && G((double*)H, ld, j + 1, j) != 0.0;
  bool above = (j > 0) && G((double*)H, ld, j, j - 1) != 0.0;
  if (!below && !above) {
    ar[j] = G((double*)H, ld, j, j);
    ai[j] = 0.0;
    be[j] = G((double*)T, ld, j, j);
    return;
  }
  int f = below ? j : j - 1;
  double a[4] = {G((double*)H, ld, f, f), G((double*)H, ld, f + 1, f), G((double*)H, ld, f, f + 1),
                 G((double*)H, ld, f + 1, f + 1)};
  double o_ar[2], o_ai[2], o_be[2];
  eig2_complex(a, G((double*)T, ld, f, f), G((double*)T, ld, f + 1, f + 1), o_ar, o_ai, o_be);
  int e = j - f;
  ar[j] = e ? o_ar[1] : o_ar[0];  // selects keep the pair in registers
  ai[j] = e ? o_ai[1] : o_ai[0];
  be[j] = e ? o_be[1] : o_be[0];
}

__global__ void k_set_identity(double* Q, int64_t ld, int n) {
  int64_t total = (int64_t)n * n;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(idx % n), j = (int)(idx / n);
    G(Q, ld, i, j) = (i == j) ? 1.0 : 0.0;
  }
}

// sum of squares of the n x n block at (o, o)
// Sum of squares in a fixed order: each block writes its partial sum, then
// one warp adds the partials in block order (no floating-point atomics, so
// the tolerances derived from the norms are identical from run to run).
constexpr int kSumsqBlocks = 592;
__global__ void k_sumsq(const double* A, int64_t ld, int o, int n, double* partial) {
  double acc = 0.0;
  int64_t total = (int64_t)n * n;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(idx % n), j = (int)(idx / n);
    double v = A[(o + i) + (int64_t)(o + j) * ld];
    acc += v * v;
  }
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  __shared__ double red[32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = acc;
  __syncthreads();
  if (wid == 0) {
    acc = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) partial[blockIdx.x] = acc;
  }
}

__global__ void k_sumsq_final(const double* partial, int np, double* out) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < np; i += 32) acc += partial[i];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if (threadIdx.x == 0) out[0] = acc;
}

// largest absolute entry, same two-stage fixed-order reduction
__global__ void k_maxabs(const double* A, int64_t ld, int o, int n, double* partial) {
  double m = 0.0;
  int64_t total = (int64_t)n * n;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(idx % n), j = (int)(idx / n);
    m = fmax(m, fabs(A[(o + i) + (int64_t)(o + j) * ld]));
  }
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
  __shared__ double red[32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = m;
  __syncthreads();
  if (wid == 0) {
    m = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    if (lane == 0) partial[blockIdx.x] = m;
  }
}

__global__ void k_max_final(const double* partial, int np, double* out) {
  double m = 0.0;
  for (int i = threadIdx.x; i < np; i += 32) m = fmax(m, partial[i]);
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
  if (threadIdx.x == 0) out[0] = m;
}

// A(0:n, 0:n) <- 2^e A (exact unless the result leaves the normal range)
__global__ void k_scale_pow2(double* A, int64_t ld, int n, int e) {
  int64_t total = (int64_t)n * n;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(idx % n), j = (int)(idx / n);
    double& a = A[i + (int64_t)j * ld];
    a = ldexp(a, e);
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
size_t aed_smem_bytes(int nw) {
  size_t d = (nw <= kWinSmemMax) ? (size_t)4 * nw * smem_ld(nw) : 0;
  d += 64 + 4 * (size_t)nw + kMsScratch + kPipeDoubles;
  return d * sizeof(double) + kSi * sizeof(int);
}
size_t chase_smem_bytes(int wk) {
  return (size_t)4 * wk * smem_ld(wk) * sizeof(double) + kMaxChain * (sizeof(Bulge) + sizeof(BulgeRec)) +
         kSi * sizeof(int);
}
size_t inf_smem_bytes(int wk) { return (size_t)4 * wk * smem_ld(wk) * sizeof(double) + kSi * sizeof(int); }

static size_t upd_smem(int k, int side) {
  int kp = (k + 15) & ~15;
  if (k > kUpdMaxK) return (size_t)k * kUpdGenTile * sizeof(double);
  if (side == 0) return ((size_t)kp * (kp + 4) + (size_t)kp * 36) * sizeof(double);
  return ((size_t)kp * (kp + 4) + (size_t)32 * (kp + 4)) * sizeof(double);
}

static size_t upd_smem_persist(int k, int side) {
  int kp = (k + 15) & ~15;
  if (side == 0) return ((size_t)kp * (kp + 4) + 2 * (size_t)kp * 36) * sizeof(double);
  return ((size_t)kp * (kp + 4) + 2 * (size_t)kUpdTile * (kp + 4)) * sizeof(double);
}

static int g_sm_count = 0;

cudaError_t kernels_init() {
  cudaError_t e;
  e = cudaFuncSetAttribute(k_aed_win<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)aed_smem_bytes(kWinSmemMax));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_aed_win<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)aed_smem_bytes(kWinSmemMax));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_aed_win<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)aed_smem_bytes(kWinSmemMax));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_chase_win, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)chase_smem_bytes(kWinSmemMax));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_inf_win, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)inf_smem_bytes(kWinSmemMax));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_update_left, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)upd_smem(kUpdMaxK, 0));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_update_right, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)upd_smem(kUpdMaxK, 1));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_update_persist<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)upd_smem_persist(kUpdMaxK, 0));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_update_persist<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)upd_smem_persist(kUpdMaxK, 1));
  if (e != cudaSuccess) return e;
  {
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
  }
  e = cudaFuncSetAttribute(k_update_left_gen, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_update_right_gen, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  return e;
}

void launch_aed(cudaStream_t st, double* H, double* T, int64_t ld, int ktop, int kwtop, int nw, const Tol& tol,
                double* Qw, double* Zw, double* shifts, int* info, double* gscratch, unsigned long long* ts, int nskip,
                int threads, int swapfail, int ms) {
  const size_t sm = aed_smem_bytes(nw);
  if (threads <= 32)
    k_aed_win<32><<<1, 32, sm, st>>>(H, T, ld, ktop, kwtop, nw, tol, Qw, Zw, shifts, info, gscratch, 30 * nw, ts, nskip,
                                     swapfail, ms);
  else if (threads <= 64)
    k_aed_win<64><<<1, 64, sm, st>>>(H, T, ld, ktop, kwtop, nw, tol, Qw, Zw, shifts, info, gscratch, 30 * nw, ts, nskip,
                                     swapfail, ms);
  else
    k_aed_win<128><<<1, 128, sm, st>>>(H, T, ld, ktop, kwtop, nw, tol, Qw, Zw, shifts, info, gscratch, 30 * nw, ts,
                                       nskip, swapfail, ms);
}
void launch_chase_wave(cudaStream_t st, double* H, double* T, int64_t ld, const ChaseWave& wave, int njob, double* U,
                       double* V, int64_t ustride) {
  if (njob <= 0) return;
  int wmax = 0;
  for (int i = 0; i < njob; ++i) wmax = wave.job[i].wk > wmax ? wave.job[i].wk : wmax;
  k_chase_win<<<njob, kChaseThreads, chase_smem_bytes(wmax), st>>>(H, T, ld, wave, U, V, ustride);
}
void launch_inf(cudaStream_t st, double* H, double* T, int64_t ld, int w0, int wk, int top, int jz, int stop,
                int deflate, double* U, double* V) {
  k_inf_win<<<1, kWinThreads, inf_smem_bytes(wk), st>>>(H, T, ld, w0, wk, top, jz, stop, deflate, U, V);
}
void launch_scan(cudaStream_t st, double* H, double* T, int64_t ld, int ifirst, int kbot, const Tol& tol, int* out) {
  k_scan<<<1, 1024, 0, st>>>(H, T, ld, ifirst, kbot, tol, out);
}
void launch_inf_top(cudaStream_t st, double* H, double* T, double* Q, int64_t ld, int n, int f, int wantq) {
  k_inf_top<<<1, 1024, 0, st>>>(H, T, Q, ld, n, f, wantq);
}
void launch_update(cudaStream_t st, const UpdBatch& B_in, int side, int persist) {
  UpdBatch B = B_in;
  int tiles = 0;
  B.k = 0;
  for (int j = 0; j < B.njobs; ++j) {
    tiles += B.job[j].tiles;
    if (B.job[j].k > B.k) B.k = B.job[j].k;
  }
  if (tiles == 0) return;
  if (B.k > kUpdMaxK) {
    if (side == 0) k_update_left_gen<<<tiles, 256, upd_smem(B.k, 0), st>>>(B);
    else k_update_right_gen<<<tiles, 256, upd_smem(B.k, 1), st>>>(B);
  } else if (persist) {
    const size_t sm = upd_smem_persist(B.k, side);
    int per_sm = (int)((220 * 1024) / sm);
    per_sm = per_sm < 1 ? 1 : (per_sm > 4 ? 4 : per_sm);
    int grid = (g_sm_count > 0 ? g_sm_count : 148) * per_sm;
    if (grid > tiles) grid = tiles;
    // one warp per 16-row (left) / 16-column (right) slice of the largest window
    int warps = ((B.k + 15) & ~15) / 16;
    warps = warps < 1 ? 1 : (warps > kUpdMaxThreads / 32 ? kUpdMaxThreads / 32 : warps);
    if (side == 0) k_update_persist<0><<<grid, 32 * warps, sm, st>>>(B, tiles);
    else k_update_persist<1><<<grid, 32 * warps, sm, st>>>(B, tiles);
  } else {
    if (side == 0) k_update_left<<<tiles, kUpdThreads, upd_smem(B.k, 0), st>>>(B);
    else k_update_right<<<tiles, kUpdThreads, upd_smem(B.k, 1), st>>>(B);
  }
}
int update_tile(int k) { return k > kUpdMaxK ? kUpdGenTile : kUpdTile; }
void launch_finalize(cudaStream_t st, double* H, double* T, double* Z, int64_t ld, int n, int wantz, double* ar,
                     double* ai, double* be) {
  if (n <= 0) return;
  k_signs<<<n, 256, 0, st>>>(H, T, Z, ld, n, wantz);
  k_eigs<<<(n + 255) / 256, 256, 0, st>>>(H, T, ld, n, ar, ai, be);
}
void launch_eigs(cudaStream_t st, const double* H, const double* T, int64_t ld, int n, double* ar, double* ai,
                 double* be) {
  if (n > 0) k_eigs<<<(n + 255) / 256, 256, 0, st>>>(H, T, ld, n, ar, ai, be);
}
void launch_identity(cudaStream_t st, double* Q, int64_t ld, int n) {
  k_set_identity<<<592, 256, 0, st>>>(Q, ld, n);
}
void launch_maxabs(cudaStream_t st, const double* A, int64_t ld, int o, int n, double* out, double* partial) {
  k_maxabs<<<kSumsqBlocks, 256, 0, st>>>(A, ld, o, n, partial);
  k_max_final<<<1, 32, 0, st>>>(partial, kSumsqBlocks, out);
}
void launch_scale_pow2(cudaStream_t st, double* A, int64_t ld, int n, int e) {
  if (n > 0 && e != 0) k_scale_pow2<<<592, 256, 0, st>>>(A, ld, n, e);
}
void launch_sumsq(cudaStream_t st, const double* A, int64_t ld, int o, int n, double* out, double* partial) {
  k_sumsq<<<kSumsqBlocks, 256, 0, st>>>(A, ld, o, n, partial);
  k_sumsq_final<<<1, 32, 0, st>>>(partial, kSumsqBlocks, out);
}

}  // namespace qz
