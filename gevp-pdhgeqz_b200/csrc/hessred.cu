// Hessenberg-triangular reduction on the device: the launch sequence of
// the windowed Givens form in hessred.cuh.
//
// Per column jc: one launch per window, from the bottom of the column up.
// CTA 0 first applies the previous window's Z rotations to the rows of B
// its own diagonal block holds (walk (a)), then loads the block and runs
// the chain; the other CTAs of the launch apply the previous window's
// rotations elsewhere (walks (e), (f), (g)), on entries CTA 0 does not
// touch (a thread per walk: these CTAs carry the block's shared memory, so
// one fits per SM).  After the column's last window, one launch applies
// that window's walks and one applies the column's G rotations to A
// (columns jc+1..n-1) and both factors to Q and Z, a warp per walk (32
// rotations per affine scan of the carried value).  The rotations of a
// column are kept in a 4n-double array indexed by pair.
//
// Bounds: the chain is a dependent sequence of two rotations per pair on
// one SM (about n^2/2 pairs); the walks stream each touched entry once per
// window (read + write), about (2 (n-jc)^2 + 3 n (n-jc)) * 16 bytes per
// column.
#include "hessred.h"

#include <algorithm>

#include "hessred.cuh"
#include "kernels.h"

namespace qz {
namespace {

constexpr int kHrChain = 128;               // chain threads: 96 far threads and the block thread's warp
constexpr int kHrThreads = kHrChain + 32;   // plus the producer's warp
constexpr int kHrSpin = 1 << 22;            // polls before a wait gives up

// The chain threads: a named barrier over them (the producer warp is not
// in it) and a bounded wait on the producer's count.
struct HrChainExec {
  int tid, nt;
  int* err;
  __device__ void sync() { asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory"); }
  __device__ bool wait(const int* p, int v) {
    for (int it = 0; it < kHrSpin; ++it)
      if (hr_ld_acq(p) >= v) return true;
    atomicExch(err, 1);
    return false;
  }
};

__device__ void cp_async8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__global__ void __launch_bounds__(kHrThreads) k_hr_zero_lower(double* B, int64_t ldb, int n) {
  const int64_t total = (int64_t)n * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(i % n), c = (int)(i / n);
    if (r > c) B[r + c * ldb] = 0.0;
  }
}

// Warp walks: the 32 lanes take 32 consecutive rotations of a walk at once.
// The carried value follows a first-order linear recurrence, carry ->
// a carry + b per rotation, so the carries of the 32 steps come from one
// warp scan of the affine maps (five shuffle rounds) instead of 32
// dependent steps, and the 32 loads of a chunk are in flight together.
// The results differ from the one-thread walks only by rounding.
constexpr unsigned kFull = 0xffffffffu;

__device__ void affine_scan(double& a, double& b, int lane) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double ap = __shfl_up_sync(kFull, a, off), bp = __shfl_up_sync(kFull, b, off);
    if (lane >= off) {
      b = a * bp + b;
      a = a * ap;
    }
  }
}

// hr_walk_g by a warp: entries (J-1, J), carry = entry J side.
__device__ void hr_wwalk_g(double* v, int64_t st, int Jhi, int Jlo, const double* rot, int lane) {
  double y = v[(int64_t)Jhi * st];
  for (int J0 = Jhi; J0 >= Jlo; J0 -= 32) {
    const int J = J0 - lane;
    const bool act = J >= Jlo;
    double x = 0.0, c = 1.0, s = 0.0;
    if (act) {
      x = v[(int64_t)(J - 1) * st];
      c = rot[4 * J];
      s = rot[4 * J + 1];
    }
    double a = act ? s : 1.0, b = act ? c * x : 0.0;
    affine_scan(a, b, lane);
    const double ynew = a * y + b;
    double yprev = __shfl_up_sync(kFull, ynew, 1);
    if (lane == 0) yprev = y;
    if (act) v[(int64_t)J * st] = -s * x + c * yprev;
    y = __shfl_sync(kFull, ynew, 31);
  }
  if (lane == 0) v[(int64_t)(Jlo - 1) * st] = y;
}

// hr_walk_z by a warp: columns (J, J-1), carry = column J side.
__device__ void hr_wwalk_z(double* row, int64_t st, int Jhi, int Jlo, const double* rot, int lane) {
  double x = row[(int64_t)Jhi * st];
  for (int J0 = Jhi; J0 >= Jlo; J0 -= 32) {
    const int J = J0 - lane;
    const bool act = J >= Jlo;
    double y = 0.0, cz = 1.0, sz = 0.0;
    if (act) {
      y = row[(int64_t)(J - 1) * st];
      cz = rot[4 * J + 2];
      sz = rot[4 * J + 3];
    }
    double a = act ? -sz : 1.0, b = act ? cz * y : 0.0;
    affine_scan(a, b, lane);
    const double xnew = a * x + b;
    double xprev = __shfl_up_sync(kFull, xnew, 1);
    if (lane == 0) xprev = x;
    if (act) row[(int64_t)J * st] = cz * xprev + sz * y;
    x = __shfl_sync(kFull, xnew, 31);
  }
  if (lane == 0) row[(int64_t)(Jlo - 1) * st] = x;
}

// hr_win_item / hr_col_item with a warp per item, for the launches without
// shared memory (the last window's walks and the column-end walks), where
// every walk can have its own warp resident.
__device__ void hr_win_item_w(const HrArgs& a, int i, int e_end, int plo, int phi, int lane) {
  const int nf = a.n - 1 - phi;
  if (i < e_end) hr_wwalk_z(a.B + i, a.ldb, phi, plo, a.rot, lane);
  else if (i < e_end + nf) hr_wwalk_g(a.B + (int64_t)(phi + 1 + i - e_end) * a.ldb, 1, phi, plo, a.rot, lane);
  else hr_wwalk_z(a.A + (i - e_end - nf), a.lda, phi, plo, a.rot, lane);
}
__device__ void hr_col_item_w(const HrArgs& a, int i, int jc, int lane) {
  const int na = a.n - 1 - jc, nq = a.wantq ? a.n : 0;
  if (i < na) {
    hr_wwalk_g(a.A + (int64_t)(jc + 1 + i) * a.lda, 1, a.ihi, jc + 2, a.rot, lane);
  } else if (i < na + nq) {
    const int r = i - na;
    if (a.qrows) hr_wwalk_g(a.Q + (int64_t)r * a.ldq, 1, a.ihi, jc + 2, a.rot, lane);
    else hr_wwalk_g(a.Q + r, a.ldq, a.ihi, jc + 2, a.rot, lane);
  } else {
    hr_wwalk_z(a.Z + (i - na - nq), a.ldz, a.ihi, jc + 2, a.rot, lane);
  }
}

// CTA 0 of a window launch: window (lo, hi) of column jc, previous window
// (plo, phi) of the column (plo < 0: none).
__device__ void hr_window_cta(const HrArgs& a, int jc, int lo, int hi, int plo, int phi, double* sm, int wmax) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int o = lo - 1, m = hi - lo + 2, ldw = hr_ldw(m);
  const HrSmem L = hr_layout(sm, wmax);
  if (plo >= 0) {
    // (a) the previous window's Z on rows lo-1..hi-1 of B, columns
    // hi..phi, staged in the block's buffer
    // (its rotation records staged too: every row walks all of them)
    const int mp = phi - hi + 1, rows = m - 1;
    double* S = L.Tw;
    for (int j = 0; j < mp; ++j)
      for (int i = tid; i < rows; i += nt) cp_async8(&S[i + j * ldw], a.B + (o + i) + (int64_t)(hi + j) * a.ldb);
    for (int i = 4 + tid; i < 4 * mp; i += nt) cp_async8(&L.gbuf[i], a.rot + 4 * hi + i);
    cp_async_wait_all();
    __syncthreads();
    for (int i = tid; i < rows; i += nt) hr_walk_z(S + i, ldw, phi - hi, plo - hi, L.gbuf);
    __syncthreads();
    for (int j = 0; j < mp; ++j)
      for (int i = tid; i < rows; i += nt) a.B[(o + i) + (int64_t)(hi + j) * a.ldb] = S[i + j * ldw];
    __syncthreads();
  }
  for (int j = 0; j < m; ++j) {
    const double* src = a.B + o + (int64_t)(o + j) * a.ldb;
    for (int i = tid; i < m; i += nt) {
      if (i <= j) cp_async8(&L.Tw[i + j * ldw], src + i);
      else L.Tw[i + j * ldw] = 0.0;
    }
  }
  for (int i = tid; i < m; i += nt) cp_async8(&L.acol[i], a.A + (o + i) + (int64_t)jc * a.lda);
  if (tid == 0) *L.gready = 0;
  cp_async_wait_all();
  __syncthreads();
  if (tid == kHrChain) {
    hr_g_chain(m, L.acol, L.gbuf, L.gready);
  } else if (tid < kHrChain) {
    HrChainExec x{tid, kHrChain, a.err};
    cta_hr_zchain(x, L.Tw, ldw, m, L.gbuf, L.gready, L.slot);
  }
  __syncthreads();
  for (int i = 4 + tid; i < 4 * m; i += nt) a.rot[4 * o + i] = L.gbuf[i];
  for (int j = 0; j < m; ++j)
    for (int i = tid; i <= j; i += nt) a.B[(o + i) + (int64_t)(o + j) * a.ldb] = L.Tw[i + j * ldw];
  for (int i = tid; i < m; i += nt) a.A[(o + i) + (int64_t)jc * a.lda] = L.acol[i];
}

// Window (lo, hi) of column jc; (plo, phi): the previous window of the
// column (plo < 0: none).  CTA 0 runs the window, the others the previous
// window's walks (e), (f), (g).
__global__ void __launch_bounds__(kHrThreads) k_hr_win(HrArgs a, int jc, int lo, int hi, int plo, int phi, int wmax) {
  extern __shared__ double sm[];
  if (blockIdx.x > 0) {
    // short walks (one window): a thread per walk keeps the most of them in
    // flight on CTAs that carry the window's shared memory
    const int e_end = lo - 1, items = hr_win_items(a, e_end, phi);
    for (int i = (blockIdx.x - 1) * blockDim.x + threadIdx.x; i < items; i += (gridDim.x - 1) * blockDim.x)
      hr_win_item(a, i, e_end, plo, phi);
    return;
  }
  hr_window_cta(a, jc, lo, hi, plo, phi, sm, wmax);
}

// The walks of column jc's last window (plo, phi): rows above it in B,
// columns right of it in B, rows of A.
__global__ void __launch_bounds__(kHrThreads) k_hr_flush(HrArgs a, int plo, int phi) {
  const int e_end = plo - 1, items = hr_win_items(a, e_end, phi), wpb = blockDim.x >> 5;
  for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < items; i += gridDim.x * wpb)
    hr_win_item_w(a, i, e_end, plo, phi, threadIdx.x & 31);
}

// Column jc's G on A (columns jc+1..n-1) and both factors on Q, Z.
__global__ void __launch_bounds__(kHrThreads) k_hr_colend(HrArgs a, int jc) {
  const int items = hr_col_items(a, jc), wpb = blockDim.x >> 5;
  for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < items; i += gridDim.x * wpb)
    hr_col_item_w(a, i, jc, threadIdx.x & 31);
}

int blocks_for(int items) { return std::max(1, (items + kHrThreads - 1) / kHrThreads); }
// a warp per walk item
int warp_blocks_for(int items) { return std::max(1, (items + kHrThreads / 32 - 1) / (kHrThreads / 32)); }

}  // namespace

cudaError_t gghrd_device(cudaStream_t st, int icompq, int icompz, bool qrows, int n, int ilo, int ihi, double* A,
                         int64_t lda, double* B, int64_t ldb, double* Q, int64_t ldq, double* Z, int64_t ldz, int wmax,
                         GghrdOut* out) {
  if (out) *out = GghrdOut{};
  if (icompq == 2) launch_identity(st, Q, ldq, n);
  if (icompz == 2) launch_identity(st, Z, ldz, n);
  if (n > 1) k_hr_zero_lower<<<std::min(1184, blocks_for(n * n)), kHrThreads, 0, st>>>(B, ldb, n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || n <= 1 || ihi - ilo < 2) return e;
  const int W = std::max(2, std::min(wmax, kHrMaxWin));
  const size_t smem = hr_smem_doubles(W) * sizeof(double);
  e = cudaFuncSetAttribute(k_hr_win, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  double* rot = nullptr;
  e = cudaMallocAsync(&rot, sizeof(double) * (4 * (size_t)n + 1), st);
  if (e != cudaSuccess) return e;
  int* err = (int*)(rot + 4 * (size_t)n);
  e = cudaMemsetAsync(err, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  HrArgs a{A, lda, B, ldb, Q, ldq, Z, ldz, rot, err, n, ihi, icompq != 0, icompz != 0, qrows};
  int64_t launches = 0, pairs = 0;
  for (int jc = ilo; jc <= ihi - 2 && e == cudaSuccess; ++jc) {
    int plo = -1, phi = -1;
    for (int hi = ihi; hi >= jc + 2;) {
      const int lo = hr_win_lo(jc, hi, W);
      const int helpers = plo >= 0 ? blocks_for(hr_win_items(a, lo - 1, phi)) : 0;
      k_hr_win<<<1 + helpers, kHrThreads, smem, st>>>(a, jc, lo, hi, plo, phi, W);
      ++launches;
      pairs += hi - lo + 1;
      plo = lo;
      phi = hi;
      hi = lo - 1;
    }
    k_hr_flush<<<warp_blocks_for(hr_win_items(a, plo - 1, phi)), kHrThreads, 0, st>>>(a, plo, phi);
    k_hr_colend<<<warp_blocks_for(hr_col_items(a, jc)), kHrThreads, 0, st>>>(a, jc);
    launches += 2;
    e = cudaGetLastError();
  }
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  const cudaError_t ef = cudaFreeAsync(rot, st);
  if (e == cudaSuccess) e = ef;
  if (e == cudaSuccess && herr != 0) e = cudaErrorLaunchTimeout;
  if (out) { out->launches = launches; out->pairs = pairs; }
  return e;
}

}  // namespace qz
