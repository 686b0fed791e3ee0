// In-place off-diagonal updates with a window's orthogonal factors.
//
// Role in the reference: PDHGEQZ6 on a 1x1 grid (PDHGEQZ6.f:276-380) and
// the identical PDGEMM updates after AED / small subproblems
// (PDHGEQZ0.f:776-864, PDHGEQZ3.f:1630-1726):
//   left :  M(r0:r0+k, c0:c0+L) <- W^T * M(r0:r0+k, c0:c0+L)
//   right:  M(r0:r0+L, c0:c0+k) <- M(r0:r0+L, c0:c0+k) * W
// with W the k x k factor U or V of one window (k = window size).
//
// B200 design: FP64 tensor cores through DMMA (mma.sync m8n8k4 .f64).
// One CTA owns a full-depth slab tile (all k rows of 32 columns for the
// left update, all k columns of 32 rows for the right update), stages it
// and W in shared memory, and writes the product back in place, so no
// temporary copy of the slab is needed and every slab element is read and
// written exactly once (16 bytes of HBM traffic per element).
#pragma once
#include <stdint.h>

namespace qz {

struct UpdJob {
  double* M;       // target matrix
  int64_t ld;      // its leading dimension
  int r0, c0;      // slab origin
  int len;         // slab extent along the non-k direction (L)
  const double* W; // k x k factor (column-major, ld = ldw)
  int ldw;
  int k;           // window size of this job
  int tiles;       // number of 32-wide tiles of this job
};

// one launch updates the slabs of several windows (a wave of chains)
constexpr int kUpdMaxJobs = 32;
struct UpdBatch {
  UpdJob job[kUpdMaxJobs];
  int njobs;
  int k;           // largest window size in the batch (sizes shared memory)
};

constexpr int kUpdTile = 32;       // slab tile width (columns for left, rows for right)
constexpr int kUpdThreads = 128;   // 4 warps (per-tile kernels)
constexpr int kUpdMaxThreads = 256;  // persistent kernels: one warp per 16-row slice, up to 8
constexpr int kUpdMaxK = 128;      // fast path limit

#ifdef QZ_DEFINE_UPDATE_KERNELS
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ int upd_find_job(const UpdBatch& B, int& tile) {
  int t = blockIdx.x;
  for (int j = 0; j < B.njobs; ++j) {
    if (t < B.job[j].tiles) { tile = t; return j; }
    t -= B.job[j].tiles;
  }
  tile = -1;
  return -1;
}

// ---------------------------------------------------------------------------
// left: out(k x 32) = W^T (k x k) * X (k x 32)
// smem: Wt[kp][kp+4] (Wt[i][kk] = W(kk,i)), Xs[kp][36]
// warps take 16-row slices; warp tile 16 x 32 = 2 x 4 mma tiles
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kUpdThreads) k_update_left(UpdBatch B) {
  extern __shared__ double smem[];
  int tile;
  int jb = upd_find_job(B, tile);
  if (jb < 0) return;
  const UpdJob J = B.job[jb];
  const int k = J.k;
  const int kp = (k + 15) & ~15;
  const int ldw = kp + 4;
  const int ldx = 36;
  double* Wt = smem;
  double* Xs = smem + kp * ldw;
  const int tid = threadIdx.x;
  const int c0 = J.c0 + tile * kUpdTile;
  const int ncol = min(kUpdTile, J.c0 + J.len - c0);
  // stage W^T
  for (int idx = tid; idx < kp * kp; idx += blockDim.x) {
    int kk = idx % kp, i = idx / kp;
    double v = (kk < k && i < k) ? J.W[kk + (int64_t)i * J.ldw] : 0.0;
    Wt[i * ldw + kk] = v;
  }
  // stage the slab tile
  for (int idx = tid; idx < kp * kUpdTile; idx += blockDim.x) {
    int kk = idx % kp, j = idx / kp;
    double v = (kk < k && j < ncol) ? J.M[(J.r0 + kk) + (int64_t)(c0 + j) * J.ld] : 0.0;
    Xs[kk * ldx + j] = v;
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  const int lr = lane >> 2, lc = lane & 3;
  const int nslice = kp / 16;
  for (int s = warp; s < nslice; s += kUpdThreads / 32) {
    double acc[2][4][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) { acc[a][b][0] = 0.0; acc[a][b][1] = 0.0; }
    const int row0 = s * 16;
    for (int kk = 0; kk < kp; kk += 4) {
      double af[2], bf[4];
#pragma unroll
      for (int a = 0; a < 2; ++a) af[a] = Wt[(row0 + a * 8 + lr) * ldw + kk + lc];
#pragma unroll
      for (int b = 0; b < 4; ++b) bf[b] = Xs[(kk + lc) * ldx + b * 8 + lr];
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma_8x8x4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          int i = row0 + a * 8 + lr;
          int j = b * 8 + lc * 2 + e;
          if (i < k && j < ncol) J.M[(J.r0 + i) + (int64_t)(c0 + j) * J.ld] = acc[a][b][e];
        }
  }
}

// ---------------------------------------------------------------------------
// right: out(32 x k) = X (32 x k) * W (k x k)
// smem: Ws[kp][kp+4] (Ws[kk][j] = W(kk,j)), Xs[32][kp+4]
// warps take 16-column slices; warp tile 32 x 16 = 4 x 2 mma tiles
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kUpdThreads) k_update_right(UpdBatch B) {
  extern __shared__ double smem[];
  int tile;
  int jb = upd_find_job(B, tile);
  if (jb < 0) return;
  const UpdJob J = B.job[jb];
  const int k = J.k;
  const int kp = (k + 15) & ~15;
  const int ldw = kp + 4;
  const int ldx = kp + 4;
  double* Ws = smem;
  double* Xs = smem + kp * ldw;
  const int tid = threadIdx.x;
  const int r0 = J.r0 + tile * kUpdTile;
  const int nrow = min(kUpdTile, J.r0 + J.len - r0);
  for (int idx = tid; idx < kp * kp; idx += blockDim.x) {
    int kk = idx % kp, j = idx / kp;
    double v = (kk < k && j < k) ? J.W[kk + (int64_t)j * J.ldw] : 0.0;
    Ws[kk * ldw + j] = v;
  }
  for (int idx = tid; idx < kUpdTile * kp; idx += blockDim.x) {
    int i = idx % kUpdTile, kk = idx / kUpdTile;
    double v = (i < nrow && kk < k) ? J.M[(r0 + i) + (int64_t)(J.c0 + kk) * J.ld] : 0.0;
    Xs[i * ldx + kk] = v;
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  const int lr = lane >> 2, lc = lane & 3;
  const int nslice = kp / 16;
  for (int s = warp; s < nslice; s += kUpdThreads / 32) {
    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) { acc[a][b][0] = 0.0; acc[a][b][1] = 0.0; }
    const int col0 = s * 16;
    for (int kk = 0; kk < kp; kk += 4) {
      double af[4], bf[2];
#pragma unroll
      for (int a = 0; a < 4; ++a) af[a] = Xs[(a * 8 + lr) * ldx + kk + lc];
#pragma unroll
      for (int b = 0; b < 2; ++b) bf[b] = Ws[(kk + lc) * ldw + col0 + b * 8 + lr];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) dmma_8x8x4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          int i = a * 8 + lr;
          int j = col0 + b * 8 + lc * 2 + e;
          if (i < nrow && j < k) J.M[(r0 + i) + (int64_t)(J.c0 + j) * J.ld] = acc[a][b][e];
        }
  }
}

// ---------------------------------------------------------------------------
// Persistent forms of the two kernels above: each CTA takes a contiguous
// run of tiles, keeps the k x k factor in shared memory while consecutive
// tiles belong to the same job, and prefetches the next slab tile with
// cp.async into a second buffer while the current one is multiplied.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void upd_cp8(void* sdst, const void* gsrc, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  const int sz = valid ? 8 : 0;  // 0: zero-fill, nothing read
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(sz) : "memory");
}
__device__ __forceinline__ void upd_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void upd_cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ int upd_locate(const UpdBatch& B, int t, int& tile) {
  for (int j = 0; j < B.njobs; ++j) {
    if (t < B.job[j].tiles) { tile = t; return j; }
    t -= B.job[j].tiles;
  }
  tile = -1;
  return -1;
}

// stage slab tile `tile` of job J into Xs (layout as in the kernels above)
__device__ __forceinline__ void upd_stage(const UpdJob& J, int tile, int side, double* Xs, int kpmax) {
  const int k = J.k;
  const int kp = (k + 15) & ~15;
  if (side == 0) {
    const int c0 = J.c0 + tile * kUpdTile;
    const int ncol = min(kUpdTile, J.c0 + J.len - c0);
    for (int idx = threadIdx.x; idx < kp * kUpdTile; idx += blockDim.x) {
      const int kk = idx % kp, j = idx / kp;
      const bool v = kk < k && j < ncol;
      upd_cp8(&Xs[kk * 36 + j], v ? &J.M[(J.r0 + kk) + (int64_t)(c0 + j) * J.ld] : J.M, v);
    }
  } else {
    const int r0 = J.r0 + tile * kUpdTile;
    const int nrow = min(kUpdTile, J.r0 + J.len - r0);
    const int ldx = kpmax + 4;
    for (int idx = threadIdx.x; idx < kUpdTile * kp; idx += blockDim.x) {
      const int i = idx % kUpdTile, kk = idx / kUpdTile;
      const bool v = i < nrow && kk < k;
      upd_cp8(&Xs[i * ldx + kk], v ? &J.M[(r0 + i) + (int64_t)(J.c0 + kk) * J.ld] : J.M, v);
    }
  }
}

template <int SIDE>
__global__ void __launch_bounds__(kUpdMaxThreads) k_update_persist(UpdBatch B, int total) {
  extern __shared__ double smem[];
  const int kpmax = (B.k + 15) & ~15;
  const int ldw = kpmax + 4;
  double* Wm = smem;                                  // kpmax x (kpmax + 4)
  const int xsz = SIDE == 0 ? kpmax * 36 : kUpdTile * (kpmax + 4);
  double* const Xbase = smem + kpmax * ldw;         // two slab buffers of xsz
  const int chunk = (total + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * chunk;
  const int t1 = min(total, t0 + chunk);
  if (t0 >= t1) return;
  const int tid = threadIdx.x;
  int tile_next;
  int jb_next = upd_locate(B, t0, tile_next);
  upd_stage(B.job[jb_next], tile_next, SIDE, Xbase, kpmax);
  upd_cp_commit();
  int cur = -1;
  for (int t = t0; t < t1; ++t) {
    const int jb = jb_next, tile = tile_next;
    const UpdJob J = B.job[jb];
    const int k = J.k;
    const int kp = (k + 15) & ~15;
    if (jb != cur) {
      // factor of this job (W^T for the left update)
      for (int idx = tid; idx < kp * kp; idx += blockDim.x) {
        const int a = idx % kp, b = idx / kp;
        const double v = (a < k && b < k) ? J.W[a + (int64_t)b * J.ldw] : 0.0;
        if (SIDE == 0) Wm[b * ldw + a] = v;   // Wt[i][kk] = W(kk, i)
        else Wm[a * ldw + b] = v;             // Ws[kk][j] = W(kk, j)
      }
      cur = jb;
    }
    if (t + 1 < t1) {
      // next tile (the next job's tile if this one is done)
      if (tile + 1 < B.job[jb].tiles) { jb_next = jb; tile_next = tile + 1; }
      else {
        jb_next = jb + 1;
        tile_next = 0;
        while (jb_next < B.njobs - 1 && B.job[jb_next].tiles == 0) ++jb_next;
      }
      upd_stage(B.job[jb_next], tile_next, SIDE, Xbase + ((t + 1 - t0) & 1) * xsz, kpmax);
      upd_cp_commit();
      upd_cp_wait<1>();
    } else {
      upd_cp_wait<0>();
    }
    __syncthreads();
    const double* Xs = Xbase + ((t - t0) & 1) * xsz;
    const int warp = tid >> 5, lane = tid & 31;
    const int lr = lane >> 2, lc = lane & 3;
    const int nslice = kp / 16;
    if (SIDE == 0) {
      const int c0 = J.c0 + tile * kUpdTile;
      const int ncol = min(kUpdTile, J.c0 + J.len - c0);
      for (int sl = warp; sl < nslice; sl += (int)(blockDim.x >> 5)) {
        double acc[2][4][2];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) { acc[a][b][0] = 0.0; acc[a][b][1] = 0.0; }
        const int row0 = sl * 16;
        for (int kk = 0; kk < kp; kk += 4) {
          double af[2], bf[4];
#pragma unroll
          for (int a = 0; a < 2; ++a) af[a] = Wm[(row0 + a * 8 + lr) * ldw + kk + lc];
#pragma unroll
          for (int b = 0; b < 4; ++b) bf[b] = Xs[(kk + lc) * 36 + b * 8 + lr];
#pragma unroll
          for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) dmma_8x8x4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int i = row0 + a * 8 + lr;
              const int j = b * 8 + lc * 2 + e;
              if (i < k && j < ncol) J.M[(J.r0 + i) + (int64_t)(c0 + j) * J.ld] = acc[a][b][e];
            }
      }
    } else {
      const int ldx = kpmax + 4;
      const int r0 = J.r0 + tile * kUpdTile;
      const int nrow = min(kUpdTile, J.r0 + J.len - r0);
      for (int sl = warp; sl < nslice; sl += (int)(blockDim.x >> 5)) {
        double acc[4][2][2];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 2; ++b) { acc[a][b][0] = 0.0; acc[a][b][1] = 0.0; }
        const int col0 = sl * 16;
        for (int kk = 0; kk < kp; kk += 4) {
          double af[4], bf[2];
#pragma unroll
          for (int a = 0; a < 4; ++a) af[a] = Xs[(a * 8 + lr) * ldx + kk + lc];
#pragma unroll
          for (int b = 0; b < 2; ++b) bf[b] = Wm[(kk + lc) * ldw + col0 + b * 8 + lr];
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) dmma_8x8x4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int i = a * 8 + lr;
              const int j = col0 + b * 8 + lc * 2 + e;
              if (i < nrow && j < k) J.M[(r0 + i) + (int64_t)(J.c0 + j) * J.ld] = acc[a][b][e];
            }
      }
    }
    __syncthreads();  // this buffer and the factor are free again
  }
}

// ---------------------------------------------------------------------------
// General k (> kUpdMaxK): FP64 SIMT, W read through L1/L2, slab tile in
// shared memory.  Used for large AED windows only.
// ---------------------------------------------------------------------------
constexpr int kUpdGenTile = 8;
__global__ void __launch_bounds__(256) k_update_left_gen(UpdBatch B) {
  extern __shared__ double smem[];
  int tile;
  int jb = upd_find_job(B, tile);
  if (jb < 0) return;
  const UpdJob J = B.job[jb];
  const int k = J.k;
  const int c0 = J.c0 + tile * kUpdGenTile;
  const int ncol = min(kUpdGenTile, J.c0 + J.len - c0);
  double* Xs = smem;  // k x 8
  for (int idx = threadIdx.x; idx < k * kUpdGenTile; idx += blockDim.x) {
    int kk = idx % k, j = idx / k;
    Xs[kk + j * k] = (j < ncol) ? J.M[(J.r0 + kk) + (int64_t)(c0 + j) * J.ld] : 0.0;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < k * ncol; idx += blockDim.x) {
    int i = idx % k, j = idx / k;
    const double* w = J.W + (int64_t)i * J.ldw;
    double acc = 0.0;
    for (int kk = 0; kk < k; ++kk) acc += w[kk] * Xs[kk + j * k];
    J.M[(J.r0 + i) + (int64_t)(c0 + j) * J.ld] = acc;
  }
}
__global__ void __launch_bounds__(256) k_update_right_gen(UpdBatch B) {
  extern __shared__ double smem[];
  int tile;
  int jb = upd_find_job(B, tile);
  if (jb < 0) return;
  const UpdJob J = B.job[jb];
  const int k = J.k;
  const int r0 = J.r0 + tile * kUpdGenTile;
  const int nrow = min(kUpdGenTile, J.r0 + J.len - r0);
  double* Xs = smem;  // 8 x k
  for (int idx = threadIdx.x; idx < k * kUpdGenTile; idx += blockDim.x) {
    int i = idx % kUpdGenTile, kk = idx / kUpdGenTile;
    Xs[i + kk * kUpdGenTile] = (i < nrow) ? J.M[(r0 + i) + (int64_t)(J.c0 + kk) * J.ld] : 0.0;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < k * nrow; idx += blockDim.x) {
    int i = idx % nrow, j = idx / nrow;
    const double* w = J.W + (int64_t)j * J.ldw;
    double acc = 0.0;
    for (int kk = 0; kk < k; ++kk) acc += Xs[i + kk * kUpdGenTile] * w[kk];
    J.M[(r0 + i) + (int64_t)(J.c0 + j) * J.ld] = acc;
  }
}

#endif  // QZ_DEFINE_UPDATE_KERNELS

}  // namespace qz
