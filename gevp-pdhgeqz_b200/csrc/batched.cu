// Batched QZ of many independent small pencils of uneven sizes.
//
// Role in the reference: none directly (PDHGEQZ solves one pencil); this is
// the batched workload of the measurement plan, built from the same
// CTA-level kernels as the endgame (PDHGEQZ4 -> KKQZ): every pencil is
// reduced to generalized Schur form with Q and Z by one CTA.
//
// One persistent launch: CTAs pull pencils from an atomic queue ordered by
// decreasing size (longest-first scheduling), solve a pencil in shared
// memory when n <= kBatchSmemMax (H, T, Q, Z with an odd leading
// dimension), in place in global memory otherwise, normalise beta >= 0 and
// write the eigenvalues.  Pencils long enough for chains of bulges are
// reduced by small-bulge multishift sweeps (cta_small_qz_ms), shorter
// ones by double-shift sweeps.  Per-pencil status words; no host round
// trip.
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "../../include/b200qz.h"
#include "kernels.h"
#include "qz_window.cuh"

namespace qz {

namespace {

struct BExec {
  int tid, nt;
  int* si;
  double* sd;
  __device__ void sync() { __syncthreads(); }
  __device__ void stamp(int) {}
  __device__ void count(int) {}
};

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  __syncthreads();
  if (threadIdx.x == 0) red[0] = t;
  __syncthreads();
  return red[0];
}

}  // namespace

__global__ void __launch_bounds__(kBatchThreads) k_batch_qz(int count, const int* __restrict__ order,
                                                            const int* __restrict__ nsz,
                                                            const int64_t* __restrict__ moff,
                                                            const int64_t* __restrict__ eoff, double* H, double* T,
                                                            double* Q, double* Z, double* AR, double* AI, double* BE,
                                                            int* status, int* counter, int smem_max) {
  extern __shared__ double smem[];
  __shared__ int s_next;
  __shared__ double red[32];
  __shared__ int si[64];
  __shared__ double sd_small[64];
  __shared__ double ms_scr[kMsScratch];  // multishift window QZ scratch
  for (;;) {
    if (threadIdx.x == 0) s_next = atomicAdd(counter, 1);
    __syncthreads();
    const int idx = s_next;
    __syncthreads();
    if (idx >= count) break;
    const int p = order[idx];
    const int n = nsz[p];
    double* Hg = H + moff[p];
    double* Tg = T + moff[p];
    double* Qg = Q + moff[p];
    double* Zg = Z + moff[p];
    // tolerances of this pencil (PDHGEQZ.f:449-458)
    double hs = 0.0, ts = 0.0;
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
      hs += Hg[k] * Hg[k];
      ts += Tg[k] * Tg[k];
    }
    hs = block_sum(hs, red);
    ts = block_sum(ts, red);
    Tol tol;
    tol.safmin = DBL_MIN;
    tol.ulp = DBL_EPSILON;
    tol.smlnum = DBL_MIN * ((double)n / DBL_EPSILON);
    tol.htol = fmax(DBL_MIN, DBL_EPSILON * sqrt(hs));
    tol.ttol = fmax(DBL_MIN, DBL_EPSILON * sqrt(ts));
    const bool in_smem = n <= smem_max;
    const int lw = in_smem ? smem_ld(n) : n;
    double *Hs, *Ts, *Qs, *Zs;
    if (in_smem) {
      Hs = smem;
      Ts = Hs + n * lw;
      Qs = Ts + n * lw;
      Zs = Qs + n * lw;
      for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
        int i = k % n, j = k / n;
        Hs[i + j * lw] = Hg[k];
        Ts[i + j * lw] = Tg[k];
        Qs[i + j * lw] = (i == j) ? 1.0 : 0.0;
        Zs[i + j * lw] = (i == j) ? 1.0 : 0.0;
      }
    } else {
      Hs = Hg;
      Ts = Tg;
      Qs = Qg;
      Zs = Zg;
      for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
        int i = k % n, j = k / n;
        Qs[k] = (i == j) ? 1.0 : 0.0;
        Zs[k] = (i == j) ? 1.0 : 0.0;
      }
    }
    __syncthreads();
    BExec x{(int)threadIdx.x, (int)blockDim.x, si, sd_small};
    WinState w;
    w.n = n;
    w.H = MatV{Hs, lw};
    w.T = MatV{Ts, lw};
    w.Q = MatV{Qs, lw};
    w.Z = MatV{Zs, lw};
    w.wantq = true;
    w.wantz = true;
    w.tol = tol;
    // pencils long enough for chains of bulges take multishift sweeps
    int info = cta_small_qz_ms(x, w, 30 * n, ms_scr);
    __syncthreads();
    if (info == 0) cta_finalize(x, w, AR + eoff[p], AI + eoff[p], BE + eoff[p]);
    if (in_smem) {
      for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
        int i = k % n, j = k / n;
        Hg[k] = Hs[i + j * lw];
        Tg[k] = Ts[i + j * lw];
        Qg[k] = Qs[i + j * lw];
        Zg[k] = Zs[i + j * lw];
      }
    }
    if (threadIdx.x == 0) status[p] = info;
    __syncthreads();
  }
}

size_t batch_smem_bytes(int smem_max) { return (size_t)4 * smem_max * smem_ld(smem_max) * sizeof(double); }

cudaError_t batch_init() {
  return cudaFuncSetAttribute(k_batch_qz, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)batch_smem_bytes(kBatchSmemMax));
}

void launch_batch(cudaStream_t st, int grid, int threads, int smem_max, int count, const int* order, const int* nsz,
                  const int64_t* moff, const int64_t* eoff, double* H, double* T, double* Q, double* Z, double* AR,
                  double* AI, double* BE, int* status, int* counter) {
  cudaMemsetAsync(counter, 0, sizeof(int), st);
  k_batch_qz<<<grid, threads, batch_smem_bytes(smem_max), st>>>(count, order, nsz, moff, eoff, H, T, Q, Z, AR, AI, BE,
                                                                status, counter, smem_max);
}

// The same launch, returning the status of this call's own memset and
// kernel launch (cudaLaunchKernel reports the launch error directly, so an
// error left pending by unrelated earlier work is neither reported as ours
// nor cleared).
static cudaError_t launch_batch_checked(cudaStream_t st, int grid, int threads, int smem_max, int count,
                                        const int* order, const int* nsz, const int64_t* moff, const int64_t* eoff,
                                        double* H, double* T, double* Q, double* Z, double* AR, double* AI,
                                        double* BE, int* status, int* counter) {
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  void* args[] = {&count, &order, &nsz, &moff, &eoff, &H, &T, &Q, &Z, &AR, &AI, &BE, &status, &counter, &smem_max};
  return cudaLaunchKernel((const void*)k_batch_qz, dim3(grid), dim3(threads), args, batch_smem_bytes(smem_max), st);
}

// ---------------------------------------------------------------------------
// Batched solve that allocates nothing.
//
// For callers that may not allocate device memory themselves: code that
// runs inside another library's memory pool or allocator, hosts that
// reserve the whole device heap up front, or real-time loops where an
// allocation could block.  The per-batch descriptors and the work-queue
// counter live in one fixed array in the library's device memory instead
// of a buffer from cudaMalloc.  Every GPU that loads the library holds the
// array (kNoAllocBytes) until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxPencils = 4096;
// moff, eoff (int64), order, n (int32), queue counter
constexpr size_t kNoAllocBytes = (size_t)kNoAllocMaxPencils * (2 * sizeof(int64_t) + 2 * sizeof(int)) + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocDev {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
  int sm_count = 0;
};
NoAllocDev g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

// Once per device, with that device current: the device address of the
// scratch array (its host-side name is only a stand-in), the SM count and
// the kernel's shared-memory limit.
int noalloc_setup(int dev, NoAllocDev** out) {
  if (dev < 0 || dev >= kNoAllocMaxDevices) return 10001;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoAllocDev& d = g_noalloc_dev[dev];
  if (!d.ready) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return 10001;
    if (cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 10001;
    if (batch_init() != cudaSuccess) return 10001;
    d.scratch = (unsigned char*)p;
    d.ready = true;
  }
  *out = &d;
  return 0;
}

}  // namespace

}  // namespace qz

extern "C" int b200qz_solve_batched_noalloc(int count, const int* n, const long long* moff, const long long* eoff,
                                            double* h, double* t, double* q, double* z, double* alphar,
                                            double* alphai, double* beta, int* info, void* stream) {
  using namespace qz;
  if (count < 0) return -1;
  if (count > kNoAllocMaxPencils) return -2;
  for (int i = 0; i < count; ++i)
    if (n[i] < 1 || n[i] > 46340) return -3;
  if (count == 0) return 0;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 10001;
  NoAllocDev* d = nullptr;
  if (noalloc_setup(dev, &d) != 0) return 10001;
  cudaStream_t st = (cudaStream_t)stream;
  // longest pencils first on the work queue (order held on the stack)
  int order[kNoAllocMaxPencils];
  for (int i = 0; i < count; ++i) order[i] = i;
  std::sort(order, order + count, [&](int a, int b) { return n[a] != n[b] ? n[a] > n[b] : a < b; });
  int64_t* d_moff = (int64_t*)d->scratch;
  int64_t* d_eoff = d_moff + kNoAllocMaxPencils;
  int* d_order = (int*)(d_eoff + kNoAllocMaxPencils);
  int* d_n = d_order + kNoAllocMaxPencils;
  int* d_counter = d_n + kNoAllocMaxPencils;
  // Host-to-device copies from pageable memory (the stack array `order`, and
  // n/moff/eoff when the caller passes ordinary memory) return only after
  // the source has been copied to a staging buffer, as the CUDA runtime
  // documents for cudaMemcpyAsync from pageable memory, so `order` may go
  // out of scope on return.  Page-locked n/moff/eoff are read when the
  // stream reaches the copy: the caller keeps them unchanged until then.
  if (cudaMemcpyAsync(d_moff, moff, count * sizeof(int64_t), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_eoff, eoff, count * sizeof(int64_t), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_order, order, count * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_n, n, count * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return 10001;
  // the queue counter is zeroed on the stream before the kernel starts
  const cudaError_t e = launch_batch_checked(st, d->sm_count, 128, kBatchSmemMax, count, d_order, d_n, d_moff, d_eoff,
                                             h, t, q, z, alphar, alphai, beta, info, d_counter);
  return e == cudaSuccess ? 0 : 10001;
}

