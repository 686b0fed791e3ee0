// Launch interface of the sm_100a kernels (see kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "qz_window.cuh"
#include "update.cuh"

namespace qz {

constexpr int kWinThreads = 128;   // threads of the one-CTA AED / zero-chase kernels
constexpr int kChaseThreads = 512; // threads of the chase kernel
constexpr int kWinSmemMax = 80;    // window size held entirely in shared memory (4 x 80^2 FP64 = 200 KB)
constexpr int kMaxChain = 26;      // bulges per chain (3*26+2 rows fit a window of 80)

// odd leading dimension of a shared-memory window: consecutive elements of
// a row then fall into distinct banks (an even one puts a whole row of an
// 80-wide window into the same bank)
__host__ __device__ constexpr int smem_ld(int n) { return (n % 2 == 0) ? n + 1 : n; }

// batched solver: threads per CTA (upper bound) and pencils held in shared memory
constexpr int kBatchThreads = 256;
constexpr int kBatchSmemMax = 80;
size_t batch_smem_bytes(int smem_max);
cudaError_t batch_init();
void launch_batch(cudaStream_t st, int grid, int threads, int smem_max, int count, const int* order, const int* nsz,
                  const int64_t* moff, const int64_t* eoff, double* H, double* T, double* Q, double* Z, double* AR,
                  double* AI, double* BE, int* status, int* counter);

// chains chased concurrently (one CTA each) by one wave launch
constexpr int kMaxWave = 8;

// window jobs travel as a kernel parameter (no host->device copy)
struct ChaseJob {
  int w0, wk, last, nb, tmax;
  Bulge bl[kMaxChain];
};
struct ChaseWave {
  ChaseJob job[kMaxWave];
};

size_t aed_smem_bytes(int nw);
size_t chase_smem_bytes(int wk);
size_t inf_smem_bytes(int wk);
cudaError_t kernels_init();

void launch_aed(cudaStream_t st, double* H, double* T, int64_t ld, int ktop, int kwtop, int nw, const Tol& tol,
                double* Qw, double* Zw, double* shifts, int* info, double* gscratch,
                unsigned long long* ts = nullptr, int nskip = 0, int threads = kWinThreads, int swapfail = 0,
                int ms = 1);
// one CTA per job; job i writes its factors to U + i*ustride, V + i*ustride
void launch_chase_wave(cudaStream_t st, double* H, double* T, int64_t ld, const ChaseWave& wave, int njob, double* U,
                       double* V, int64_t ustride);
void launch_inf(cudaStream_t st, double* H, double* T, int64_t ld, int w0, int wk, int top, int jz, int stop,
                int deflate, double* U, double* V);
void launch_scan(cudaStream_t st, double* H, double* T, int64_t ld, int ifirst, int kbot, const Tol& tol, int* out);
void launch_inf_top(cudaStream_t st, double* H, double* T, double* Q, int64_t ld, int n, int f, int wantq);
// persist: one CTA per SM slot walking a run of tiles (factor kept, next tile prefetched)
void launch_update(cudaStream_t st, const UpdBatch& B, int side, int persist = 1);
int update_tile(int k);
void launch_finalize(cudaStream_t st, double* H, double* T, double* Z, int64_t ld, int n, int wantz, double* ar,
                     double* ai, double* be);
void launch_identity(cudaStream_t st, double* Q, int64_t ld, int n);
// eigenvalues (alphar, alphai, beta) of the diagonal blocks of a standardised Schur form
void launch_eigs(cudaStream_t st, const double* H, const double* T, int64_t ld, int n, double* ar, double* ai,
                 double* be);
// out[0] = largest |A(i,j)| over A(o:o+n, o:o+n); partial: 592 doubles of scratch
void launch_maxabs(cudaStream_t st, const double* A, int64_t ld, int o, int n, double* out, double* partial);
// A(0:n, 0:n) <- 2^e A
void launch_scale_pow2(cudaStream_t st, double* A, int64_t ld, int n, int e);
// out[0] = sum of squares of A(o:o+n, o:o+n); partial: 592 doubles of scratch
void launch_sumsq(cudaStream_t st, const double* A, int64_t ld, int o, int n, double* out, double* partial);

}  // namespace qz
