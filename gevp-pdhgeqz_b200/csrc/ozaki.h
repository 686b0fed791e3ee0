// Split-precision (Ozaki, INT8 slices on tcgen05) off-diagonal updates:
// job descriptions and launchers (ozaki.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qz {

constexpr int kOzMaxSlices = 8;   // 7-bit signed digits per FP64 entry (7 or 8)
constexpr int kOzMaxK = 80;       // largest window size on this path
constexpr int kOzMaxKp = 96;      // K padded to the MMA's K = 32
constexpr int kOzMaxFac = 16;     // factors prepared per launch (U, V of 8 windows)
constexpr int kOzMaxJobs = 32;
// one factor's digits (S x kp x Kp bytes) and column scales (kp ints)
constexpr size_t kOzFacBytes = 61952;
static_assert((size_t)kOzMaxSlices * kOzMaxK * kOzMaxKp + 4 * kOzMaxK <= kOzFacBytes, "factor slot too small");

struct OzJob {
  double* M;    // target matrix (column-major, leading dimension ld)
  int64_t ld;
  int r0, c0;   // slab origin
  int len;      // slab extent along the non-k direction
  int k;        // window size (<= kOzMaxK)
  int left;     // 1: M(r0:r0+k, c0:c0+len) <- W^T M; 0: M(r0:r0+len, c0:c0+k) <- M W
  int fac;      // index of W's prepared digits
  int tiles;    // 128-row tiles of this job
};

struct OzBatch {
  OzJob job[kOzMaxJobs];
  int njobs;
  const uint8_t* bslices;  // kOzFacBytes per factor
  int* err;                // set to 1 if a tensor-core wait timed out
};

struct OzPrep {
  const double* W[kOzMaxFac];
  int ldw[kOzMaxFac];
  int k[kOzMaxFac];
  int nfac;
  uint8_t* out;
};

size_t ozaki_smem_bytes(int slices);
cudaError_t ozaki_init();
void launch_ozaki_prep(cudaStream_t st, const OzPrep& P, int slices);
void launch_ozaki_update(cudaStream_t st, const OzBatch& B, int slices);

}  // namespace qz
