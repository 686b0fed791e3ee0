// Split-precision (Ozaki, INT8 slices on tcgen05) off-diagonal updates:
// job descriptions and launchers (ozaki.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define QZ_HD_OZ __host__ __device__
#else
#define QZ_HD_OZ
#endif

namespace qz {

constexpr int kOzMaxSlices = 8;   // 7-bit signed digits per FP64 entry (7 or 8)
constexpr int kOzMaxK = 80;       // largest window size on this path
constexpr int kOzMaxKp = 96;      // K padded to the MMA's K = 32
constexpr int kOzMaxFac = 16;     // factors prepared per launch (U, V of 8 windows)
constexpr int kOzMaxJobs = 32;
constexpr int kOzMaxMaps = 12;    // TMA tensor maps per launch
// TMA boxes of the FP64 slab tile, loaded in two halves of 64 rows of A:
// right update (A = M(rows, cols c0..c0+k-1)): 66 matrix rows (the start
// rounded down to an even row, the TMA rule for 8-byte elements) x k columns;
// left update (A = M(r0..r0+k-1, cols)^T): kbox = k+1 rounded up to even
// matrix rows x 64 columns
constexpr int kOzBoxRows = 66;
QZ_HD_OZ constexpr int oz_left_box(int k) { return (k + 2) & ~1; }
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
  int map;      // TMA tensor map of M for this job's box (-1: plain loads)
};

struct OzBatch {
  CUtensorMap maps[kOzMaxMaps];  // 2-D maps of the target matrices (FP64, no swizzle)
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
// Tensor map of a rows x cols column-major FP64 matrix (leading dimension
// ld, a multiple of 2) with the slab box of a left or right update of window
// size k; boxes reaching past rows or cols read zeros there.  Returns false
// when the matrix does not meet TMA's rules (then the job uses plain loads).
bool ozaki_tensor_map(CUtensorMap* map, const double* M, int64_t ld, int rows, int cols, int left, int k);
cudaError_t ozaki_init();
void launch_ozaki_prep(cudaStream_t st, const OzPrep& P, int slices);
void launch_ozaki_update(cudaStream_t st, const OzBatch& B, int slices);

}  // namespace qz
