// Hessenberg-triangular reduction on the device (LAPACK DGGHRD semantics;
// the role of the reference's PDGGHRD, src/ab2ht/PDGGHRD.f:13).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace qz {

struct GghrdOut {
  int64_t pairs = 0;     // rotation pairs
  int64_t launches = 0;  // kernel launches
};

// Reduce columns ilo..ihi-2 (0-based) of A to upper Hessenberg form while
// keeping B upper triangular (B's strict lower triangle is set to zero
// first, as DGGHRD does).  icompq / icompz: 0 do not touch Q / Z, 1 update
// the given matrix, 2 set it to the identity first.  qrows: Q accumulates
// the row rotations from the left (Q <- G Q, the transposed Q that
// PDGGHRD returns) instead of Q <- Q G^T (DGGHRD).  wmax: pairs per window
// (<= kHrMaxWin).  All pointers are device pointers.
constexpr int kHrMaxWin = 160;
cudaError_t gghrd_device(cudaStream_t st, int icompq, int icompz, bool qrows, int n, int ilo, int ihi, double* A,
                         int64_t lda, double* B, int64_t ldb, double* Q, int64_t ldq, double* Z, int64_t ldz, int wmax,
                         GghrdOut* out);

}  // namespace qz
