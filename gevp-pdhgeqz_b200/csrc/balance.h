// Balancing of a general pencil (A, B) on the device, with the semantics
// of LAPACK DGGBAL (permutations isolating eigenvalues, then row and
// column scaling by powers of ten), and the back transformation of
// eigenvector or Schur-vector matrices with the semantics of DGGBAK.
// The reference driver takes the ILO/IHI this produces
// (src/pdhgeqz/PDHGEQZ.f:155-161); DGGBAL itself comes from LAPACK.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace qz {

// job: 'N', 'P', 'S' or 'B'.  A (lda) and B (ldb) are device arrays,
// transformed in place.  ilo/ihi are returned 1-based; lscale/rscale are
// host arrays of n values (permutation indices, 1-based, outside
// ilo..ihi; scale factors inside).  Returns 0, or a CUDA error code.
cudaError_t ggbal_device(cudaStream_t st, char job, int n, double* a, int64_t lda, double* b, int64_t ldb, int* ilo,
                         int* ihi, double* lscale, double* rscale);

// job: 'N', 'P', 'S' or 'B'; side: 'L' (uses lscale) or 'R' (rscale).
// v is a device array of n rows and m columns (ldv), transformed in place.
cudaError_t ggbak_device(cudaStream_t st, char job, char side, int n, int ilo, int ihi, const double* lscale,
                         const double* rscale, int m, double* v, int64_t ldv);

}  // namespace qz
