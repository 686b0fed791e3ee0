// Reordering of a generalized real Schur form on the device (the step
// after the solve; LAPACK DTGSEN semantics, the role of the reference's
// PDTGSEN/PDTGORD, src/reorder/PDTGSEN.f:1, PDTGORD.f:1).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace qz {

struct ReorderOut {
  int m = 0;        // dimension of the selected deflating subspaces
  double pl = 1.0;  // reciprocal norms of the projections (ijob 1)
  double pr = 1.0;
  int info = 0;     // 1: a swap was rejected (the pencil is partly reordered)
  int swaps = 0;    // block swaps attempted
  int windows = 0;  // window launches
  double dif[2] = {0.0, 0.0};  // Difu, Difl estimates (ijob 3 and 5)
};

// select: host array of n flags.  S (lds), T (ldt), Q (ldq), Z (ldz) are
// device arrays; Q/Z may be null when wantq/wantz is false.
// alphar/alphai/beta: device arrays of n values.  ijob 0 (reorder), 1 (and
// PL, PR), 3 (and the 1-norm Dif estimates), 5 (PL, PR and Dif).
cudaError_t tgsen_device(cudaStream_t st, int ijob, bool wantq, bool wantz, const int* select, int n, double* S,
                         int64_t lds, double* T, int64_t ldt, double* Q, int64_t ldq, double* Z, int64_t ldz,
                         double* alphar, double* alphai, double* beta, ReorderOut* out);

}  // namespace qz
