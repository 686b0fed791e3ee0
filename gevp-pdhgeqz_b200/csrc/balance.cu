// Balancing of a general pencil on the device (DGGBAL semantics) and the
// back transformation (DGGBAK semantics).
//
// Permutation: rows whose nonzeros (in A or B) among the active columns
// lie in at most one column are moved to the bottom of the active block,
// that column with them, the row searched from the bottom up; then columns
// whose nonzeros among the active rows lie in at most one row are moved to
// the top, searched from the left.  An empty row takes the last active
// column, an empty column the last active row.  The nonzero counts of all
// rows and columns come from one pass over the matrices on the whole GPU;
// the isolation loop runs in one CTA and keeps the counts current in O(n)
// per isolated row or column.
//
// Scaling (Ward, "Balancing the generalized eigenvalue problem", SIAM J.
// Sci. Stat. Comput. 2 (1981)): row and column exponents r, c minimise
// sum over the nonzeros of (log10|a_ij| + r_i + c_j)^2 + (log10|b_ij| +
// r_i + c_j)^2.  The normal equations M [r; c] = g are solved by
// preconditioned conjugate gradients with the pseudo-inverse of M for a
// dense pencil as the preconditioner: for nr active rows,
//   z_r = g_r / (2 nr) + (s_c - 3 s_r) / (8 nr^2),
//   z_c = g_c / (2 nr) + (s_r - 3 s_c) / (8 nr^2),   s_* = sum of g_*,
// at most nr + 2 iterations, stopping when no exponent moves by 1/2.  The
// exponents are rounded half away from zero, limited so that no row or
// column overflows, and applied as powers of ten (rows first).  Products
// M p use a byte matrix of nonzero counts; every reduction has a fixed
// order, so the result does not depend on scheduling.
#include "balance.h"

#include <cfloat>
#include <climits>
#include <cmath>
#include <vector>

namespace qz {
namespace {

__device__ __forceinline__ bool nz_ab(const double* A, int64_t lda, const double* B, int64_t ldb, int i, int j) {
  return A[i + (int64_t)j * lda] != 0.0 || B[i + (int64_t)j * ldb] != 0.0;
}

// nonzero counts of every row (over all columns) and every column (over
// all rows); 32 x 32 tiles, block (32, 8)
__global__ void k_bal_counts(const double* A, int64_t lda, const double* B, int64_t ldb, int n, int* rowcnt,
                             int* colcnt) {
  __shared__ int part[8][32];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int r = blockIdx.x * 32 + tx;
  const int c0 = blockIdx.y * 32;
  int cr = 0;
  for (int k = 0; k < 4; ++k) {
    const int c = c0 + ty + 8 * k;
    const bool nz = (r < n && c < n) && nz_ab(A, lda, B, ldb, r, c);
    cr += nz;
    const unsigned bal = __ballot_sync(0xffffffffu, nz);
    if (tx == 0 && bal) atomicAdd(&colcnt[c], __popc(bal));
  }
  part[ty][tx] = cr;
  __syncthreads();
  if (ty == 0 && r < n) {
    int s = 0;
    for (int k = 0; k < 8; ++k) s += part[k][tx];
    if (s) atomicAdd(&rowcnt[r], s);
  }
}

constexpr int kPermThreads = 1024;

// maximum of v over the block, returned to every thread
__device__ int block_max_int(int v, int* red) {
  for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  v = ((int)(threadIdx.x & 31) < (int)(blockDim.x >> 5)) ? red[threadIdx.x & 31] : INT_MIN;
  for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ void swap_rows2(double* A, int64_t lda, double* B, int64_t ldb, int n, int r1, int r2) {
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    double t = A[r1 + (int64_t)c * lda];
    A[r1 + (int64_t)c * lda] = A[r2 + (int64_t)c * lda];
    A[r2 + (int64_t)c * lda] = t;
    t = B[r1 + (int64_t)c * ldb];
    B[r1 + (int64_t)c * ldb] = B[r2 + (int64_t)c * ldb];
    B[r2 + (int64_t)c * ldb] = t;
  }
}
__device__ void swap_cols2(double* A, int64_t lda, double* B, int64_t ldb, int n, int c1, int c2) {
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    double t = A[r + (int64_t)c1 * lda];
    A[r + (int64_t)c1 * lda] = A[r + (int64_t)c2 * lda];
    A[r + (int64_t)c2 * lda] = t;
    t = B[r + (int64_t)c1 * ldb];
    B[r + (int64_t)c1 * ldb] = B[r + (int64_t)c2 * ldb];
    B[r + (int64_t)c2 * ldb] = t;
  }
}

// The isolation loop (one CTA).  rowcnt/colcnt: counts over the whole
// matrix on entry.  out = {lo, hi} (0-based); lrec/rrec[p] = the row and
// column moved to position p, for p outside lo..hi.
__global__ void __launch_bounds__(kPermThreads) k_bal_perm(double* A, int64_t lda, double* B, int64_t ldb, int n,
                                                           int* rowcnt, int* colcnt, int* out, int* lrec, int* rrec) {
  __shared__ int red[32];
  int lo = 0, hi = n - 1;
  // rows with at most one nonzero among the active columns, to the bottom
  while (hi > lo) {
    int cand = -1;
    for (int r = hi - (int)threadIdx.x; r >= lo; r -= blockDim.x)
      if (rowcnt[r] <= 1) { cand = r; break; }
    const int rs = block_max_int(cand, red);
    if (rs < 0) break;
    int jc = hi;
    if (rowcnt[rs] != 0) {
      int cj = -1;
      for (int j = lo + (int)threadIdx.x; j <= hi; j += blockDim.x)
        if (nz_ab(A, lda, B, ldb, rs, j)) cj = j;
      jc = block_max_int(cj, red);
    }
    if (threadIdx.x == 0) { lrec[hi] = rs; rrec[hi] = jc; }
    if (rs != hi) swap_rows2(A, lda, B, ldb, n, rs, hi);
    __syncthreads();  // the two swaps share four elements
    if (jc != hi) swap_cols2(A, lda, B, ldb, n, jc, hi);
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = rowcnt[rs]; rowcnt[rs] = rowcnt[hi]; rowcnt[hi] = t;
      t = colcnt[jc]; colcnt[jc] = colcnt[hi]; colcnt[hi] = t;
    }
    __syncthreads();
    // column hi leaves the active columns
    for (int r = lo + (int)threadIdx.x; r < hi; r += blockDim.x)
      if (nz_ab(A, lda, B, ldb, r, hi)) rowcnt[r] -= 1;
    __syncthreads();
    --hi;
  }
  // columns with at most one nonzero among the active rows, to the top
  while (lo < hi) {
    int cand = -1;  // the smallest such column, as a maximum of -c
    for (int c = lo + (int)threadIdx.x; c <= hi; c += blockDim.x)
      if (colcnt[c] <= 1) { cand = INT_MAX - c; break; }
    const int m = block_max_int(cand, red);
    if (m < 0) break;
    const int cs = INT_MAX - m;
    int ir = hi;
    if (colcnt[cs] != 0) {
      int ci = -1;
      for (int i = lo + (int)threadIdx.x; i <= hi; i += blockDim.x)
        if (nz_ab(A, lda, B, ldb, i, cs)) ci = i;
      ir = block_max_int(ci, red);
    }
    if (threadIdx.x == 0) { lrec[lo] = ir; rrec[lo] = cs; }
    if (cs != lo) swap_cols2(A, lda, B, ldb, n, cs, lo);
    __syncthreads();
    if (ir != lo) swap_rows2(A, lda, B, ldb, n, ir, lo);
    __syncthreads();
    if (threadIdx.x == 0) { int t = colcnt[cs]; colcnt[cs] = colcnt[lo]; colcnt[lo] = t; }
    __syncthreads();
    // row lo leaves the active rows
    for (int c = lo + 1 + (int)threadIdx.x; c <= hi; c += blockDim.x)
      if (nz_ab(A, lda, B, ldb, lo, c)) colcnt[c] -= 1;
    __syncthreads();
    ++lo;
  }
  if (threadIdx.x == 0) { out[0] = lo; out[1] = hi; }
}

constexpr int kColChunk = 512;  // columns per partial row sum

// active block rows lo..lo+nr-1, columns lo..lo+nr-1: nonzero-count byte
// matrix E (nr x nr, column-major) and partial row sums of log10|a| +
// log10|b| and row counts over column chunks (fixed order)
__global__ void k_bal_rowlogs(const double* A, int64_t lda, const double* B, int64_t ldb, int lo, int nr,
                              unsigned char* E, double* part, int* cpart) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int ch = blockIdx.y;
  if (i >= nr) return;
  const int j0 = ch * kColChunk, j1 = min(nr, j0 + kColChunk);
  double s = 0.0;
  int cnt = 0;
  for (int j = j0; j < j1; ++j) {
    const double a = A[(lo + i) + (int64_t)(lo + j) * lda], b = B[(lo + i) + (int64_t)(lo + j) * ldb];
    double ta = 0.0, tb = 0.0;
    int e = 0;
    if (a != 0.0) { ta = log10(fabs(a)); ++e; }
    if (b != 0.0) { tb = log10(fabs(b)); ++e; }
    s += ta + tb;
    cnt += e;
    E[i + (int64_t)j * nr] = (unsigned char)e;
  }
  part[(int64_t)ch * nr + i] = s;
  cpart[(int64_t)ch * nr + i] = cnt;
}
__global__ void k_bal_rowsum(int nr, int nch, const double* part, const int* cpart, double* g, int* cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr) return;
  double s = 0.0;
  int c = 0;
  for (int ch = 0; ch < nch; ++ch) { s += part[(int64_t)ch * nr + i]; c += cpart[(int64_t)ch * nr + i]; }
  g[i] = -s;
  cnt[i] = c;
}
// column sums of the logs and column counts: one warp per column
__global__ void k_bal_collogs(const double* A, int64_t lda, const double* B, int64_t ldb, int lo, int nr, double* g,
                              int* cnt) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= nr) return;
  double s = 0.0;
  int c = 0;
  for (int i = lane; i < nr; i += 32) {
    const double a = A[(lo + i) + (int64_t)(lo + j) * lda], b = B[(lo + i) + (int64_t)(lo + j) * ldb];
    double ta = 0.0, tb = 0.0;
    if (a != 0.0) { ta = log10(fabs(a)); ++c; }
    if (b != 0.0) { tb = log10(fabs(b)); ++c; }
    s += ta + tb;
  }
  for (int o = 16; o; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if (lane == 0) { g[j] = -s; cnt[j] = c; }
}

// PCG state in one device block
struct BalCg {
  double gamma, pgamma, cmax;
  int done, it;
};

constexpr int kCgThreads = 1024;

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  v = ((int)(threadIdx.x & 31) < (int)(blockDim.x >> 5)) ? red[threadIdx.x & 31] : 0.0;
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ double block_maxd(double v, double* red) {
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  v = ((int)(threadIdx.x & 31) < (int)(blockDim.x >> 5)) ? red[threadIdx.x & 31] : 0.0;
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// first half of an iteration: preconditioned residual, gamma, new direction
__global__ void __launch_bounds__(kCgThreads) k_bal_cg_a(int nr, const double* gr, const double* gc, double* pr,
                                                         double* pc, BalCg* cg) {
  __shared__ double red[32];
  if (cg->done) return;
  double sr = 0.0, sc = 0.0, gg = 0.0;
  for (int i = threadIdx.x; i < nr; i += blockDim.x) {
    sr += gr[i];
    sc += gc[i];
    gg += gr[i] * gr[i] + gc[i] * gc[i];
  }
  sr = block_sum(sr, red);
  sc = block_sum(sc, red);
  gg = block_sum(gg, red);
  const double coef = 1.0 / (2.0 * nr), coef2 = coef * coef, coef5 = 0.5 * coef2;
  const double gamma = coef * gg - coef2 * (sr * sr + sc * sc) - coef5 * (sr - sc) * (sr - sc);
  const int it = cg->it;
  __syncthreads();
  if (gamma == 0.0) {
    if (threadIdx.x == 0) cg->done = 1;
    return;
  }
  const double beta = (it == 1) ? 0.0 : gamma / cg->pgamma;
  const double tr = coef5 * (sc - 3.0 * sr), tc = coef5 * (sr - 3.0 * sc);
  for (int i = threadIdx.x; i < nr; i += blockDim.x) {
    pr[i] = (beta * pr[i] + coef * gr[i]) + tr;
    pc[i] = (beta * pc[i] + coef * gc[i]) + tc;
  }
  if (threadIdx.x == 0) cg->gamma = gamma;
}

// q = M p: rows (partial sums over column chunks, fixed order)
__global__ void k_bal_mv_rows(int nr, const unsigned char* E, const double* pc, double* part, const BalCg* cg) {
  if (cg->done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int ch = blockIdx.y;
  if (i >= nr) return;
  const int j0 = ch * kColChunk, j1 = min(nr, j0 + kColChunk);
  double s = 0.0;
  for (int j = j0; j < j1; ++j) s += (double)E[i + (int64_t)j * nr] * pc[j];
  part[(int64_t)ch * nr + i] = s;
}
__global__ void k_bal_mv_rowsum(int nr, int nch, const double* part, const int* rowcnt, const double* pr, double* qr,
                                const BalCg* cg) {
  if (cg->done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr) return;
  double s = 0.0;
  for (int ch = 0; ch < nch; ++ch) s += part[(int64_t)ch * nr + i];
  qr[i] = (double)rowcnt[i] * pr[i] + s;
}
// columns: one warp per column
__global__ void k_bal_mv_cols(int nr, const unsigned char* E, const double* pr, const int* colcnt, const double* pc,
                              double* qc, const BalCg* cg) {
  if (cg->done) return;
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= nr) return;
  double s = 0.0;
  for (int i = lane; i < nr; i += 32) s += (double)E[i + (int64_t)j * nr] * pr[i];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) qc[j] = (double)colcnt[j] * pc[j] + s;
}

// second half: step length, exponent corrections, residual update
__global__ void __launch_bounds__(kCgThreads) k_bal_cg_b(int nr, double* gr, double* gc, const double* pr,
                                                         const double* pc, const double* qr, const double* qc,
                                                         double* xr, double* xc, BalCg* cg) {
  __shared__ double red[32];
  if (cg->done) return;
  double pq = 0.0;
  for (int i = threadIdx.x; i < nr; i += blockDim.x) pq += pr[i] * qr[i] + pc[i] * qc[i];
  pq = block_sum(pq, red);
  const double alpha = cg->gamma / pq;
  double cmax = 0.0;
  for (int i = threadIdx.x; i < nr; i += blockDim.x) {
    const double a = alpha * pr[i], b = alpha * pc[i];
    cmax = fmax(cmax, fmax(fabs(a), fabs(b)));
    xr[i] += a;
    xc[i] += b;
  }
  cmax = block_maxd(cmax, red);
  const bool stop = !(cmax >= 0.5);
  if (!stop)
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
      gr[i] -= alpha * qr[i];
      gc[i] -= alpha * qc[i];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    cg->cmax = cmax;
    cg->pgamma = cg->gamma;
    cg->it += 1;
    if (stop || cg->it > nr + 2) cg->done = 1;
  }
}

// largest magnitude of each active row over columns lo..n-1 and of each
// active column over rows 0..hi (bit patterns of non-negative doubles
// order like the values)
__global__ void k_bal_rowmax(const double* A, int64_t lda, const double* B, int64_t ldb, int n, int lo, int nr,
                             unsigned long long* rab) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr) return;
  const int j0 = lo + blockIdx.y * kColChunk, j1 = min(n, j0 + kColChunk);
  double m = 0.0;
  for (int j = j0; j < j1; ++j)
    m = fmax(m, fmax(fabs(A[(lo + i) + (int64_t)j * lda]), fabs(B[(lo + i) + (int64_t)j * ldb])));
  if (m > 0.0) atomicMax(&rab[i], (unsigned long long)__double_as_longlong(m));
}
__global__ void k_bal_colmax(const double* A, int64_t lda, const double* B, int64_t ldb, int lo, int hi,
                             double* cab) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int nr = hi - lo + 1;
  if (j >= nr) return;
  double m = 0.0;
  for (int i = lane; i <= hi; i += 32)
    m = fmax(m, fmax(fabs(A[i + (int64_t)(lo + j) * lda]), fabs(B[i + (int64_t)(lo + j) * ldb])));
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) cab[j] = m;
}

// A(i, j) *= ls(i) for rows lo..hi, columns lo..n-1; then *= rs(j) for
// columns lo..hi, rows 0..hi
__global__ void k_bal_apply(double* A, int64_t lda, double* B, int64_t ldb, int n, int lo, int hi, const double* ls,
                            const double* rs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // row 0..hi
  if (i > hi) return;
  for (int j = lo + blockIdx.y; j < n; j += gridDim.y) {  // column lo..n-1
    double a = A[i + (int64_t)j * lda], b = B[i + (int64_t)j * ldb];
    if (i >= lo) { a *= ls[i - lo]; b *= ls[i - lo]; }
    if (j <= hi) { a *= rs[j - lo]; b *= rs[j - lo]; }
    A[i + (int64_t)j * lda] = a;
    B[i + (int64_t)j * ldb] = b;
  }
}

// rows of V scaled; then gathered by a permutation
__global__ void k_bak_scale(double* V, int64_t ldv, int m, int lo, int hi, const double* sc) {
  const int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i > hi) return;
  for (int c = blockIdx.y; c < m; c += gridDim.y) V[i + (int64_t)c * ldv] *= sc[i - lo];
}
__global__ void k_bak_gather(const double* V, int64_t ldv, int n, int m, const int* src, double* W) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = blockIdx.y; c < m; c += gridDim.y) W[i + (int64_t)c * n] = V[src[i] + (int64_t)c * ldv];
}
__global__ void k_bak_copy(const double* W, int n, int m, double* V, int64_t ldv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = blockIdx.y; c < m; c += gridDim.y) V[i + (int64_t)c * ldv] = W[i + (int64_t)c * n];
}
inline unsigned gy(int m) { return (unsigned)(m < 65535 ? m : 65535); }

// 10^k by binary powering (exact for |k| <= 22), reciprocal for k < 0
double pow10i(int k) {
  int m = k < 0 ? -k : k;
  double x = 10.0, r = 1.0;
  while (m) {
    if (m & 1) r *= x;
    m >>= 1;
    if (m) x *= x;
  }
  return k < 0 ? 1.0 / r : r;
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

inline int upper(char c) { return (c >= 'a' && c <= 'z') ? c - 32 : c; }

}  // namespace

cudaError_t ggbal_device(cudaStream_t st, char job, int n, double* a, int64_t lda, double* b, int64_t ldb, int* ilo,
                         int* ihi, double* lscale, double* rscale) {
  job = (char)upper(job);
  if (n <= 0) {
    *ilo = 1;
    *ihi = 0;
    return cudaSuccess;
  }
  const bool perm = job == 'P' || job == 'B', scale = job == 'S' || job == 'B';
  for (int i = 0; i < n; ++i) lscale[i] = rscale[i] = 1.0;
  *ilo = 1;
  *ihi = n;
  if ((!perm && !scale) || n == 1) return cudaSuccess;
  cudaError_t e;
  int lo = 0, hi = n - 1;
  if (perm) {
    DevBuf buf;
    e = cudaMalloc(&buf.p, sizeof(int) * (4 * (size_t)n + 2));
    if (e != cudaSuccess) return e;
    int* rowcnt = (int*)buf.p;
    int* colcnt = rowcnt + n;
    int* lrec = colcnt + n;
    int* rrec = lrec + n;
    int* out = rrec + n;
    e = cudaMemsetAsync(rowcnt, 0, sizeof(int) * 2 * (size_t)n, st);
    if (e != cudaSuccess) return e;
    const int nt = (n + 31) / 32;
    k_bal_counts<<<dim3(nt, nt), dim3(32, 8), 0, st>>>(a, lda, b, ldb, n, rowcnt, colcnt);
    k_bal_perm<<<1, kPermThreads, 0, st>>>(a, lda, b, ldb, n, rowcnt, colcnt, out, lrec, rrec);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    std::vector<int> h(2 * (size_t)n + 2);
    e = cudaMemcpyAsync(h.data(), lrec, sizeof(int) * (2 * (size_t)n + 2), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    lo = h[2 * (size_t)n];
    hi = h[2 * (size_t)n + 1];
    for (int p = 0; p < n; ++p)
      if (p < lo || p > hi) {
        lscale[p] = h[p] + 1;
        rscale[p] = h[n + p] + 1;
      }
    *ilo = lo + 1;
    *ihi = hi + 1;
  }
  if (!scale || lo == hi) return cudaSuccess;

  const int nr = hi - lo + 1;
  const int nch = (nr + kColChunk - 1) / kColChunk;
  const int nchn = (n - lo + kColChunk - 1) / kColChunk;
  // doubles: gr gc pr pc qr qc xr xc cab (9 nr) + partial sums (nch nr);
  // rab (nr 64-bit); ints: rowcnt colcnt (2 nr) + partial counts (nch nr);
  // BalCg; bytes: E (nr^2)
  const size_t nd = 9 * (size_t)nr + (size_t)nch * nr;
  const size_t ni = 2 * (size_t)nr + (size_t)nch * nr;
  const size_t bytes = nd * 8 + (size_t)nr * 8 + ni * 4 + 8 + 64 + (size_t)nr * nr;
  DevBuf buf;
  e = cudaMalloc(&buf.p, bytes);
  if (e != cudaSuccess) return e;
  double* gr = (double*)buf.p;
  double* gc = gr + nr;
  double* pr = gc + nr;
  double* pc = pr + nr;
  double* qr = pc + nr;
  double* qc = qr + nr;
  double* xr = qc + nr;
  double* xc = xr + nr;
  double* cab = xc + nr;
  double* part = cab + nr;
  unsigned long long* rab = (unsigned long long*)(part + (size_t)nch * nr);
  int* rowcnt = (int*)(rab + nr);
  int* colcnt = rowcnt + nr;
  int* cpart = colcnt + nr;
  BalCg* cg = (BalCg*)(cpart + (size_t)nch * nr + ((size_t)nch * nr) % 2);
  unsigned char* E = (unsigned char*)(cg) + 64;

  e = cudaMemsetAsync(pr, 0, sizeof(double) * 6 * (size_t)nr, st);  // pr pc qr qc xr xc
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(rab, 0, sizeof(unsigned long long) * (size_t)nr, st);
  if (e != cudaSuccess) return e;
  BalCg h0{0.0, 0.0, 0.0, 0, 1};
  e = cudaMemcpyAsync(cg, &h0, sizeof(BalCg), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  const int rb = (nr + 255) / 256;
  k_bal_rowlogs<<<dim3(rb, nch), 256, 0, st>>>(a, lda, b, ldb, lo, nr, E, part, cpart);
  k_bal_rowsum<<<rb, 256, 0, st>>>(nr, nch, part, cpart, gr, rowcnt);
  k_bal_collogs<<<(nr + 7) / 8, 256, 0, st>>>(a, lda, b, ldb, lo, nr, gc, colcnt);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  BalCg hc{};
  for (int it = 1; it <= nr + 2; ++it) {
    k_bal_cg_a<<<1, kCgThreads, 0, st>>>(nr, gr, gc, pr, pc, cg);
    k_bal_mv_rows<<<dim3(rb, nch), 256, 0, st>>>(nr, E, pc, part, cg);
    k_bal_mv_rowsum<<<rb, 256, 0, st>>>(nr, nch, part, rowcnt, pr, qr, cg);
    k_bal_mv_cols<<<(nr + 7) / 8, 256, 0, st>>>(nr, E, pr, colcnt, pc, qc, cg);
    k_bal_cg_b<<<1, kCgThreads, 0, st>>>(nr, gr, gc, pr, pc, qr, qc, xr, xc, cg);
    e = cudaMemcpyAsync(&hc, cg, sizeof(BalCg), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    if (hc.done) break;
  }
  // exponents, limited so that no scaled row or column leaves the range
  k_bal_rowmax<<<dim3(rb, nchn), 256, 0, st>>>(a, lda, b, ldb, n, lo, nr, rab);
  k_bal_colmax<<<(nr + 7) / 8, 256, 0, st>>>(a, lda, b, ldb, lo, hi, cab);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  std::vector<double> hx(4 * (size_t)nr);
  e = cudaMemcpyAsync(hx.data(), xr, sizeof(double) * 2 * (size_t)nr, cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(hx.data() + 2 * (size_t)nr, cab, sizeof(double) * (size_t)nr, cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(hx.data() + 3 * (size_t)nr, rab, sizeof(double) * (size_t)nr, cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  const double sfmin = DBL_MIN;
  const int lsfmin = (int)(log10(sfmin) + 1.0);
  const int lsfmax = (int)(log10(1.0 / sfmin));
  std::vector<double> sc(2 * (size_t)nr);
  for (int k = 0; k < nr; ++k) {
    const double xrk = hx[k], xck = hx[nr + k], cabk = hx[2 * (size_t)nr + k], rabk = hx[3 * (size_t)nr + k];
    const int lrab = (int)(log10(rabk + sfmin) + 1.0);
    int ir = (int)(xrk + (xrk >= 0.0 ? 0.5 : -0.5));
    ir = std::min(std::max(ir, lsfmin), std::min(lsfmax, lsfmax - lrab));
    const int lcab = (int)(log10(cabk + sfmin) + 1.0);
    int jc = (int)(xck + (xck >= 0.0 ? 0.5 : -0.5));
    jc = std::min(std::max(jc, lsfmin), std::min(lsfmax, lsfmax - lcab));
    sc[k] = pow10i(ir);
    sc[nr + k] = pow10i(jc);
    lscale[lo + k] = sc[k];
    rscale[lo + k] = sc[nr + k];
  }
  e = cudaMemcpyAsync(gr, sc.data(), sizeof(double) * 2 * (size_t)nr, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  k_bal_apply<<<dim3((hi + 1 + 255) / 256, gy(n - lo)), 256, 0, st>>>(a, lda, b, ldb, n, lo, hi, gr, gr + nr);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(st);
}

cudaError_t ggbak_device(cudaStream_t st, char job, char side, int n, int ilo, int ihi, const double* lscale,
                         const double* rscale, int m, double* v, int64_t ldv) {
  job = (char)upper(job);
  side = (char)upper(side);
  if (n <= 0 || m <= 0 || job == 'N') return cudaSuccess;
  const double* s = (side == 'R') ? rscale : lscale;
  const int lo = ilo - 1, hi = ihi - 1;
  cudaError_t e;
  DevBuf buf;
  if ((job == 'S' || job == 'B') && lo != hi) {
    const int nr = hi - lo + 1;
    e = cudaMalloc(&buf.p, sizeof(double) * (size_t)nr);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(buf.p, s + lo, sizeof(double) * (size_t)nr, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    k_bak_scale<<<dim3((nr + 255) / 256, gy(m)), 256, 0, st>>>(v, ldv, m, lo, hi, (const double*)buf.p);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (job == 'P' || job == 'B') {
    // the row interchanges, last recorded first above ilo and in recorded
    // order below ihi, composed into one gather
    std::vector<int> src(n);
    for (int i = 0; i < n; ++i) src[i] = i;
    bool any = false;
    for (int i = lo - 1; i >= 0; --i) {
      const int k = (int)s[i] - 1;
      if (k != i && k >= 0 && k < n) { std::swap(src[i], src[k]); any = true; }
    }
    for (int i = hi + 1; i < n; ++i) {
      const int k = (int)s[i] - 1;
      if (k != i && k >= 0 && k < n) { std::swap(src[i], src[k]); any = true; }
    }
    if (any) {
      DevBuf w;
      e = cudaMalloc(&w.p, sizeof(double) * (size_t)n * m + sizeof(int) * (size_t)n);
      if (e != cudaSuccess) return e;
      double* W = (double*)w.p;
      int* dsrc = (int*)(W + (size_t)n * m);
      e = cudaMemcpyAsync(dsrc, src.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) return e;
      k_bak_gather<<<dim3((n + 255) / 256, gy(m)), 256, 0, st>>>(v, ldv, n, m, dsrc, W);
      k_bak_copy<<<dim3((n + 255) / 256, gy(m)), 256, 0, st>>>(W, n, m, v, ldv);
      e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      return cudaStreamSynchronize(st);
    }
  }
  return cudaStreamSynchronize(st);
}

}  // namespace qz
