/*
 * b200qz: B200-native multishift QZ (generalized real Schur form of a
 * Hessenberg-triangular pencil) behind the PDHGEQZ calling convention.
 *
 * Plain C ABI: pointers, sizes and characters only.  Every entry point is
 * exported from libb200qz.so (gevp-pdhgeqz_b200/libb200qz.so).
 *
 * Matrices are FP64 column-major.  Conventions follow the reference
 * routine PDHGEQZ (src/pdhgeqz/PDHGEQZ.f:35-214): on exit
 *   Q_in * H_in * Z_in^T = Q_out * S * Z_out^T,  the same for T and P,
 * S quasi upper triangular with standardised 2x2 blocks, P upper
 * triangular with non-negative diagonal (2x2 blocks: diagonal, positive),
 * and lambda_j = (ALPHAR(j) + i*ALPHAI(j)) / BETA(j).
 *
 * The steps either side of the solve have entries of their own:
 * balancing (b200qz_ggbal_*, b200qz_ggbak_*; DGGBAL/DGGBAK semantics),
 * Hessenberg-triangular reduction (b200qz_gghrd_*, DGGHRD semantics, and
 * the pdgghrd_ drop-in for the reference's PDGGHRD) and reordering of the
 * Schur form (b200qz_tgsen_*, DTGSEN semantics).
 */
#ifndef B200QZ_H
#define B200QZ_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct b200qz_ctx b200qz_ctx;

/* ------------------------------------------------------------------ */
/* Drop-in for the reference's Fortran entry point.                     */
/* ------------------------------------------------------------------ */

/* Replaces SUBROUTINE PDHGEQZ( JOB, COMPQ, COMPZ, N, ILO, IHI, H, DESCH,
 * T, DESCT, ALPHAR, ALPHAI, BETA, Q, DESCQ, Z, DESCZ, DWORK, LDWORK,
 * IWORK, LIWORK, INFO ) of src/pdhgeqz/PDHGEQZ.f:15-31, with the gfortran
 * by-reference convention and hidden CHARACTER lengths.  Only the 1x1
 * process grid is supported: H, T, Q, Z are full N x N local arrays with
 * leading dimension DESC(9).  DESC(5) = DESC(6) = NB >= 5 is required
 * (PDHGEQZ.f:396-399).  Workspace query: LDWORK = -1 or LIWORK = -1
 * returns the sizes in DWORK(1), IWORK(1) (PDHGEQZ.f:409-430).
 * INFO: -1 JOB, -2 COMPQ, -3 COMPZ, -4 N, -5 ILO, -6 IHI, -7 NB < 5,
 * -8 NB /= MB, -9 LDWORK, -10 LIWORK (PDHGEQZ.f:383-444), -(i*1000+9)
 * for a bad leading dimension of argument i; > 0 the index of the first
 * unconverged row (PDHGEQZ0.f:1207), also returned when no eigenvalue
 * deflates for "stall_limit" iterations; 10001 a CUDA error; 10002
 * non-finite entries in the active block. */
void pdhgeqz_(const char* job, const char* compq, const char* compz, const int* n, const int* ilo,
              const int* ihi, double* h, const int* desch, double* t, const int* desct, double* alphar,
              double* alphai, double* beta, double* q, const int* descq, double* z, const int* descz,
              double* dwork, const int* ldwork, int* iwork, const int* liwork, int* info,
              size_t len_job, size_t len_compq, size_t len_compz);

/* Replaces SUBROUTINE KKQZCONF( EPS ) (src/kkqz/kkqzconf.f:45-170), which
 * every reference caller invokes first (testing/EXRAND1.f:96-98) to fill
 * the COMMON parameter blocks.  Here the parameters live in a per-call
 * context, so this is an accepted no-op. */
void kkqzconf_(const double* eps);

/* ------------------------------------------------------------------ */
/* Native C entry points.                                                */
/* ------------------------------------------------------------------ */

/* Create / destroy a solver context on a CUDA device.  A context owns its
 * stream and device workspace; distinct contexts may be used from
 * different host threads concurrently. Returns 0 or a CUDA error code. */
int b200qz_create(b200qz_ctx** ctx, int device);
void b200qz_destroy(b200qz_ctx* ctx);

/* Solve with all arrays already resident on the device (one leading
 * dimension ld >= n for H, T, Q, Z).  job/compq/compz and ilo/ihi
 * (1-based) as in PDHGEQZ.  alphar/alphai/beta are device arrays of
 * length n.  Returns INFO (0 ok, > 0 unconverged row, < 0 bad argument,
 * 10001 CUDA error, 10002 non-finite entries, 10003 stopped by the
 * "aed_limit" parameter).  When T's largest entry is more than 2^30 away
 * from H's, T is scaled by a power of two during the iteration and scaled
 * back before returning. */
int b200qz_solve_dev(b200qz_ctx* ctx, char job, char compq, char compz, int n, int ilo, int ihi,
                     double* h, double* t, double* q, double* z, int ld,
                     double* alphar, double* alphai, double* beta);

/* Solve with host arrays (each with its own leading dimension); copies to
 * the device (buffers cached in the context and grown on demand), solves,
 * copies back.  Pinned host memory gives the fastest copies. */
int b200qz_solve_host(b200qz_ctx* ctx, char job, char compq, char compz, int n, int ilo, int ihi,
                      double* h, int ldh, double* t, int ldt, double* q, int ldq, double* z, int ldz,
                      double* alphar, double* alphai, double* beta);

/* Statistics of the last solve, written into out[0..nout):
 * 0 seconds (device time), 1 iterations, 2 AEDs, 3 AED deflations,
 * 4 sweeps, 5 chains, 6 windows, 7 endgames, 8 infinite-eigenvalue
 * steps, 9 shifts used, 10 update flops (FP64-equivalent), 11 window
 * kernel bytes; with B200QZ_PROFILE=1 set during the solve also device
 * milliseconds per phase: 12 scan, 13 AED, 14 AED updates, 15 chase,
 * 16 chase updates, 17 infinite-eigenvalue deflation, 18 finalisation,
 * and inside the AED kernel 19 small QZ, 20 reordering, 21 spike
 * reflector + RQ update, 22 Hessenberg-triangular re-reduction;
 * 23 kernel launches issued by the solve, 24 AED windows whose small QZ
 * did not converge (they deflate nothing and supply diagonal shifts),
 * 25 sweeps run with exceptional shifts (after 40 iterations without
 * deflation), 26 rows left unconverged, 27/28 active block where an
 * "aed_limit" stopped the solve, 29 deflated fraction of the last AED
 * window, 30 AED decisions taken by the learned policy, 31 algorithmic
 * bytes of the AED/endgame window kernels (6*8*w^2 per window of order w),
 * 32 their launches, 33 algorithmic bytes of the chase windows, 34 chase
 * launches (one per wave of concurrent windows); with B200QZ_PROFILE=1
 * also 35 double-shift steps, 36 block swaps, 37 re-reduction rotation
 * pairs and 38 multishift window sweeps executed inside the AED kernels.
 * Returns the number of values written. */
int b200qz_get_stats(const b200qz_ctx* ctx, double* out, int nout);

/* Tunables: nw_max (AED window), w_chase (chase window), nmin (blocks
 * solved by one CTA), nibble (percent), ns_max (shift cap), maxit factor.
 * A value < 0 keeps the current setting. Returns 0 or -i for argument i. */
int b200qz_set_params(b200qz_ctx* ctx, int nw_max, int w_chase, int nmin, int nibble, int ns_max,
                      int maxit_factor);

/* Set one tunable by name: "nw_max", "w_chase", "nmin", "nibble",
 * "ns_max", "maxit_factor", "chain_max" (bulges per chain), "aed_nskip"
 * (AED spike test stops after this many consecutive undeflatable blocks,
 * 0 = whole window), "max_wave" (chains chased concurrently, 1..8),
 * "stall_limit" (iterations without deflation before INFO > 0),
 * "split" (0, 7 or 8 INT8 Ozaki slices for the off-diagonal updates),
 * "aed_threads" (32, 64 or 128), "upd_persist" (0 or 1), "aed_limit"
 * (stop before that AED, INFO 10003), "aed_swap_fail" (1: every block swap
 * inside the AED reports failure, which exercises the swap-failure branch
 * of the reference, qzearly.f:321-326).
 * Returns 0, -2 for an unknown name, -3 for a value out of range. */
int b200qz_set_param(b200qz_ctx* ctx, const char* name, double value);

/* ------------------------------------------------------------------ */
/* Learned (nw, ns) policy: replaces the fixed tuning table of          */
/* PIPARMQ / PILAENVX (src/pdhgeqz/piparmq.f:438-535) at every AED       */
/* decision; the table stays the fallback.                              */
/* ------------------------------------------------------------------ */

/* Number of FP32 parameters of the 64-128-128-2 MLP (flat, row-major
 * out x in: W1[128x64] b1[128] W2[128x128] b2[128] W3[2x128] b3[2]). */
int b200qz_policy_nparams(void);

/* Load the MLP's parameters (host array of b200qz_policy_nparams() floats)
 * into the context; from then on every AED decision takes nw and ns from
 * the network (outputs y0, y1 clamped to [0,1]: nw = 16 + 64*y0, at most
 * the AED window limit; ns = y1*nw, even, at least 2).  params = NULL or
 * nparams = 0 switches back to the table.  Returns 0, -2 (non-finite
 * parameter), -3 (wrong count) or 10001. */
int b200qz_set_policy(b200qz_ctx* ctx, const float* params, int nparams);

/* The 64 features of the active block [ktop, kbot] (0-based) of the device
 * matrix h (leading dimension ld): 62 log-spaced bins over the distance
 * from the bottom of the mean -log10(|h(k+1,k)|/(|h(k,k)|+|h(k+1,k+1)|))/16
 * (clipped to [0,1]), log2(nh)/14 and lastfrac (the deflated fraction of
 * the previous AED window).  out: host array of 64 floats. */
int b200qz_policy_features(b200qz_ctx* ctx, const double* h, int ld, int ktop, int kbot, double lastfrac,
                           float* out);

/* MLP forward and backward on device buffers (FP32, stream = cudaStream_t
 * or NULL): x[batch x 64], a1, a2 [batch x 128] activations, y[batch x 2];
 * the backward pass of the loss mean((y - target)^2) over batch x 2 fills
 * dy[batch x 2], d2, d1 [batch x 128] and grad[nparams]. */
int b200qz_mlp_forward(const float* params, const float* x, int batch, float* a1, float* a2, float* y,
                       void* stream);
int b200qz_mlp_backward(const float* params, const float* x, const float* target, int batch, const float* a1,
                        const float* a2, const float* y, float* dy, float* d2, float* d1, float* grad,
                        void* stream);

/* Train the MLP in place (params: device, nparams floats) with Adam on the
 * device for `epochs` full-batch steps; loss (host, may be NULL) receives
 * the final mean squared error. */
int b200qz_mlp_train(float* params, const float* x, const float* target, int batch, int epochs, float lr,
                     float* loss);

/* ------------------------------------------------------------------ */
/* Batched independent pencils (sizes may differ).                      */
/* ------------------------------------------------------------------ */

/* Reduce count independent pencils to generalized Schur form with Q, Z in
 * one persistent launch (CUDA-graph captured, replayed while the layout
 * stays the same).  Device buffers h, t, q, z hold pencil p (size n[p],
 * leading dimension n[p]) at offset moff[p] (in doubles); its eigenvalues
 * go to alphar/alphai/beta at offset eoff[p]; info[p] (device) is 0 or the
 * 1-based row that did not converge.  n, moff, eoff are host arrays.
 * Returns 0, a negative argument error, or 10001 (CUDA error).  No
 * reference counterpart (the reference solves one pencil per call). */
int b200qz_solve_batched_dev(b200qz_ctx* ctx, int count, const int* n, const long long* moff,
                             const long long* eoff, double* h, double* t, double* q, double* z,
                             double* alphar, double* alphai, double* beta, int* info);

/* Device seconds of the last batched launch. */
double b200qz_batched_seconds(const b200qz_ctx* ctx);

/* Autotune the batched launch (threads per CTA, largest pencil kept in
 * shared memory, CTAs per SM) on a copy of `sample` pencils spread over the
 * size range of the batch; keeps the fastest configuration in the context.
 * h, t are device buffers laid out as for b200qz_solve_batched_dev; they are
 * not modified.  best_seconds (host, may be NULL) receives the best time. */
int b200qz_batched_autotune(b200qz_ctx* ctx, int count, const int* n, const long long* moff,
                            const double* h, const double* t, int sample, double* best_seconds);

/* Current batched configuration. */
int b200qz_batched_config(const b200qz_ctx* ctx, int* threads, int* smem_max, int* ctas_per_sm);

/* Batched solve that allocates no memory, for callers that cannot call
 * cudaMalloc: code running inside another library's memory pool or
 * allocator, hosts that reserve the device heap up front, and loops where
 * an allocation could block.  Same arguments and results as
 * b200qz_solve_batched_dev (device buffers h, t, q, z, alphar, alphai,
 * beta, info; host arrays n, moff, eoff), but no context and its own return
 * codes (below): it runs on the current device and on `stream` (a
 * cudaStream_t, NULL for the default stream) and returns without waiting
 * for the GPU.  n, moff and eoff in ordinary (pageable) memory may be
 * reused as soon as the call returns; page-locked ones are read when the
 * stream reaches the copy and must stay unchanged until then.  The batch
 * descriptors and the work-queue counter live in one fixed array in the
 * library's device memory (about 96 KB, held by every GPU that loads the
 * library until the process exits), so at most 4096 pencils per call: a
 * larger count returns -2.  The first call on a device sets that device up
 * (it looks up the array's device address and raises the kernel's shared-
 * memory limit), so make it before any stream capture.  All calls share
 * the array: calls whose work overlaps on the GPU (different streams, or
 * host threads racing) corrupt each other's batches.  Returns 0, -1 bad
 * count, -2 count above 4096, -3 a size outside 1..46340, or 10001 on a
 * CUDA error of this call.  No counterpart in the reference. */
int b200qz_solve_batched_noalloc(int count, const int* n, const long long* moff, const long long* eoff,
                                 double* h, double* t, double* q, double* z, double* alphar, double* alphai,
                                 double* beta, int* info, void* stream);

/* ------------------------------------------------------------------ */
/* Kernel-level entry points (device pointers), for parity tests.       */
/* ------------------------------------------------------------------ */

/* AED on the window H(kwtop:kbot, kwtop:kbot) (0-based, inclusive) of the
 * active block starting at ktop; the role of PDHGEQZ2 + QZEARLY
 * (PDHGEQZ2.f:315-389, qzearly.f:229-449) without the off-diagonal
 * updates.  qw, zw: nw x nw outputs (ld nw); shifts: 3*nw outputs
 * (alphar, alphai, beta of the undeflated part, each at stride nw);
 * info3 (host): {undeflated m, status, transformed}.  When ktop == kwtop
 * the whole window is reduced to Schur form (the PDHGEQZ4/KKQZ role). */
int b200qz_aed_window(b200qz_ctx* ctx, double* h, double* t, int ld, int ktop, int kwtop, int kbot,
                      double* qw, double* zw, double* shifts, int* info3);

/* Chase one chain of bulges through the window H(w:w+wk, w:w+wk); the
 * role of PDHGEQZB + DHGEQZ5 (PDHGEQZB.f:356-408, DHGEQZ5.f:128-250)
 * and, for bulges with intro = 1, PDHGEQZA's introduction.  bulges is a
 * host array of nb records {base, tlo, thi, intro} (int[4]) and coef a
 * host array of nb x {c2, c1, c0}.  last = last active row inside the
 * window (window coordinates).  u, v: wk x wk outputs (ld wk). */
int b200qz_chase_window(b200qz_ctx* ctx, double* h, double* t, int ld, int w, int wk, int last,
                        const int* bulges, const double* coef, int nb, int tmax, double* u, double* v);

/* In-place update of a slab with a k x k factor (the role of PDHGEQZ6,
 * PDHGEQZ6.f:276-380): side 'L': M(r0:r0+k, c0:c0+len) <- W^T M(...);
 * side 'R': M(r0:r0+len, c0:c0+k) <- M(...) W. */
int b200qz_update(b200qz_ctx* ctx, char side, double* m, int ldm, int r0, int c0, int len,
                  const double* w, int ldw, int k);

/* The same update through the split-precision path: the slab and W are
 * split into `slices` (7 or 8) signed 7-bit INT8 digit matrices (Ozaki
 * scheme, exact INT32 accumulation on the tensor cores, tcgen05.mma
 * kind::i8), and the significant slice products (28 or 36) are recombined
 * in FP64.  Error per entry about 2^-48 (7 slices) or 2^-55 (8 slices)
 * times |a_i|_max |w_j|_max k.  k <= 80.  Returns 0, -1/-2 bad argument,
 * 10001 CUDA error, 10004 tensor-core wait timed out.  Replaces the same
 * DGEMM of PDHGEQZ6.f:296-375.  Solver parameter "split" = 7 or 8 routes
 * every off-diagonal update of windows up to 80 through this path. */
int b200qz_update_split(b200qz_ctx* ctx, char side, double* m, int ldm, int r0, int c0, int len, const double* w,
                        int ldw, int k, int slices);

/* ------------------------------------------------------------------ */
/* Balancing: the step that produces ILO/IHI for PDHGEQZ                */
/* ------------------------------------------------------------------ */

/* Balance a general pencil (A, B) with the semantics of LAPACK DGGBAL,
 * whose ILO/IHI output the reference's driver takes (PDHGEQZ.f:155-161;
 * DGGBAL itself is LAPACK's, not the reference's).  job: 'N' nothing,
 * 'P' permute only, 'S' scale only, 'B' both.  Permutation moves rows
 * whose nonzeros lie in at most one active column to the bottom (searched
 * from the bottom) and then columns whose nonzeros lie in at most one
 * active row to the top (searched from the left), so that A and B are
 * upper triangular outside rows/columns ILO..IHI.  Scaling multiplies
 * rows and columns ILO..IHI by powers of ten chosen by Ward's
 * least-squares method (conjugate gradients, at most IHI-ILO+3
 * iterations).  ilo/ihi are returned 1-based (ilo = 1, ihi = 0 for
 * n = 0); lscale/rscale (host arrays of n doubles) hold, for positions
 * outside ILO..IHI, the 1-based row/column interchanged with that
 * position, and inside it the row/column scale factors.  The _dev form
 * takes device arrays (transformed in place on the context's stream),
 * the _host form host arrays.  Returns 0; -1 bad job, -2 n < 0, -4 lda,
 * -6 ldb (DGGBAL's argument positions); 10001 on a CUDA error. */
int b200qz_ggbal_dev(b200qz_ctx* ctx, char job, int n, double* a, int lda, double* b, int ldb, int* ilo, int* ihi,
                     double* lscale, double* rscale);
int b200qz_ggbal_host(b200qz_ctx* ctx, char job, int n, double* a, int lda, double* b, int ldb, int* ilo, int* ihi,
                      double* lscale, double* rscale);

/* Back-transform the n x m matrix V (eigenvectors, or the Schur vectors
 * Q (side 'L') / Z (side 'R') of the balanced pencil) with the semantics
 * of LAPACK DGGBAK: rows ILO..IHI scaled by lscale ('L') or rscale ('R')
 * when job is 'S' or 'B', then the recorded row interchanges undone when
 * job is 'P' or 'B'.  lscale/rscale are the host arrays ggbal returned.
 * Returns 0; -1 job, -2 side, -3 n, -4 ilo, -5 ihi, -8 m, -10 ldv
 * (DGGBAK's argument positions); 10001 on a CUDA error. */
int b200qz_ggbak_dev(b200qz_ctx* ctx, char job, char side, int n, int ilo, int ihi, const double* lscale,
                     const double* rscale, int m, double* v, int ldv);
int b200qz_ggbak_host(b200qz_ctx* ctx, char job, char side, int n, int ilo, int ihi, const double* lscale,
                      const double* rscale, int m, double* v, int ldv);

/* ------------------------------------------------------------------ */
/* Reordering: the step after the solve                                 */
/* ------------------------------------------------------------------ */

/* Reorder a generalized real Schur form (S, T) (standardised, as the
 * solve returns it) and its Schur vectors so that the eigenvalues
 * flagged in select (host array of n ints; a 2x2 block moves when either
 * of its flags is set) lead, with the semantics of LAPACK DTGSEN for
 * IJOB 0, 1, 3 and 5 (the role of the reference's PDTGSEN / PDTGORD,
 * src/reorder/PDTGSEN.f:1, PDTGORD.f:1).  Selected blocks move up by
 * adjacent block swaps inside windows of up to 80 rows on one CTA; the
 * windows' orthogonal factors are applied to the rest of S, T, Q, Z on the
 * tensor cores.  1x1 blocks with a negative T entry then have their rows
 * of S and T and column of Q negated.  alphar/alphai/beta receive the
 * reordered eigenvalues; m the dimension of the selected deflating
 * subspaces; for ijob = 1 and 5, pl/pr the reciprocal norms of the
 * projections onto the left/right deflating subspaces (from the
 * generalized Sylvester equation S11 R - L S22 = S12, T11 R - L T22 =
 * T12), else 1; for ijob = 3 and 5, dif[0..1] the 1-norm estimates of
 * Difu and Difl (DTGSEN's DIF: the separations of (S11, T11) and
 * (S22, T22), from Higham's 1-norm estimator over generalized Sylvester
 * solves and their transposes; ||(S, T)||_F when m is 0 or n), else dif
 * (may be NULL) is not written.  info = 1 when a swap was rejected (the
 * pair is then partly reordered).  ijob 2 and 4 (the Frobenius-norm Dif
 * estimates) are not provided (-1).  The _dev form takes device
 * arrays (alphar/alphai/beta on the device too), the _host form host
 * arrays; counts (may be NULL) receives {swaps, windows}.  Returns 0;
 * -1 ijob, -5 n, -7 lds, -9 ldt, -14 ldq, -16 ldz (DTGSEN's argument
 * positions); 10001 on a CUDA error. */
int b200qz_tgsen_dev(b200qz_ctx* ctx, int ijob, int wantq, int wantz, const int* select, int n, double* s, int lds,
                     double* t, int ldt, double* q, int ldq, double* z, int ldz, double* alphar, double* alphai,
                     double* beta, int* m, double* pl, double* pr, double* dif, int* info, int* counts);
int b200qz_tgsen_host(b200qz_ctx* ctx, int ijob, int wantq, int wantz, const int* select, int n, double* s, int lds,
                      double* t, int ldt, double* q, int ldq, double* z, int ldz, double* alphar, double* alphai,
                      double* beta, int* m, double* pl, double* pr, double* dif, int* info);

/* Hessenberg-triangular reduction (LAPACK DGGHRD semantics; replaces the
 * reference's PDGGHRD, src/ab2ht/PDGGHRD.f:13, the step before the solve
 * at examples/EXRAND2.f:334).  B must be upper triangular on entry (its
 * strict lower triangle is set to zero).  Reduces A to upper Hessenberg
 * form in columns ilo..ihi-2 (1-based; A is assumed upper triangular
 * outside rows/columns ilo..ihi) by Givens rotations in LAPACK's order and
 * sign convention, keeping B upper triangular: Q^T A Z = H, Q^T B Z = T.
 * compq / compz: 'N' Q / Z not referenced, 'I' set to the orthogonal
 * factor, 'V' multiplied into the given matrix (Q1 Q, Z1 Z).  The _dev
 * form takes device arrays, the _host form host arrays.  Returns 0;
 * -1 compq, -2 compz, -3 n, -4 ilo, -5 ihi, -7 lda, -9 ldb, -11 ldq,
 * -13 ldz (DGGHRD's argument positions); 10001 on a CUDA error.  The
 * parameter "hr_win" (b200qz_set_param, 2..160, default 128) sets the
 * rotation pairs per shared-memory window. */
int b200qz_gghrd_dev(b200qz_ctx* ctx, char compq, char compz, int n, int ilo, int ihi, double* a, int lda, double* b,
                     int ldb, double* q, int ldq, double* z, int ldz);
int b200qz_gghrd_host(b200qz_ctx* ctx, char compq, char compz, int n, int ilo, int ihi, double* a, int lda, double* b,
                      int ldb, double* q, int ldq, double* z, int ldz);

/* Drop-in for the reference's PDGGHRD on a 1x1 process grid
 * (src/ab2ht/PDGGHRD.f:13-31): host arrays with ScaLAPACK descriptors
 * (LLD_ = desc[8]), hidden CHARACTER lengths.  Like the reference, N <= 1
 * returns at once; LWORK = -1 returns DESCA(MB_) in WORK(1); INFO -1
 * COMPQ, -2 COMPZ, -3 N, -4 ILO, -5 IHI, -6 MB_ != NB_, -7 LWORK < MB_.
 * Q is returned transposed, as the reference returns it: on exit Q holds
 * G Q_in, where G is the product of the row rotations (so with COMPQ = 'I'
 * the caller's A = Q^T H Z^T). */
void pdgghrd_(const char* compq, const char* compz, const int* n, const int* ilo, const int* ihi, double* a,
              const int* desca, double* b, const int* descb, double* q, const int* descq, double* z, const int* descz,
              double* work, const int* lwork, int* info, size_t len_compq, size_t len_compz);

#ifdef __cplusplus
}
#endif

#endif /* B200QZ_H */
