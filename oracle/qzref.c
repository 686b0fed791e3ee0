/*
 * qzref.c -- CPU restatement of the reference's multishift QZ path on a
 * 1x1 process grid.  TEST INFRASTRUCTURE ONLY: the oracle tests/ compare
 * the GPU path with, and bench.py's timed CPU baseline ("port").  The
 * product (libb200qz.so) never links or calls it.
 *
 * Parity status: the reference ships no golden vectors (testing/EXRAND1.f
 * only checks residual thresholds on non-reproducible inputs), so this
 * restatement is pinned against LAPACK DHGEQZ -- the serial QZ whose call
 * the reference keeps commented out in src/kkqz/qzearly.f:224-227 -- by
 * eigenvalue sets and backward errors (tests/test_cpu_qzref.py).
 *
 * LAPACK/BLAS leaves are those the reference calls (DLARFG, DLARTG, DROT,
 * DGEMM, DGERQF/DORGRQ, DTGEXC, DGGHRD, DLAGV2, DHGEQZ), resolved in the
 * OpenBLAS build bundled with scipy (symbols prefixed scipy_).
 *
 * Simplifications relative to the reference (each noted where it applies):
 *  - window Schur forms use LAPACK DHGEQZ instead of QZDACK/KKQZ
 *    (qzearly.f:229-236, PDHGEQZ4.f:329-372);
 *  - chase windows are always of the "cross border" kind of PDHGEQZ5
 *    (MOVEDIST = CHAINSIZE+1, WSIZE = 2*(CHAINSIZE+1), PDHGEQZ5.f:454-468);
 *  - interior infinite eigenvalues are chased to the bottom with the
 *    unwindowed Givens sequence instead of PDHGEQZ8/9's windows.
 * Column-major storage, 1-based comments, 0-based code.
 */
#define _POSIX_C_SOURCE 199309L
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static double wall_seconds(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ---- LAPACK / BLAS through scipy's OpenBLAS ------------------------------ */
typedef size_t flen;
extern void scipy_dlarfg_(const int* n, double* alpha, double* x, const int* incx, double* tau);
extern void scipy_dlartg_(const double* f, const double* g, double* c, double* s, double* r);
extern void scipy_drot_(const int* n, double* x, const int* incx, double* y, const int* incy, const double* c,
                        const double* s);
extern void scipy_dgemm_(const char* ta, const char* tb, const int* m, const int* n, const int* k,
                         const double* alpha, const double* a, const int* lda, const double* b, const int* ldb,
                         const double* beta, double* c, const int* ldc, flen, flen);
extern void scipy_dgerqf_(const int* m, const int* n, double* a, const int* lda, double* tau, double* work,
                          const int* lwork, int* info);
extern void scipy_dorgrq_(const int* m, const int* n, const int* k, double* a, const int* lda, const double* tau,
                          double* work, const int* lwork, int* info);
extern void scipy_dhgeqz_(const char* job, const char* compq, const char* compz, const int* n, const int* ilo,
                          const int* ihi, double* h, const int* ldh, double* t, const int* ldt, double* ar,
                          double* ai, double* be, double* q, const int* ldq, double* z, const int* ldz,
                          double* work, const int* lwork, int* info, flen, flen, flen);
extern void scipy_dtgexc_(const int* wantq, const int* wantz, const int* n, double* a, const int* lda, double* b,
                          const int* ldb, double* q, const int* ldq, double* z, const int* ldz, int* ifst, int* ilst,
                          double* work, const int* lwork, int* info);
extern void scipy_dgghrd_(const char* cq, const char* cz, const int* n, const int* ilo, const int* ihi, double* a,
                          const int* lda, double* b, const int* ldb, double* q, const int* ldq, double* z,
                          const int* ldz, int* info, flen, flen);
extern void scipy_dlagv2_(double* a, const int* lda, double* b, const int* ldb, double* ar, double* ai, double* be,
                          double* csl, double* snl, double* csr, double* snr);
extern double scipy_dlamch_(const char* c, flen);

static const int I1 = 1;

#define M(A, ld, i, j) ((A)[(size_t)(i) + (size_t)(j) * (size_t)(ld)])

static double dmax(double a, double b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

typedef struct {
  int n, ld;
  double *H, *T, *Q, *Z;
  int wantq, wantz;
  double ulp, smlnum, safmin, ttol, htol;
  int nb;  /* descriptor block size (tuning hint) */
  /* counters */
  long iters, aeds, sweeps, smallsub, infs;
  double upd_flops;
  /* bounded runs (CPU-baseline samples): stop before AED number aed_limit
     (-1: never); aed_clock[k] receives the wall-clock seconds since the
     start of the solve at which AED k began (up to aed_cap entries) */
  long aed_limit;
  double* aed_clock;
  long aed_cap;
  double t_start;
} Ctx;

/* ---- QZFCOL (src/kkqz/qzfcol.f:1-116) -----------------------------------
 * First column (multiple of) of the shift polynomial for NSHIFT shifts
 * (NSHIFT even, <= 12); H, T the leading (NSHIFT+1)-square parts. */
static void qzfcol(int nshift, const double* sr, const double* si, const double* sb, const double* H, int ldh,
                   const double* T, int ldt, double* v) {
  enum { L = 13 };
  double tmp[L * L], cs1[13], sn1[13], cs2[13], sn2[13], cse = 1, sne = 0, scal, alpha;
  int ngiv = 0;
#define TM(i, j) tmp[(i) + (j) * L]
  for (int I = nshift; I >= 2; I -= 2) {
    int i = I - 1; /* 0-based index of shift I */
    if (ngiv > 0) {
      for (int c = 0; c <= ngiv; ++c)
        for (int r = 0; r <= ngiv; ++r) TM(r, c) = M(T, ldt, r, c);
      for (int J = ngiv; J >= 1; --J) {
        int j = J - 1, len = ngiv - J + 2;
        scipy_drot_(&len, &TM(j, j), &(int){L}, &TM(j + 1, j), &(int){L}, &cs1[j], &sn1[j]);
        alpha = TM(j + 1, j + 1);
        scipy_dlartg_(&alpha, &TM(j + 1, j), &cs2[j], &sn2[j], &TM(j + 1, j + 1));
        sn2[j] = -sn2[j];
        int jl = J;
        scipy_drot_(&jl, &TM(0, j), &I1, &TM(0, j + 1), &I1, &cs2[j], &sn2[j]);
      }
      scal = TM(0, 0);
    } else {
      scal = M(T, ldt, 0, 0);
    }
    for (int c = 0; c < ngiv + 2; ++c)
      for (int r = 0; r < ngiv + 2; ++r) TM(r, c) = M(H, ldh, r, c);
    for (int J = 1; J <= ngiv + 2; ++J) {
      int j = J - 1;
      int len = imin(J + 1, ngiv + 2);
      for (int r = 0; r < len; ++r) TM(r, j) *= sb[i];
      for (int r = 0; r < J; ++r) TM(r, j) -= sr[i] * M(T, ldt, r, j);
    }
    for (int J = ngiv; J >= 1; --J) {
      int j = J - 1, len = ngiv + 2;
      scipy_drot_(&len, &TM(0, j), &I1, &TM(0, j + 1), &I1, &cs2[j], &sn2[j]);
    }
    for (int J = ngiv + 1; J >= 1; --J) {
      int j = J - 1;
      alpha = TM(j, 0);
      scipy_dlartg_(&alpha, &TM(j + 1, 0), &cs2[j], &sn2[j], &TM(j, 0));
    }
    ngiv += 1;
    double g = si[i] * scal;
    scipy_dlartg_(&TM(0, 0), &g, &cse, &sne, &alpha);
    for (int c = 0; c <= ngiv; ++c)
      for (int r = 0; r <= ngiv; ++r) TM(r, c) = M(T, ldt, r, c);
    for (int J = ngiv; J >= 1; --J) {
      int j = J - 1, len = ngiv - J + 2;
      scipy_drot_(&len, &TM(j, j), &(int){L}, &TM(j + 1, j), &(int){L}, &cs2[j], &sn2[j]);
      alpha = TM(j + 1, j + 1);
      scipy_dlartg_(&alpha, &TM(j + 1, j), &cs2[j], &sn2[j], &TM(j + 1, j + 1));
      sn2[j] = -sn2[j];
      int jl = J;
      scipy_drot_(&jl, &TM(0, j), &I1, &TM(0, j + 1), &I1, &cs2[j], &sn2[j]);
    }
    {
      double f = cse, gg = -sne * TM(0, 0);
      scipy_dlartg_(&f, &gg, &cse, &sne, &alpha);
      sne = -sne;
    }
    for (int c = 0; c < ngiv + 2; ++c)
      for (int r = 0; r < ngiv + 2; ++r) TM(r, c) = M(H, ldh, r, c);
    for (int J = 1; J <= ngiv + 2; ++J) {
      int j = J - 1;
      int len = imin(J + 1, ngiv + 2);
      for (int r = 0; r < len; ++r) TM(r, j) *= sb[i - 1];
      for (int r = 0; r < J; ++r) TM(r, j) -= sr[i - 1] * M(T, ldt, r, j);
    }
    for (int J = ngiv; J >= 1; --J) {
      int j = J - 1, len = ngiv + 2;
      scipy_drot_(&len, &TM(0, j), &I1, &TM(0, j + 1), &I1, &cs2[j], &sn2[j]);
    }
    /* DLASET('All', NGIV+2, NGIV+1, 0, -SI(I-1), TMP(1,2)) */
    for (int c = 1; c <= ngiv + 1; ++c)
      for (int r = 0; r < ngiv + 2; ++r) TM(r, c) = (r == c - 1) ? -si[i - 1] : 0.0;
    for (int J = ngiv - 1; J >= 1; --J) {
      int j = J - 1, len = ngiv;
      scipy_drot_(&len, &TM(0, j + 1), &I1, &TM(0, j + 2), &I1, &cs1[j], &sn1[j]);
    }
    {
      int len = ngiv + 2;
      scipy_drot_(&len, &TM(0, 0), &I1, &TM(0, 1), &I1, &cse, &sne);
    }
    if (I > 2) {
      for (int J = ngiv + 1; J >= 1; --J) {
        int j = J - 1;
        alpha = TM(j, 0);
        scipy_dlartg_(&alpha, &TM(j + 1, 0), &cs1[j], &sn1[j], &TM(j, 0));
      }
      ngiv += 1;
    } else {
      for (int r = 0; r < ngiv + 2; ++r) v[r] = TM(r, 0);
    }
  }
#undef TM
}

/* ---- INVHSE (src/kkqz/invhse.f:1-75, PARA_ITOPP=2: RQ branch) ----------- */
static void invhse3(const double* T, int ldt, double* tau, double* v) {
  double tmp[9], nu[3], work[64];
  int n = 3, lw = 64, info;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) tmp[r + 3 * c] = M(T, ldt, r, c);
  scipy_dgerqf_(&n, &n, tmp, &n, nu, work, &lw, &info);
  scipy_dorgrq_(&n, &n, &n, tmp, &n, nu, work, &lw, &info);
  for (int i = 0; i < 3; ++i) v[i] = tmp[0 + 3 * i];
  int two = 2;
  scipy_dlarfg_(&n, &v[0], &v[1], &I1, tau);
  (void)two;
  v[0] = 1.0;
}

/* apply a 3-reflector (v(0)=1) */
static inline void refl3(double tau, const double* v, double* a0, double* a1, double* a2) {
  double t = tau * (*a0 + v[1] * *a1 + v[2] * *a2);
  *a0 -= t;
  *a1 -= t * v[1];
  *a2 -= t * v[2];
}

/* ---- DHGEQZ5 (src/pdhgeqz/DHGEQZ5.f:128-275) ----------------------------
 * Chase one bulge NSTEP-NCOL+1 columns down the window (A,B) of size
 * wsize (ld lda), starting at row index IR (0-based offset).  eshift points
 * to the bulge's two shifts (for reintroduction of a collapsed bulge).
 * Q, Z (ld ldqz) accumulate the left / right transformations. */
static void dhgeqz5(const Ctx* C, int nstep, double* A, int lda, double* B, int ldb, int ir, int ncol, int wsize,
                    const double* sr, const double* si, const double* sb, double* Q, double* Z, int ldqz) {
  double v[3], v1[3], tau, tau1;
  for (int J = 2 + ir; J <= nstep - ncol + ir; ++J) {
    int j = J - 1; /* 0-based row of the reflector */
    v[0] = M(A, lda, j, j - 1);
    v[1] = M(A, lda, j + 1, j - 1);
    v[2] = M(A, lda, j + 2, j - 1);
    int three = 3;
    scipy_dlarfg_(&three, &v[0], &v[1], &I1, &tau);
    if (M(A, lda, j + 2, j - 1) != 0.0 || M(A, lda, j + 2, j) != 0.0 || M(A, lda, j + 2, j + 1) == 0.0) {
      M(A, lda, j, j - 1) = v[0];
      M(A, lda, j + 1, j - 1) = 0.0;
      M(A, lda, j + 2, j - 1) = 0.0;
    } else {
      /* collapsed bulge: try to reintroduce (DHGEQZ5.f:141-189) */
      qzfcol(2, sr, si, sb, &M(A, lda, j, j), lda, &M(B, ldb, j, j), ldb, v1);
      scipy_dlarfg_(&three, &v1[0], &v1[1], &I1, &tau1);
      M(A, lda, j + 1, j - 1) = 0.0;
      M(A, lda, j + 2, j - 1) = 0.0;
      double refsum = tau1 * (M(A, lda, j, j - 1) + v1[1] * M(A, lda, j + 1, j - 1));
      if (fabs(M(A, lda, j + 1, j - 1) - refsum * v1[1]) + fabs(refsum * v1[2]) >
          C->ulp * (fabs(M(A, lda, j - 1, j - 1)) + fabs(M(A, lda, j, j)) + fabs(M(A, lda, j + 1, j + 1)))) {
        M(A, lda, j, j - 1) = v[0];
      } else {
        M(A, lda, j, j - 1) = M(A, lda, j, j - 1) - refsum;
        tau = tau1;
        v[1] = v1[1];
        v[2] = v1[2];
      }
    }
    v[0] = 1.0;
    for (int jc = j; jc < wsize; ++jc) {
      refl3(tau, v, &M(A, lda, j, jc), &M(A, lda, j + 1, jc), &M(A, lda, j + 2, jc));
      refl3(tau, v, &M(B, ldb, j, jc), &M(B, ldb, j + 1, jc), &M(B, ldb, j + 2, jc));
    }
    for (int jr = 0; jr < wsize; ++jr)
      refl3(tau, v, &M(Q, ldqz, jr, j), &M(Q, ldqz, jr, j + 1), &M(Q, ldqz, jr, j + 2));
    double vv[3];
    invhse3(&M(B, ldb, j, j), ldb, &tau, vv);
    for (int jr = 0; jr < imin(J + 3, wsize); ++jr)
      refl3(tau, vv, &M(A, lda, jr, j), &M(A, lda, jr, j + 1), &M(A, lda, jr, j + 2));
    for (int jr = 0; jr < imin(J + 2, wsize); ++jr)
      refl3(tau, vv, &M(B, ldb, jr, j), &M(B, ldb, jr, j + 1), &M(B, ldb, jr, j + 2));
    M(B, ldb, j + 1, j) = 0.0;
    M(B, ldb, j + 2, j) = 0.0;
    for (int jr = 0; jr < wsize; ++jr)
      refl3(tau, vv, &M(Z, ldqz, jr, j), &M(Z, ldqz, jr, j + 1), &M(Z, ldqz, jr, j + 2));
  }
  /* vigilant deflation check (DHGEQZ5.f:254-275) */
  for (int J = 2 + ir; J <= nstep - ncol + ir; ++J) {
    int j = J - 1;
    if (M(A, lda, j, j - 1) != 0.0) {
      double tst1 = fabs(M(A, lda, j - 1, j - 1)) + fabs(M(A, lda, j, j));
      if (fabs(M(A, lda, j, j - 1)) <= dmax(C->smlnum, C->ulp * tst1)) {
        double h12 = dmax(fabs(M(A, lda, j, j - 1)), fabs(M(A, lda, j - 1, j)));
        double h21 = fmin(fabs(M(A, lda, j, j - 1)), fabs(M(A, lda, j - 1, j)));
        double h11 = dmax(fabs(M(A, lda, j, j)), fabs(M(A, lda, j - 1, j - 1) - M(A, lda, j, j)));
        double h22 = fmin(fabs(M(A, lda, j, j)), fabs(M(A, lda, j - 1, j - 1) - M(A, lda, j, j)));
        double scl = h11 + h12;
        double tst2 = h22 * (h11 / scl);
        if (tst2 == 0.0 || h21 * (h12 / scl) <= dmax(C->smlnum, C->ulp * tst2)) M(A, lda, j, j - 1) = 0.0;
      }
    }
  }
}

/* push a bulge off the bottom of the window (PDHGEQZB.f:373-406) */
static void pushoff(double* A, int lda, double* B, int ldb, int ws, double* U, double* V, int ldqz) {
  double c, s, temp;
  int two = 2;
  temp = M(A, lda, ws - 2, ws - 3);
  scipy_dlartg_(&temp, &M(A, lda, ws - 1, ws - 3), &c, &s, &M(A, lda, ws - 2, ws - 3));
  M(A, lda, ws - 1, ws - 3) = 0.0;
  scipy_drot_(&two, &M(A, lda, ws - 2, ws - 2), &lda, &M(A, lda, ws - 1, ws - 2), &lda, &c, &s);
  scipy_drot_(&two, &M(B, ldb, ws - 2, ws - 2), &ldb, &M(B, ldb, ws - 1, ws - 2), &ldb, &c, &s);
  scipy_drot_(&ws, &M(U, ldqz, 0, ws - 2), &I1, &M(U, ldqz, 0, ws - 1), &I1, &c, &s);
  temp = M(B, ldb, ws - 1, ws - 1);
  scipy_dlartg_(&temp, &M(B, ldb, ws - 1, ws - 2), &c, &s, &M(B, ldb, ws - 1, ws - 1));
  M(B, ldb, ws - 1, ws - 2) = 0.0;
  scipy_drot_(&ws, &M(A, lda, 0, ws - 1), &I1, &M(A, lda, 0, ws - 2), &I1, &c, &s);
  int wm1 = ws - 1;
  scipy_drot_(&wm1, &M(B, ldb, 0, ws - 1), &I1, &M(B, ldb, 0, ws - 2), &I1, &c, &s);
  scipy_drot_(&ws, &M(V, ldqz, 0, ws - 1), &I1, &M(V, ldqz, 0, ws - 2), &I1, &c, &s);
}

/* ---- PDHGEQZ6, single-process case (PDHGEQZ6.f:276-380) ----------------
 * Off-diagonal updates of the window j..j+w-1 with U (left) and V (right):
 * rows of H,T right of the window, columns above it, Q and Z. */
static void update6(Ctx* C, int j, int w, const double* U, const double* V, int lduv) {
  int n = C->n, ld = C->ld;
  double one = 1.0, zero = 0.0;
  int kln = n - (j + w);
  double* tmp = (double*)malloc(sizeof(double) * (size_t)w * (size_t)imax(n, 1));
  if (kln > 0) {
    double* mats[2] = {C->H, C->T};
    for (int m = 0; m < 2; ++m) {
      scipy_dgemm_("T", "N", &w, &kln, &w, &one, U, &lduv, &M(mats[m], ld, j, j + w), &ld, &zero, tmp, &w, 1, 1);
      for (int c = 0; c < kln; ++c) memcpy(&M(mats[m], ld, j, j + w + c), tmp + (size_t)c * w, sizeof(double) * w);
    }
    C->upd_flops += 4.0 * w * w * kln;
  }
  if (j > 0) {
    double* mats[2] = {C->H, C->T};
    for (int m = 0; m < 2; ++m) {
      scipy_dgemm_("N", "N", &j, &w, &w, &one, &M(mats[m], ld, 0, j), &ld, V, &lduv, &zero, tmp, &j, 1, 1);
      for (int c = 0; c < w; ++c) memcpy(&M(mats[m], ld, 0, j + c), tmp + (size_t)c * j, sizeof(double) * j);
    }
    C->upd_flops += 4.0 * w * w * j;
  }
  if (C->wantq) {
    scipy_dgemm_("N", "N", &n, &w, &w, &one, &M(C->Q, ld, 0, j), &ld, U, &lduv, &zero, tmp, &n, 1, 1);
    for (int c = 0; c < w; ++c) memcpy(&M(C->Q, ld, 0, j + c), tmp + (size_t)c * n, sizeof(double) * n);
    C->upd_flops += 2.0 * w * w * n;
  }
  if (C->wantz) {
    scipy_dgemm_("N", "N", &n, &w, &w, &one, &M(C->Z, ld, 0, j), &ld, V, &lduv, &zero, tmp, &n, 1, 1);
    for (int c = 0; c < w; ++c) memcpy(&M(C->Z, ld, 0, j + c), tmp + (size_t)c * n, sizeof(double) * n);
    C->upd_flops += 2.0 * w * w * n;
  }
  free(tmp);
}

static void eye(double* A, int n, int ld) {
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < n; ++r) M(A, ld, r, c) = (r == c) ? 1.0 : 0.0;
}

/* ---- chain sweep (PDHGEQZ5 with NUMWIN = 1, PDHGEQZA, PDHGEQZB) --------
 * Chase nbulge bulges with shifts (sr,si,sb)[0..2*nbulge) through the
 * active block [ktop, kbot].  Bulge b uses shifts 2b, 2b+1. */
static void chain_sweep(Ctx* C, int ktop, int kbot, int nbulge, const double* sr, const double* si, const double* sb,
                        int phase) {
  int ld = C->ld;
  int chain = 3 * nbulge;
  int nh = kbot - ktop + 1;
  int maxw = imin(nh, 2 * (chain + 1) + 4);
  double* A = (double*)malloc(sizeof(double) * maxw * maxw * 4);
  double* B = A + maxw * maxw;
  double* U = B + maxw * maxw;
  double* V = U + maxw * maxw;
  /* ---- introduction in the window [ktop, ktop+ws) (PDHGEQZA.f:325-420) */
  int j = ktop;
  int ws = imin(chain + 1, nh);
  if (ws < 3) { free(A); return; }
  for (int c = 0; c < ws; ++c)
    for (int r = 0; r < ws; ++r) {
      M(A, ws, r, c) = M(C->H, ld, j + r, j + c);
      M(B, ws, r, c) = M(C->T, ld, j + r, j + c);
    }
  eye(U, ws, ws);
  eye(V, ws, ws);
  int nb_in = 0;
  if (phase == 2) {
    /* bulges already introduced: topmost at column ktop, spacing 3 */
    nb_in = nbulge;
    goto chase;
  }
  for (int ib = 0; ib < nbulge; ++ib) {
    if (ws < 3) break;
    double v[3], tau, vv[3];
    qzfcol(2, sr + 2 * ib, si + 2 * ib, sb + 2 * ib, A, ws, B, ws, v);
    int three = 3;
    scipy_dlarfg_(&three, &v[0], &v[1], &I1, &tau);
    v[0] = 1.0;
    for (int c = 0; c < ws; ++c) {
      refl3(tau, v, &M(A, ws, 0, c), &M(A, ws, 1, c), &M(A, ws, 2, c));
      refl3(tau, v, &M(B, ws, 0, c), &M(B, ws, 1, c), &M(B, ws, 2, c));
    }
    for (int r = 0; r < ws; ++r) refl3(tau, v, &M(U, ws, r, 0), &M(U, ws, r, 1), &M(U, ws, r, 2));
    invhse3(B, ws, &tau, vv);
    for (int r = 0; r < 3; ++r) refl3(tau, vv, &M(B, ws, r, 0), &M(B, ws, r, 1), &M(B, ws, r, 2));
    M(B, ws, 1, 0) = 0.0;
    M(B, ws, 2, 0) = 0.0;
    for (int r = 0; r < imin(4, ws); ++r) refl3(tau, vv, &M(A, ws, r, 0), &M(A, ws, r, 1), &M(A, ws, r, 2));
    for (int r = 0; r < ws; ++r) refl3(tau, vv, &M(V, ws, r, 0), &M(V, ws, r, 1), &M(V, ws, r, 2));
    nb_in = ib + 1;
    if (nb_in < nbulge) {
      /* hunt bulges one step (3 columns) forward (PDHGEQZA.f:364-418) */
      for (int b = nb_in - 1; b >= 0; --b) {
        int ncols = 3;
        int jj = 3 * b; /* window row of bulge b (0-based, first introduced is deepest) */
        int nnb = imin(3 + 1 + ncols, ws - jj);
        if (nnb <= 0) continue;
        if (jj + nnb == ws && j + ws - 1 == kbot) ncols = 2;
        if (jj + 2 >= ws) continue;
        int ib_shift = nb_in - 1 - b;
        dhgeqz5(C, nnb, A, ws, B, ws, jj, ncols, ws, sr + 2 * ib_shift, si + 2 * ib_shift, sb + 2 * ib_shift, U, V, ws);
        if (ncols == 2) pushoff(A, ws, B, ws, ws, U, V, ws);
      }
    }
  }
  for (int c = 0; c < ws; ++c)
    for (int r = 0; r < ws; ++r) {
      M(C->H, ld, j + r, j + c) = M(A, ws, r, c);
      M(C->T, ld, j + r, j + c) = M(B, ws, r, c);
    }
  update6(C, j, ws, U, V, ws);
  if (phase == 1) { free(A); return; }
chase:;
  /* ---- chase (PDHGEQZB, cross-border windows) ---- */
  /* bulge b (0 = deepest) now sits with its column j0+3b... track the top
     row of the chain: the top bulge (last introduced) is at row j */
  int top = j;
  /* keep chasing until the topmost bulge has left the active block, as
     PDHGEQZ5 does until every window reports CHASECOMPLETE */
  while (top <= kbot - 2) {
    int movedist = chain + 1;
    int wsz = imin(kbot - top + 1, 2 * (chain + 1));
    if (wsz < 3) break;
    for (int c = 0; c < wsz; ++c)
      for (int r = 0; r < wsz; ++r) {
        M(A, wsz, r, c) = M(C->H, ld, top + r, top + c);
        M(B, wsz, r, c) = M(C->T, ld, top + r, top + c);
      }
    eye(U, wsz, wsz);
    eye(V, wsz, wsz);
    for (int ib = nb_in; ib >= 1; --ib) {
      int ncols = 3;
      int jj = (ib - 1) * 3;
      if (top + jj > kbot - 2) continue; /* already pushed off */
      int nnb = imin(ncols + movedist + 1, wsz - jj);
      if (nnb <= 0) continue;
      if (top + jj + nnb - 1 == kbot) ncols = 2;
      /* bulge ib (1 = topmost, nb_in = deepest) uses shift pair nb_in-ib */
      dhgeqz5(C, nnb, A, wsz, B, wsz, jj, ncols, wsz, sr + 2 * (nb_in - ib), si + 2 * (nb_in - ib),
              sb + 2 * (nb_in - ib), U, V, wsz);
      if (ncols == 2) pushoff(A, wsz, B, wsz, wsz, U, V, wsz);
    }
    for (int c = 0; c < wsz; ++c)
      for (int r = 0; r < wsz; ++r) {
        M(C->H, ld, top + r, top + c) = M(A, wsz, r, c);
        M(C->T, ld, top + r, top + c) = M(B, wsz, r, c);
      }
    update6(C, top, wsz, U, V, wsz);
    top += movedist;
  }
  free(A);
}

/* ---- PDLASMSUB (PDLASMSUB.f:344-368): bottom-up deflation search ------- */
static int lasmsub(Ctx* C, int ifirst, int kbot) {
  int ld = C->ld;
  for (int k = kbot; k > ifirst; --k) {
    double tst1 = fabs(M(C->H, ld, k - 1, k - 1)) + fabs(M(C->H, ld, k, k));
    if (tst1 == 0.0) {
      tst1 = 0.0;
      for (int c = ifirst; c <= kbot; ++c)
        for (int r = ifirst; r <= imin(c + 1, kbot); ++r) tst1 += fabs(M(C->H, ld, r, c));
    }
    if (fabs(M(C->H, ld, k, k - 1)) <= dmax(C->ulp * tst1, C->smlnum)) return k;
  }
  return ifirst;
}

static void rot_rows(Ctx* C, double* A, int r, int c0, double c, double s) {
  int len = C->n - c0;
  if (len > 0) scipy_drot_(&len, &M(A, C->ld, r, c0), &C->ld, &M(A, C->ld, r + 1, c0), &C->ld, &c, &s);
}
static void rot_cols(Ctx* C, double* A, int c1, int c2, int rows, double c, double s) {
  if (rows > 0) scipy_drot_(&rows, &M(A, C->ld, 0, c1), &I1, &M(A, C->ld, 0, c2), &I1, &c, &s);
}

/* ---- PDHGEQZ7 single-process restatement (PDHGEQZ7.f:355-540):
 * detect |t(k,k)| <= max(ttol, smlnum); deflate at the bottom (precheck
 * 1), at the top (precheck 2), interior zeros chased down (DHGEQZ7 role).
 * Returns the number of infinite eigenvalues deflated; updates *ktop,*kbot. */
static int pdhgeqz7(Ctx* C, int* ktop, int* kbot) {
  int ld = C->ld, nd = 0;
  double tol = dmax(C->ttol, C->smlnum);
  for (int iter = 0; iter < C->n + 1; ++iter) {
    int kt = *ktop, kb = *kbot;
    if (kb <= kt) break;
    int jz = -1;
    for (int j = kb; j >= kt; --j)
      if (fabs(M(C->T, ld, j, j)) <= tol) { M(C->T, ld, j, j) = 0.0; jz = j; break; }
    if (jz < 0) break;
    double c, s, r, temp;
    if (jz == kt) {
      /* top: rotation of rows kt, kt+1 zeroing H(kt+1,kt) */
      temp = M(C->H, ld, kt, kt);
      scipy_dlartg_(&temp, &M(C->H, ld, kt + 1, kt), &c, &s, &r);
      M(C->H, ld, kt, kt) = r;
      M(C->H, ld, kt + 1, kt) = 0.0;
      rot_rows(C, C->H, kt, kt + 1, c, s);
      rot_rows(C, C->T, kt, kt + 1, c, s);
      if (C->wantq) rot_cols(C, C->Q, kt, kt + 1, C->n, c, s);
      *ktop = kt + 1;
      nd++;
      continue;
    }
    /* chase the zero from jz down to kb (LAPACK zero chasing) */
    for (int jch = jz; jch < kb; ++jch) {
      temp = M(C->T, ld, jch, jch + 1);
      scipy_dlartg_(&temp, &M(C->T, ld, jch + 1, jch + 1), &c, &s, &M(C->T, ld, jch, jch + 1));
      M(C->T, ld, jch + 1, jch + 1) = 0.0;
      rot_rows(C, C->T, jch, jch + 2, c, s);
      rot_rows(C, C->H, jch, jch > kt ? jch - 1 : jch, c, s);
      if (C->wantq) rot_cols(C, C->Q, jch, jch + 1, C->n, c, s);
      if (jch > kt) {
        temp = M(C->H, ld, jch + 1, jch);
        scipy_dlartg_(&temp, &M(C->H, ld, jch + 1, jch - 1), &c, &s, &M(C->H, ld, jch + 1, jch));
        M(C->H, ld, jch + 1, jch - 1) = 0.0;
        rot_cols(C, C->H, jch, jch - 1, jch + 1, c, s);
        rot_cols(C, C->T, jch, jch - 1, jch, c, s);
        if (C->wantz) rot_cols(C, C->Z, jch, jch - 1, C->n, c, s);
      }
    }
    /* bottom: column rotation zeroing H(kb, kb-1) (precheck 1) */
    temp = M(C->H, ld, kb, kb);
    scipy_dlartg_(&temp, &M(C->H, ld, kb, kb - 1), &c, &s, &M(C->H, ld, kb, kb));
    M(C->H, ld, kb, kb - 1) = 0.0;
    rot_cols(C, C->H, kb, kb - 1, kb, c, s);
    rot_cols(C, C->T, kb, kb - 1, kb, c, s);
    if (C->wantz) rot_cols(C, C->Z, kb, kb - 1, C->n, c, s);
    *kbot = kb - 1;
    nd++;
  }
  return nd;
}

/* ---- small subproblem on [ktop, kbot] (PDHGEQZ4: serial QZ + updates) - */
static int small_solve(Ctx* C, int ktop, int kbot) {
  int nw = kbot - ktop + 1, ld = C->ld, info = 0;
  double* A = (double*)malloc(sizeof(double) * nw * nw * 4);
  double *B = A + nw * nw, *U = B + nw * nw, *V = U + nw * nw;
  for (int c = 0; c < nw; ++c)
    for (int r = 0; r < nw; ++r) {
      M(A, nw, r, c) = M(C->H, ld, ktop + r, ktop + c);
      M(B, nw, r, c) = M(C->T, ld, ktop + r, ktop + c);
    }
  eye(U, nw, nw);
  eye(V, nw, nw);
  double* ar = (double*)malloc(sizeof(double) * 3 * nw);
  int one = 1, lw = -1;
  double wq;
  scipy_dhgeqz_("S", "V", "V", &nw, &one, &nw, A, &nw, B, &nw, ar, ar + nw, ar + 2 * nw, U, &nw, V, &nw, &wq, &lw,
                &info, 1, 1, 1);
  lw = (int)wq + 1;
  double* work = (double*)malloc(sizeof(double) * lw);
  scipy_dhgeqz_("S", "V", "V", &nw, &one, &nw, A, &nw, B, &nw, ar, ar + nw, ar + 2 * nw, U, &nw, V, &nw, work, &lw,
                &info, 1, 1, 1);
  free(work);
  free(ar);
  for (int c = 0; c < nw; ++c)
    for (int r = 0; r < nw; ++r) {
      M(C->H, ld, ktop + r, ktop + c) = M(A, nw, r, c);
      M(C->T, ld, ktop + r, ktop + c) = M(B, nw, r, c);
    }
  update6(C, ktop, nw, U, V, nw);
  free(A);
  return info;
}

/* ---- QZEARLY (src/kkqz/qzearly.f:229-449) on an nw-window with spike s.
 * Returns the number of deflated eigenvalues; the undeflated eigenvalues
 * (shifts) are left in sr/si/sb[0..nw-nd). */
static int qzearly(Ctx* C, int nw, double s, double* A, double* B, double* U, double* V, double* sr, double* si,
                   double* sb) {
  int one = 1, info = 0, lw = -1;
  double wq;
  eye(U, nw, nw);
  eye(V, nw, nw);
  scipy_dhgeqz_("S", "V", "V", &nw, &one, &nw, A, &nw, B, &nw, sr, si, sb, U, &nw, V, &nw, &wq, &lw, &info, 1, 1, 1);
  lw = (int)wq + 4 * nw + 16;
  double* work = (double*)malloc(sizeof(double) * (size_t)imax(lw, 4 * nw + 16));
  scipy_dhgeqz_("S", "V", "V", &nw, &one, &nw, A, &nw, B, &nw, sr, si, sb, U, &nw, V, &nw, work, &lw, &info, 1, 1, 1);
  if (info != 0) { free(work); return 0; }
  int ilst = 1, kbot = nw, knt = 0; /* 1-based as in the reference */
  while (knt < nw) {
    int bulge = (kbot == 1) ? 0 : (M(A, nw, kbot - 1, kbot - 2) != 0.0);
    int dflate;
    if (!bulge) {
      knt += 1;
      double temp = fabs(s) + fabs(M(A, nw, kbot - 1, kbot - 1));
      dflate = fabs(s * M(U, nw, 0, kbot - 1)) <= dmax(C->ulp * temp, C->smlnum);
    } else {
      knt += 2;
      double h11 = M(A, nw, kbot - 2, kbot - 2), h21 = M(A, nw, kbot - 1, kbot - 2);
      double h12 = M(A, nw, kbot - 2, kbot - 1), h22 = M(A, nw, kbot - 1, kbot - 1);
      double rtdet;
      if (h11 == 0.0 && h21 == 0.0) rtdet = 0.0;
      else if (fabs(h11) >= fabs(h21)) rtdet = sqrt(fabs(h11)) * sqrt(fabs(h22 - (h21 / h11) * h12));
      else rtdet = sqrt(fabs(h21)) * sqrt(fabs(h12 - (h11 / h21) * h22));
      double temp = fabs(s) + rtdet;
      dflate = dmax(fabs(s * M(U, nw, 0, kbot - 1)), fabs(s * M(U, nw, 0, kbot - 2))) <= dmax(C->ulp * temp, C->smlnum);
    }
    if (dflate) {
      kbot -= bulge ? 2 : 1;
    } else {
      int ifst = kbot, ierr = 0, t1 = 1;
      int lwx = imax(lw, 4 * nw + 16);
      scipy_dtgexc_(&t1, &t1, &nw, A, &nw, B, &nw, U, &nw, V, &nw, &ifst, &ilst, work, &lwx, &ierr);
      if (ierr != 0) break; /* qzearly.f:321-326: go to re-reduction */
      int nbk = bulge ? 2 : 1;
      /* rotate shifts (qzearly.f:331-363) */
      double tr[2], ti[2], tb[2];
      for (int q = 0; q < nbk; ++q) { tr[q] = sr[kbot - nbk + q]; ti[q] = si[kbot - nbk + q]; tb[q] = sb[kbot - nbk + q]; }
      for (int q = kbot - nbk - 1; q >= ilst - 1; --q) { sr[q + nbk] = sr[q]; si[q + nbk] = si[q]; sb[q + nbk] = sb[q]; }
      for (int q = 0; q < nbk; ++q) { sr[ilst - 1 + q] = tr[q]; si[ilst - 1 + q] = ti[q]; sb[ilst - 1 + q] = tb[q]; }
      ilst += nbk;
    }
  }
  /* return to Hessenberg-triangular form (qzearly.f:369-449) */
  int kb = kbot;
  if (kb > 0 && s != 0.0 && kb < nw) {
    double* d = work;
    for (int i = 0; i < kb; ++i) d[i] = M(U, nw, 0, i);
    double alpha = d[0], tau;
    int kbm1 = kb - 1;
    scipy_dlarfg_(&kb, &alpha, d + 1, &I1, &tau);
    d[0] = 1.0;
    /* H <- P H (rows 1:kb, all columns); U <- U P */
    for (int c = 0; c < nw; ++c) {
      double t = 0.0;
      for (int i = 0; i < kb; ++i) t += d[i] * M(A, nw, i, c);
      t *= tau;
      for (int i = 0; i < kb; ++i) M(A, nw, i, c) -= t * d[i];
    }
    for (int r = 0; r < nw; ++r) {
      double t = 0.0;
      for (int i = 0; i < kb; ++i) t += M(U, nw, r, i) * d[i];
      t *= tau;
      for (int i = 0; i < kb; ++i) M(U, nw, r, i) -= t * d[i];
    }
    if (kb > 1) {
      /* RQ update with 2*kb-2 Givens rotations (PARA_AGGRQUP, qzearly.f:396-446) */
      for (int c = kb; c < nw; ++c) {
        double t = 0.0;
        for (int i = 0; i < kb; ++i) t += d[i] * M(B, nw, i, c);
        t *= tau;
        for (int i = 0; i < kb; ++i) M(B, nw, i, c) -= t * d[i];
      }
      double* wv = d + kb;
      double* cs = d + 2 * kb;
      double* sn = d + 3 * kb;
      for (int c = 0; c < kb; ++c) {
        double t = 0.0;
        for (int i = 0; i <= c; ++i) t += M(B, nw, i, c) * d[i];
        wv[c] = -tau * t;
      }
      for (int i = 0; i < kb - 1; ++i) {
        double a = wv[i + 1];
        scipy_dlartg_(&a, &wv[i], &cs[i], &sn[i], &wv[i + 1]);
        sn[i] = -sn[i];
        int len = i + 2;
        scipy_drot_(&len, &M(B, nw, 0, i), &I1, &M(B, nw, 0, i + 1), &I1, &cs[i], &sn[i]);
      }
      for (int i = 0; i < kb; ++i) M(B, nw, i, kb - 1) += wv[kb - 1] * d[i];
      for (int i = 0; i < kb - 1; ++i)
        scipy_drot_(&kb, &M(A, nw, 0, i), &I1, &M(A, nw, 0, i + 1), &I1, &cs[i], &sn[i]);
      for (int i = 0; i < kb - 1; ++i)
        scipy_drot_(&nw, &M(V, nw, 0, i), &I1, &M(V, nw, 0, i + 1), &I1, &cs[i], &sn[i]);
      for (int i = kb - 2; i >= 0; --i) {
        double a = M(B, nw, i + 1, i + 1);
        scipy_dlartg_(&a, &M(B, nw, i + 1, i), &cs[i], &sn[i], &M(B, nw, i + 1, i + 1));
        sn[i] = -sn[i];
        M(B, nw, i + 1, i) = 0.0;
        int len = i + 1;
        scipy_drot_(&len, &M(B, nw, 0, i), &I1, &M(B, nw, 0, i + 1), &I1, &cs[i], &sn[i]);
      }
      for (int i = kb - 2; i >= 0; --i)
        scipy_drot_(&kb, &M(A, nw, 0, i), &I1, &M(A, nw, 0, i + 1), &I1, &cs[i], &sn[i]);
      for (int i = kb - 2; i >= 0; --i)
        scipy_drot_(&nw, &M(V, nw, 0, i), &I1, &M(V, nw, 0, i + 1), &I1, &cs[i], &sn[i]);
    }
    (void)kbm1;
    int ierr;
    scipy_dgghrd_("V", "V", &nw, &one, &kb, A, &nw, B, &nw, U, &nw, V, &nw, &ierr, 1, 1);
  }
  free(work);
  return nw - kbot;
}

/* ---- AED driver (PDHGEQZ2.f:315-408) ----------------------------------- */
static int aed(Ctx* C, int ktop, int kbot, int nw, double* sr, double* si, double* sb, int* nshift) {
  int ld = C->ld;
  int kwtop = kbot - nw + 1;
  double s = (kwtop > ktop) ? M(C->H, ld, kwtop, kwtop - 1) : 0.0;
  double* A = (double*)malloc(sizeof(double) * nw * nw * 4);
  double *B = A + nw * nw, *U = B + nw * nw, *V = U + nw * nw;
  for (int c = 0; c < nw; ++c)
    for (int r = 0; r < nw; ++r) {
      M(A, nw, r, c) = M(C->H, ld, kwtop + r, kwtop + c);
      M(B, nw, r, c) = M(C->T, ld, kwtop + r, kwtop + c);
    }
  int nd = qzearly(C, nw, s, A, B, U, V, sr, si, sb);
  *nshift = nw - nd;
  if (nd > 0) {
    for (int c = 0; c < nw; ++c)
      for (int r = 0; r < nw; ++r) {
        M(C->H, ld, kwtop + r, kwtop + c) = M(A, nw, r, c);
        M(C->T, ld, kwtop + r, kwtop + c) = M(B, nw, r, c);
      }
    if (kwtop > ktop) M(C->H, ld, kwtop, kwtop - 1) = s * M(U, nw, 0, 0);
    update6(C, kwtop, nw, U, V, nw);
  }
  free(A);
  return nd;
}

/* tuning (piparmq.f:438-535) */
static int ns_table(int nh) {
  int ns = 2;
  if (nh >= 30) ns = 4;
  if (nh >= 60) ns = 10;
  if (nh >= 150) ns = imax(10, (int)(nh / lround(log((double)nh) / log(2.0))));
  if (nh >= 590) ns = 64;
  if (nh >= 3000) ns = 128;
  if (nh >= 6000) ns = 256;
  if (nh >= 12000) ns = 512;
  return imax(2, ns - ns % 2);
}

/* ---- main iteration (PDHGEQZ1.f:466-763; PDHGEQZ0.f:505-1202 table for
 * nh > 6000) ------------------------------------------------------------ */
static int iterate(Ctx* C, int ilo, int ihi) {
  int ld = C->ld;
  int nmin = 201;
  int ifirst = ilo, kbot = ihi;
  long maxit = 30L * imax(1, ihi - ilo + 1);
  int nwmax = imax(C->nb, 4);
  double* sh = (double*)malloc(sizeof(double) * 3 * 1024);
  for (long it = 0; it < maxit; ++it) {
    if (kbot < ifirst) { free(sh); return 0; }
    C->iters++;
    int nh = kbot - ifirst + 1;
    int ktop = (nh <= nmin) ? ifirst : lasmsub(C, ifirst, kbot);
    if (ktop > ifirst) M(C->H, ld, ktop, ktop - 1) = 0.0;
    int okt = ktop, okb = kbot;
    int ndinf = pdhgeqz7(C, &ktop, &kbot);
    if (ndinf > 0) {
      C->infs += ndinf;
      if (ktop != okt && okt == ifirst) ifirst = ktop;
      (void)okb;
      if (kbot < ifirst) continue;
      continue;
    }
    nh = kbot - ktop + 1;
    if (nh < nmin) {
      /* small subproblem: 1x1, 2x2 (DLAGV2), or serial QZ (PDHGEQZ4) */
      C->smallsub++;
      if (nh > 2) {
        if (small_solve(C, ktop, kbot) != 0) { free(sh); return kbot + 1; }
      }
      kbot = ktop - 1;
      if (kbot < ifirst) { free(sh); return 0; }
      continue;
    }
    int dblk, nib, nsmax;
    if (ihi - ilo + 1 <= 6000) {
      dblk = imin(nh, imin(nmin, nwmax));
      nib = 14;
      nsmax = dblk;
    } else {
      nsmax = ns_table(nh);
      dblk = imin(nh, 3 * nsmax / 2);
      if (dblk > 1000) dblk = 1000;
      nib = imin(100, (int)ceil(335.0 * pow((double)nh, -0.44)));
    }
    if (C->aed_limit >= 0 && C->aeds >= C->aed_limit) { free(sh); return -2; }
    if (C->aed_clock && C->aeds < C->aed_cap) C->aed_clock[C->aeds] = wall_seconds() - C->t_start;
    C->aeds++;
    int nshift = 0;
    int nd = aed(C, ktop, kbot, dblk, sh, sh + 1024, sh + 2048, &nshift);
    kbot -= nd;
    if (kbot < ifirst) break;
    if (kbot < ktop) continue;
    if (100 * nd > nib * dblk) continue;
    /* sweep: undeflated eigenvalues as shifts, paired (PDHGEQZ1.f:608-629) */
    int ns = imin(nsmax, nshift);
    ns -= ns % 2;
    double *sr = sh, *si = sh + 1024, *sb = sh + 2048;
    for (int i = ns - 1; i >= 2; i -= 2) {
      if (si[i] == 0.0 && si[i - 1] != 0.0) {
        double t;
        t = sr[i]; sr[i] = sr[i - 1]; sr[i - 1] = sr[i - 2]; sr[i - 2] = t;
        t = si[i]; si[i] = si[i - 1]; si[i - 1] = si[i - 2]; si[i - 2] = t;
        t = sb[i]; sb[i] = sb[i - 1]; sb[i - 1] = sb[i - 2]; sb[i - 2] = t;
      }
    }
    if (ns < 2 || kbot - ktop + 1 < 4) continue;
    C->sweeps++;
    int spw = imax(imin(ns, C->nb / 3 - 1), 2);
    spw -= spw % 2;
    for (int p0 = 0; p0 + 2 <= ns; p0 += spw) {
      int cnt = imin(spw, ns - p0);
      cnt -= cnt % 2;
      if (cnt < 2) break;
      chain_sweep(C, ktop, kbot, cnt / 2, sr + p0, si + p0, sb + p0, 0);
    }
  }
  free(sh);
  return kbot + 1;
}

/* standardise 2x2 blocks (DLAGV2, PDHGEQZ0.f:622-677), beta >= 0, and
 * read the eigenvalues */
static void finalize(Ctx* C, double* ar, double* ai, double* be) {
  int n = C->n, ld = C->ld, j = 0;
  while (j < n) {
    if (j + 1 < n && M(C->H, ld, j + 1, j) != 0.0) {
      double csl, snl, csr, snr;
      int two = 2;
      scipy_dlagv2_(&M(C->H, ld, j, j), &ld, &M(C->T, ld, j, j), &ld, &ar[j], &ai[j], &be[j], &csl, &snl, &csr, &snr);
      /* rows j, j+1 right of the block; columns above it; Q, Z */
      int len = n - j - 2;
      if (len > 0) {
        scipy_drot_(&len, &M(C->H, ld, j, j + 2), &ld, &M(C->H, ld, j + 1, j + 2), &ld, &csl, &snl);
        scipy_drot_(&len, &M(C->T, ld, j, j + 2), &ld, &M(C->T, ld, j + 1, j + 2), &ld, &csl, &snl);
      }
      if (j > 0) {
        scipy_drot_(&j, &M(C->H, ld, 0, j), &I1, &M(C->H, ld, 0, j + 1), &I1, &csr, &snr);
        scipy_drot_(&j, &M(C->T, ld, 0, j), &I1, &M(C->T, ld, 0, j + 1), &I1, &csr, &snr);
      }
      if (C->wantq) scipy_drot_(&n, &M(C->Q, ld, 0, j), &I1, &M(C->Q, ld, 0, j + 1), &I1, &csl, &snl);
      if (C->wantz) scipy_drot_(&n, &M(C->Z, ld, 0, j), &I1, &M(C->Z, ld, 0, j + 1), &I1, &csr, &snr);
      (void)two;
      if (M(C->H, ld, j + 1, j) == 0.0) continue; /* split into a real pair: revisit j as 1x1 */
      /* positive diagonal of T in the block (PDHGEQZ.f:51-58 convention):
         negate the offending column of H, T and Z */
      for (int k = j; k <= j + 1; ++k)
        if (M(C->T, ld, k, k) < 0.0) {
          for (int r = 0; r <= j + 1; ++r) { M(C->H, ld, r, k) = -M(C->H, ld, r, k); M(C->T, ld, r, k) = -M(C->T, ld, r, k); }
          if (C->wantz)
            for (int r = 0; r < n; ++r) M(C->Z, ld, r, k) = -M(C->Z, ld, r, k);
        }
      {
        double a[4] = {M(C->H, ld, j, j), M(C->H, ld, j + 1, j), M(C->H, ld, j, j + 1), M(C->H, ld, j + 1, j + 1)};
        double b0 = M(C->T, ld, j, j), b1 = M(C->T, ld, j + 1, j + 1);
        /* eigenvalues of diag(b)^-1 A: lambda = wr +- i wi */
        double m00 = a[0] / b0, m01 = a[2] / b0, m10 = a[1] / b1, m11 = a[3] / b1;
        double tr = 0.5 * (m00 + m11), d = 0.5 * (m00 - m11), disc = d * d + m01 * m10;
        double wi = sqrt(fabs(fmin(disc, 0.0)));
        ar[j] = tr * b0; ai[j] = wi * b0; be[j] = b0;
        ar[j + 1] = tr * b1; ai[j + 1] = -wi * b1; be[j + 1] = b1;
      }
      j += 2;
    } else {
      if (M(C->T, ld, j, j) < 0.0) {
        for (int r = 0; r <= j; ++r) { M(C->H, ld, r, j) = -M(C->H, ld, r, j); M(C->T, ld, r, j) = -M(C->T, ld, r, j); }
        if (C->wantz)
          for (int r = 0; r < n; ++r) M(C->Z, ld, r, j) = -M(C->Z, ld, r, j);
      }
      ar[j] = M(C->H, ld, j, j);
      ai[j] = 0.0;
      be[j] = M(C->T, ld, j, j);
      j += 1;
    }
  }
}

/* Public entry of the restatement: same argument meaning as PDHGEQZ on a
 * 1x1 grid (job 'S'/'E', compq/compz 'N'/'I'/'V', 1-based ilo/ihi).
 * stats (may be NULL): iters, aeds, sweeps, small subproblems, infinite
 * eigenvalues, update flops. */
int qzref_pdhgeqz_ex(char job, char compq, char compz, int n, int ilo, int ihi, double* H, double* T, double* Q,
                     double* Z, int ld, int nb, double* ar, double* ai, double* be, double* stats, long aed_limit,
                     double* aed_clock, long aed_cap) {
  (void)job;
  if (n <= 0) return 0;
  Ctx C;
  memset(&C, 0, sizeof(C));
  C.aed_limit = aed_limit;
  C.aed_clock = aed_clock;
  C.aed_cap = aed_cap;
  C.t_start = wall_seconds();
  C.n = n; C.ld = ld; C.H = H; C.T = T; C.Q = Q; C.Z = Z;
  C.wantq = (compq != 'N' && compq != 'n');
  C.wantz = (compz != 'N' && compz != 'n');
  C.nb = nb;
  if (compq == 'I' || compq == 'i') eye(Q, n, ld);
  if (compz == 'I' || compz == 'i') eye(Z, n, ld);
  double unfl = scipy_dlamch_("S", 1);
  C.safmin = unfl;
  C.ulp = scipy_dlamch_("P", 1);
  int nh = ihi - ilo + 1;
  C.smlnum = unfl * (nh / C.ulp);
  double hn = 0, tn = 0;
  for (int c = ilo - 1; c < ihi; ++c)
    for (int r = ilo - 1; r < ihi; ++r) { hn += M(H, ld, r, c) * M(H, ld, r, c); tn += M(T, ld, r, c) * M(T, ld, r, c); }
  C.htol = dmax(unfl, C.ulp * sqrt(hn));
  C.ttol = dmax(unfl, C.ulp * sqrt(tn));
  for (int i = ilo - 1; i < ihi; ++i) { ar[i] = -1.0; ai[i] = -1.0; be[i] = -1.0; }
  int info = iterate(&C, ilo - 1, ihi - 1);
  if (info != -2) finalize(&C, ar, ai, be);
  if (stats) {
    stats[0] = C.iters; stats[1] = C.aeds; stats[2] = C.sweeps; stats[3] = C.smallsub; stats[4] = C.infs;
    stats[5] = C.upd_flops;
  }
  return info;
}

/* The restatement without the bounded-run options; returns INFO, or -2
 * when an AED limit stopped it (only through qzref_pdhgeqz_ex). */
int qzref_pdhgeqz(char job, char compq, char compz, int n, int ilo, int ihi, double* H, double* T, double* Q,
                  double* Z, int ld, int nb, double* ar, double* ai, double* be, double* stats) {
  return qzref_pdhgeqz_ex(job, compq, compz, n, ilo, ihi, H, T, Q, Z, ld, nb, ar, ai, be, stats, -1, NULL, 0);
}

/* ---- kernel-level restatements exported for parity tests --------------- */

/* one bulge chased nstep-ncol+1 steps (DHGEQZ5) inside a window */
void qzref_dhgeqz5(int nstep, double* A, int lda, double* B, int ldb, int ir, int ncol, int wsize, const double* sr,
                   const double* si, const double* sb, double* U, double* V, int lduv) {
  Ctx C;
  memset(&C, 0, sizeof(C));
  C.ulp = scipy_dlamch_("P", 1);
  C.smlnum = scipy_dlamch_("S", 1) * (wsize / C.ulp);
  dhgeqz5(&C, nstep, A, lda, B, ldb, ir, ncol, wsize, sr, si, sb, U, V, lduv);
}

/* QZFCOL for two shifts */
void qzref_qzfcol2(const double* sr, const double* si, const double* sb, const double* H, int ldh, const double* T,
                   int ldt, double* v) {
  qzfcol(2, sr, si, sb, H, ldh, T, ldt, v);
}

/* INVHSE on a 3x3 block */
void qzref_invhse3(const double* T, int ldt, double* tau, double* v) { invhse3(T, ldt, tau, v); }

/* push-off step at the bottom of a window (PDHGEQZB.f:373-406) */
void qzref_pushoff(double* A, int lda, double* B, int ldb, int ws, double* U, double* V, int lduv) {
  pushoff(A, lda, B, ldb, ws, U, V, lduv);
}

/* One multishift sweep of nbulge bulges over a standalone n x n pencil,
 * in the window sequence of PDHGEQZ5/A/B; Q and Z accumulate (pass
 * identities for the sweep's own factors).  Bulge b uses shifts 2b, 2b+1
 * of (sr, si, sb).  phase 0: introduction + chase + push-off; 1: only the
 * introduction (PDHGEQZA); 2: only the chase + push-off of a chain already
 * in the pencil with its topmost bulge in column 0 (PDHGEQZB). */
void qzref_sweep(int n, double* H, double* T, double* Q, double* Z, int ld, int nbulge, const double* sr,
                 const double* si, const double* sb, int phase) {
  Ctx C;
  memset(&C, 0, sizeof(C));
  C.n = n; C.ld = ld; C.H = H; C.T = T; C.Q = Q; C.Z = Z;
  C.wantq = 1; C.wantz = 1;
  C.ulp = scipy_dlamch_("P", 1);
  C.smlnum = scipy_dlamch_("S", 1) * (n / C.ulp);
  chain_sweep(&C, 0, n - 1, nbulge, sr, si, sb, phase);
}
