// CTA-level QZ algorithms on one square window (one thread block).
//
// Each routine is a template over an executor X that supplies
//   int tid, nt;   thread index / count inside the block
//   void sync();   block barrier
//   void stamp(int k);  optional phase timestamp k (profiling)
//   void count(int k);  optional event counter k (profiling)
//   int* si; double* sd;  small shared scratch (>= 64 ints, >= 256 doubles)
// On the device X is a thin wrapper over threadIdx/__syncthreads and shared
// memory.  Data-parallel loops are written "for (i = tid; i < n; i += nt)"
// and every value that decides control flow is either computed redundantly
// by all threads from data no thread writes in the same phase, or computed
// by thread 0 and published through shared scratch across a barrier.
//
// Algorithms (all FP64, written from the published mathematics):
//  * cta_small_qz: implicit double-shift QZ (Moler-Stewart) with zero-
//    chasing for infinite eigenvalues and 2x2 standardisation; the role of
//    the reference's serial small QZ kernels QZDACK/QZLAP
//    (src/kkqz/qzdack.f, src/kkqz/qzlap.f) inside QZEARLY (qzearly.f:229-236)
//    and of KKQZ in the endgame (PDHGEQZ4.f:329-372).
//  * cta_swap / cta_move_block: reordering of 1x1/2x2 blocks of a
//    generalized real Schur form by direct swapping (generalized Sylvester
//    equation, Kagstrom-Poromaa), the role of DTGEXC/DTGEX2
//    (src/reorder/dtgexc.f, dtgex2.f) called at qzearly.f:315.
// The AED routine built on these (cta_aed) is in qz_window.cuh.
#pragma once
#include "qz_prims.cuh"

namespace qz {

// ---------------------------------------------------------------------------
// data-parallel helpers
// ---------------------------------------------------------------------------
template <class X>
QZ_HD void par_rot_rows(X& x, MatV M, int r0, int r1, double c, double s, int c_lo, int c_hi) {
  for (int j = c_lo + x.tid; j < c_hi; j += x.nt) {
    double a = M(r0, j), b = M(r1, j);
    M(r0, j) = c * a + s * b;
    M(r1, j) = -s * a + c * b;
  }
}
template <class X>
QZ_HD void par_rot_cols(X& x, MatV M, int c0, int c1, double c, double s, int r_lo, int r_hi) {
  for (int i = r_lo + x.tid; i < r_hi; i += x.nt) {
    double a = M(i, c0), b = M(i, c1);
    M(i, c0) = c * a + s * b;
    M(i, c1) = -s * a + c * b;
  }
}
template <class X>
QZ_HD void par_refl_rows(X& x, MatV M, int r, double tau, double v1, double v2, int c_lo, int c_hi) {
  for (int j = c_lo + x.tid; j < c_hi; j += x.nt) {
    double a0 = M(r, j), a1 = M(r + 1, j), a2 = M(r + 2, j);
    refl3(tau, v1, v2, a0, a1, a2);
    M(r, j) = a0; M(r + 1, j) = a1; M(r + 2, j) = a2;
  }
}
template <class X>
QZ_HD void par_refl_cols(X& x, MatV M, int c, double tau, double v1, double v2, int r_lo, int r_hi) {
  for (int i = r_lo + x.tid; i < r_hi; i += x.nt) {
    double a0 = M(i, c), a1 = M(i, c + 1), a2 = M(i, c + 2);
    refl3(tau, v1, v2, a0, a1, a2);
    M(i, c) = a0; M(i, c + 1) = a1; M(i, c + 2) = a2;
  }
}
template <class X>
QZ_HD void par_house_rows(X& x, MatV M, int r, const House3& h, int c_lo, int c_hi) {
  for (int j = c_lo + x.tid; j < c_hi; j += x.nt) {
    double a0 = M(r, j), a1 = M(r + 1, j), a2 = M(r + 2, j);
    house3_apply(h, a0, a1, a2);
    M(r, j) = a0; M(r + 1, j) = a1; M(r + 2, j) = a2;
  }
}
template <class X>
QZ_HD void par_house_cols(X& x, MatV M, int c, const House3& h, int r_lo, int r_hi) {
  for (int i = r_lo + x.tid; i < r_hi; i += x.nt) {
    double a0 = M(i, c), a1 = M(i, c + 1), a2 = M(i, c + 2);
    house3_apply(h, a0, a1, a2);
    M(i, c) = a0; M(i, c + 1) = a1; M(i, c + 2) = a2;
  }
}

// One transformation applied to several vector sets at once, the items of
// all sets spread over every thread (instead of one loop per set, which
// leaves most threads idle when the sets are short).  Item i of a set is
// the vector p + i*step, p + i*step + stride (+ 2*stride for a reflector).
struct Seg {
  double* p;
  int64_t step;
  int64_t stride;
  int count;
};
QZ_HD Seg seg_rows(MatV M, int r, int c_lo, int c_hi) {  // rows r.. of columns c_lo..c_hi-1
  return Seg{&M(r, c_lo), (int64_t)M.ld, 1, c_hi - c_lo};
}
QZ_HD Seg seg_cols(MatV M, int c, int r_lo, int r_hi) {  // columns c.. of rows r_lo..r_hi-1
  return Seg{&M(r_lo, c), 1, (int64_t)M.ld, r_hi - r_lo};
}
// item idx of the sets a, b, c (a's items first): its first element and stride
QZ_HD bool seg_item(const Seg& a, const Seg& b, const Seg& c, int idx, double*& q, int64_t& st) {
  const int na = a.count > 0 ? a.count : 0, nb = b.count > 0 ? b.count : 0, nc = c.count > 0 ? c.count : 0;
  if (idx < na) { q = a.p + (int64_t)idx * a.step; st = a.stride; return true; }
  idx -= na;
  if (idx < nb) { q = b.p + (int64_t)idx * b.step; st = b.stride; return true; }
  idx -= nb;
  if (idx < nc) { q = c.p + (int64_t)idx * c.step; st = c.stride; return true; }
  return false;
}
// Steps that transform a small block on one thread and the far parts on all
// threads use index ownership: thread t applies the step to every vector
// indexed t (column t of the rows a left transformation touches, row t of
// the columns a right one touches, row t of Q and Z), so each thread has a
// few independent short chains and no per-item dispatch.  The small block
// goes to the CTA's last thread, whose warp has no index work while the
// window is at most nt - 32 wide.
template <class X>
QZ_HD bool block_thread(const X& x) {
  return x.tid == x.nt - 1;
}
QZ_HD void house3_vec(const House3& h, double* q, int64_t st) {
  double a0 = q[0], a1 = q[st], a2 = q[2 * st];
  house3_apply(h, a0, a1, a2);
  q[0] = a0; q[st] = a1; q[2 * st] = a2;
}
QZ_HD void rot_vec(double c, double s, double* q, int64_t st) {
  const double u = q[0], v = q[st];
  q[0] = c * u + s * v;
  q[st] = -s * u + c * v;
}

QZ_HD int seg_total(const Seg& a, const Seg& b, const Seg& c) {
  return (a.count > 0 ? a.count : 0) + (b.count > 0 ? b.count : 0) + (c.count > 0 ? c.count : 0);
}
template <class X>
QZ_HD void par_house_segs(X& x, const House3& h, const Seg& a, const Seg& b, const Seg& c) {
  const int total = seg_total(a, b, c);
  for (int idx = x.tid; idx < total; idx += x.nt) {
    double* q;
    int64_t st;
    if (!seg_item(a, b, c, idx, q, st)) break;
    double a0 = q[0], a1 = q[st], a2 = q[2 * st];
    house3_apply(h, a0, a1, a2);
    q[0] = a0; q[st] = a1; q[2 * st] = a2;
  }
}
template <class X>
QZ_HD void par_rot_segs(X& x, double c, double s, const Seg& a, const Seg& b, const Seg& d) {
  const int total = seg_total(a, b, d);
  for (int idx = x.tid; idx < total; idx += x.nt) {
    double* q;
    int64_t st;
    if (!seg_item(a, b, d, idx, q, st)) break;
    const double u = q[0], v = q[st];
    q[0] = c * u + s * v;
    q[st] = -s * u + c * v;
  }
}
QZ_HD Seg no_seg() { return Seg{nullptr, 0, 0, 0}; }

template <class X>
QZ_HD void par_neg_row(X& x, MatV M, int r, int c_lo, int c_hi) {
  for (int j = c_lo + x.tid; j < c_hi; j += x.nt) M(r, j) = -M(r, j);
}
template <class X>
QZ_HD void par_neg_col(X& x, MatV M, int c, int r_lo, int r_hi) {
  for (int i = r_lo + x.tid; i < r_hi; i += x.nt) M(i, c) = -M(i, c);
}
template <class X>
QZ_HD void par_set_identity(X& x, MatV M, int n) {
  for (int k = x.tid; k < n * n; k += x.nt) {
    int i = k % n, j = k / n;
    M(i, j) = (i == j) ? 1.0 : 0.0;
  }
}

// Window state shared by the routines below.  Q and Z accumulate the left
// and right transformations of the window (H_in = Q H_out Z^T).
struct WinState {
  int n;
  MatV H, T, Q, Z;
  bool wantq, wantz;
  Tol tol;
};

// ---------------------------------------------------------------------------
// 2x2 standardisation of block (j, j+1) inside the window.
// Applies rotations to rows/cols of the whole window (Schur mode).
// ---------------------------------------------------------------------------
template <class X>
QZ_HD void cta_std2x2(X& x, WinState& w, int j) {
  // every thread computes the same rotations from the same 8 values
  double A[4] = {w.H(j, j), w.H(j + 1, j), w.H(j, j + 1), w.H(j + 1, j + 1)};
  double B[4] = {w.T(j, j), w.T(j + 1, j), w.T(j, j + 1), w.T(j + 1, j + 1)};
  Std2 o;
  std2x2(A, B, o);
  x.sync();  // all reads of the block done before anyone writes
  int n = w.n;
  {
    // rows: columns j+2..n-1 (the block itself is written from o.a/o.b);
    // cols: rows 0..j-1 (disjoint entries, so one pass)
    const Seg sl0 = seg_rows(w.H, j, j + 2, n);
    const Seg sl1 = seg_rows(w.T, j, j + 2, n);
    const Seg sl2 = w.wantq ? seg_cols(w.Q, j, 0, n) : no_seg();
    par_rot_segs(x, o.csl, o.snl, sl0, sl1, sl2);
    const Seg sr0 = seg_cols(w.H, j, 0, j);
    const Seg sr1 = seg_cols(w.T, j, 0, j);
    const Seg sr2 = w.wantz ? seg_cols(w.Z, j, 0, n) : no_seg();
    par_rot_segs(x, o.csr, o.snr, sr0, sr1, sr2);
  }
  x.sync();
  if (o.negrow0) {
    par_neg_row(x, w.H, j, j + 2, n);
    par_neg_row(x, w.T, j, j + 2, n);
    if (w.wantq) par_neg_col(x, w.Q, j, 0, n);
  }
  if (o.negrow1) {
    par_neg_row(x, w.H, j + 1, j + 2, n);
    par_neg_row(x, w.T, j + 1, j + 2, n);
    if (w.wantq) par_neg_col(x, w.Q, j + 1, 0, n);
  }
  if (x.tid == 0) {
    w.H(j, j) = o.a[0]; w.H(j + 1, j) = o.a[1]; w.H(j, j + 1) = o.a[2]; w.H(j + 1, j + 1) = o.a[3];
    w.T(j, j) = o.b[0]; w.T(j + 1, j) = 0.0;    w.T(j, j + 1) = o.b[2]; w.T(j + 1, j + 1) = o.b[3];
  }
  x.sync();
}

// ---------------------------------------------------------------------------
// Standardise every 2x2 block of the window at once.  A block's rotations
// touch rows j, j+1 right of the block and columns j, j+1 above it, never
// another block's diagonal entries, so all blocks are computed in one
// phase (one thread per block, which also writes its own 2x2 entries), all
// row rotations (and sign changes) applied in a second and all column
// rotations in a third.  Scratch: 6 doubles per slot, 3n in sd.
// ---------------------------------------------------------------------------
template <class X>
QZ_HD void cta_std_all(X& x, WinState& w, double* sd) {
  const int n = w.n;
  const int nslot = n / 2;  // block starts are >= 2 apart: slot j/2 is unique
  for (int k = x.tid; k < nslot; k += x.nt) sd[6 * k] = 0.0;
  x.sync();
  // phase A: block j (H(j+1, j) != 0) -> rotations, signs, new block
  for (int j = x.tid; j + 1 < n; j += x.nt) {
    if (w.H(j + 1, j) == 0.0 || (j > 0 && w.H(j, j - 1) != 0.0)) continue;
    double A[4] = {w.H(j, j), w.H(j + 1, j), w.H(j, j + 1), w.H(j + 1, j + 1)};
    double B[4] = {w.T(j, j), w.T(j + 1, j), w.T(j, j + 1), w.T(j + 1, j + 1)};
    Std2 o;
    std2x2(A, B, o);
    double* r = sd + 6 * (j / 2);
    r[0] = (double)(j + 1);
    r[1] = o.csl; r[2] = o.snl; r[3] = o.csr; r[4] = o.snr;
    r[5] = (double)(o.negrow0 + 2 * o.negrow1);
    w.H(j, j) = o.a[0]; w.H(j + 1, j) = o.a[1]; w.H(j, j + 1) = o.a[2]; w.H(j + 1, j + 1) = o.a[3];
    w.T(j, j) = o.b[0]; w.T(j + 1, j) = 0.0; w.T(j, j + 1) = o.b[2]; w.T(j + 1, j + 1) = o.b[3];
  }
  x.sync();
  // phase B: row rotation then sign changes of every block; items =
  // (block, column of H or T right of it, or row of Q)
  const int per = 3 * n;
  for (int idx = x.tid; idx < nslot * per; idx += x.nt) {
    const double* r = sd + 6 * (idx / per);
    if (r[0] == 0.0) continue;
    const int j = (int)r[0] - 1, it = idx % per;
    const int neg = (int)r[5];
    double* p0;
    double* p1;
    if (it < n) {
      if (it < j + 2) continue;
      p0 = &w.H(j, it); p1 = &w.H(j + 1, it);
    } else if (it < 2 * n) {
      const int c = it - n;
      if (c < j + 2) continue;
      p0 = &w.T(j, c); p1 = &w.T(j + 1, c);
    } else {
      if (!w.wantq) continue;
      const int rr = it - 2 * n;
      p0 = &w.Q(rr, j); p1 = &w.Q(rr, j + 1);
    }
    const double a = *p0, b = *p1;
    double u = r[1] * a + r[2] * b, v = -r[2] * a + r[1] * b;
    if (neg & 1) u = -u;
    if (neg & 2) v = -v;
    *p0 = u; *p1 = v;
  }
  x.sync();
  // phase C: column rotation of every block (H, T rows above it, Z rows)
  for (int idx = x.tid; idx < nslot * per; idx += x.nt) {
    const double* r = sd + 6 * (idx / per);
    if (r[0] == 0.0) continue;
    const int j = (int)r[0] - 1, it = idx % per;
    double* p0;
    double* p1;
    if (it < n) {
      if (it >= j) continue;
      p0 = &w.H(it, j); p1 = &w.H(it, j + 1);
    } else if (it < 2 * n) {
      const int rr = it - n;
      if (rr >= j) continue;
      p0 = &w.T(rr, j); p1 = &w.T(rr, j + 1);
    } else {
      if (!w.wantz) continue;
      const int rr = it - 2 * n;
      p0 = &w.Z(rr, j); p1 = &w.Z(rr, j + 1);
    }
    const double a = *p0, b = *p1;
    *p0 = r[3] * a + r[4] * b;
    *p1 = -r[4] * a + r[3] * b;
  }
  x.sync();
}

// ---------------------------------------------------------------------------
// Infinite eigenvalues: zero at T(jz,jz) in the active block [f, l].
// ---------------------------------------------------------------------------
// top of the block: row rotation zeroing H(f+1,f) splits off the 1x1 (inf)
template <class X>
QZ_HD void cta_inf_top(X& x, WinState& w, int f) {
  double c, s, r;
  lartg(w.H(f, f), w.H(f + 1, f), c, s, r);
  x.sync();
  par_rot_rows(x, w.H, f, f + 1, c, s, f + 1, w.n);
  par_rot_rows(x, w.T, f, f + 1, c, s, f + 1, w.n);
  if (w.wantq) par_rot_cols(x, w.Q, f, f + 1, c, s, 0, w.n);
  if (x.tid == 0) { w.H(f, f) = r; w.H(f + 1, f) = 0.0; }
  x.sync();
}
// bottom of the block: T(l,l)=0, column rotation zeroing H(l,l-1)
template <class X>
QZ_HD void cta_inf_bottom(X& x, WinState& w, int l) {
  double c, s, r;
  // pair (col l, col l-1): zero the second entry of row l
  lartg(w.H(l, l), w.H(l, l - 1), c, s, r);
  x.sync();
  par_rot_cols(x, w.H, l, l - 1, c, s, 0, l);
  par_rot_cols(x, w.T, l, l - 1, c, s, 0, l);
  if (w.wantz) par_rot_cols(x, w.Z, l, l - 1, c, s, 0, w.n);
  if (x.tid == 0) { w.H(l, l) = r; w.H(l, l - 1) = 0.0; }
  x.sync();
}
// chase the zero at T(jz,jz) down to T(l,l) (Moler-Stewart zero chasing)
template <class X>
QZ_HD void cta_inf_chase_down(X& x, WinState& w, int f, int jz, int l) {
  int n = w.n;
  for (int j = jz; j < l; ++j) {
    double c, s, r;
    // (a) rows (j, j+1): zero T(j+1,j+1)
    lartg(w.T(j, j + 1), w.T(j + 1, j + 1), c, s, r);
    x.sync();
    int hc0 = (j > f) ? j - 1 : j;
    par_rot_rows(x, w.H, j, j + 1, c, s, hc0, n);
    par_rot_rows(x, w.T, j, j + 1, c, s, j + 2, n);
    if (w.wantq) par_rot_cols(x, w.Q, j, j + 1, c, s, 0, n);
    if (x.tid == 0) { w.T(j, j + 1) = r; w.T(j + 1, j + 1) = 0.0; }
    x.sync();
    if (j > f) {
      // (b) cols (j, j-1): zero H(j+1, j-1)
      lartg(w.H(j + 1, j), w.H(j + 1, j - 1), c, s, r);
      x.sync();
      par_rot_cols(x, w.H, j, j - 1, c, s, 0, j + 1);
      par_rot_cols(x, w.T, j, j - 1, c, s, 0, j);
      if (w.wantz) par_rot_cols(x, w.Z, j, j - 1, c, s, 0, n);
      if (x.tid == 0) { w.H(j + 1, j) = r; w.H(j + 1, j - 1) = 0.0; }
      x.sync();
    }
  }
}

// ---------------------------------------------------------------------------
// One implicit double-shift QZ sweep over the active block [f, l]
// (l - f + 1 >= 3) with shift polynomial c2*M^2 - c1*M + c0.
//
// Two barriers per step.  Every thread computes the step's reflectors from
// the bulge column and the T block; thread 0 also forms the small block
// that both reflectors touch (H rows j..j+3 x columns j..j+2, the T block)
// in registers.  After the first barrier (all inputs read) the far parts
// (rows j..j+2 right of the block, columns j..j+2 above it, Q and Z), which
// are disjoint, are transformed in one pass over all threads while thread 0
// stores its block; the second barrier publishes the step.
// ---------------------------------------------------------------------------
template <class X>
QZ_HD void cta_ds_sweep_sync(X& x, WinState& w, int f, int l, double c2, double c1, double c0) {
  int n = w.n;
  for (int j = f; j < l; ++j) {
    x.count(0);
    if (j < l - 1) {
      // ---- 3x3 step at rows/cols j..j+2 ----
      double a0, a1, a2;
      if (j == f) {
        shift_column(w.H(f, f), w.H(f + 1, f), w.H(f, f + 1), w.H(f + 1, f + 1), w.H(f + 2, f + 1),
                     w.T(f, f), w.T(f, f + 1), w.T(f + 1, f + 1), c2, c1, c0, a0, a1, a2);
      } else {
        a0 = w.H(j, j - 1); a1 = w.H(j + 1, j - 1); a2 = w.H(j + 2, j - 1);
      }
      House3 PL, PR;
      double beta;
      house3(a0, a1, a2, PL, beta);
      double tb[9];
      for (int cc = 0; cc < 3; ++cc)
        for (int rr = 0; rr < 3; ++rr) tb[rr + 3 * cc] = w.T(j + rr, j + cc);
      for (int cc = 0; cc < 3; ++cc) house3_apply(PL, tb[3 * cc], tb[3 * cc + 1], tb[3 * cc + 2]);
      opposite_house3(tb, PR);
      for (int rr = 0; rr < 3; ++rr) house3_apply(PR, tb[rr], tb[rr + 3], tb[rr + 6]);
      tb[1] = 0.0; tb[2] = 0.0;
      // rows of the block touched by PR: up to j+3 while j+3 <= l
      const int nr = (j + 3 <= l) ? 4 : 3;
      const bool bt = block_thread(x);
      double hb[12];
      if (bt) {
        for (int cc = 0; cc < 3; ++cc)
          for (int rr = 0; rr < 4; ++rr) hb[rr + 4 * cc] = (rr < nr) ? w.H(j + rr, j + cc) : 0.0;
        for (int cc = 0; cc < 3; ++cc) house3_apply(PL, hb[4 * cc], hb[4 * cc + 1], hb[4 * cc + 2]);
        for (int rr = 0; rr < 4; ++rr) house3_apply(PR, hb[rr], hb[rr + 4], hb[rr + 8]);
      }
      x.sync();  // everyone has read H(.,j-1), the T block and the block
      // far parts, by index: H, T rows j..j+2 right of the block (PL), Q
      // columns j..j+2 (PL), H, T columns j..j+2 above it (PR), Z columns
      for (int t = x.tid; t < n; t += x.nt) {
        if (t >= j + 3) {
          house3_vec(PL, &w.H(j, t), 1);
          house3_vec(PL, &w.T(j, t), 1);
        }
        if (w.wantq) house3_vec(PL, &w.Q(t, j), w.Q.ld);
        if (t < j) {
          house3_vec(PR, &w.H(t, j), w.H.ld);
          house3_vec(PR, &w.T(t, j), w.T.ld);
        }
        if (w.wantz) house3_vec(PR, &w.Z(t, j), w.Z.ld);
      }
      if (bt) {
        for (int cc = 0; cc < 3; ++cc) {
          for (int rr = 0; rr < 3; ++rr) w.T(j + rr, j + cc) = tb[rr + 3 * cc];
          for (int rr = 0; rr < nr; ++rr) w.H(j + rr, j + cc) = hb[rr + 4 * cc];
        }
        if (j > f) { w.H(j, j - 1) = beta; w.H(j + 1, j - 1) = 0.0; w.H(j + 2, j - 1) = 0.0; }
      }
      x.sync();
    } else {
      // ---- final 2x2 step at rows/cols l-1, l ----
      double c, s, r;
      lartg(w.H(j, j - 1), w.H(j + 1, j - 1), c, s, r);
      double t00 = w.T(j, j), t01 = w.T(j, j + 1), t10 = w.T(j + 1, j), t11 = w.T(j + 1, j + 1);
      rot2(c, s, t00, t10);
      rot2(c, s, t01, t11);
      double cr, sr;
      opposite_rot2(t10, t11, cr, sr);
      rot2(cr, sr, t00, t01);
      rot2(cr, sr, t10, t11);
      t10 = 0.0;
      double hb[4];
      const bool bt = block_thread(x);
      if (bt) {
        hb[0] = w.H(j, j); hb[1] = w.H(j + 1, j); hb[2] = w.H(j, j + 1); hb[3] = w.H(j + 1, j + 1);
        rot2(c, s, hb[0], hb[1]);
        rot2(c, s, hb[2], hb[3]);
        rot2(cr, sr, hb[0], hb[2]);
        rot2(cr, sr, hb[1], hb[3]);
      }
      x.sync();
      // far parts by index: H, T rows j, j+1 right of the block, Q columns
      // (row rotation); H, T columns j, j+1 above it, Z columns (column one)
      for (int t = x.tid; t < n; t += x.nt) {
        if (t >= j + 2) {
          rot_vec(c, s, &w.H(j, t), 1);
          rot_vec(c, s, &w.T(j, t), 1);
        }
        if (w.wantq) rot_vec(c, s, &w.Q(t, j), w.Q.ld);
        if (t < j) {
          rot_vec(cr, sr, &w.H(t, j), w.H.ld);
          rot_vec(cr, sr, &w.T(t, j), w.T.ld);
        }
        if (w.wantz) rot_vec(cr, sr, &w.Z(t, j), w.Z.ld);
      }
      if (bt) {
        w.T(j, j) = t00; w.T(j + 1, j) = 0.0; w.T(j, j + 1) = t01; w.T(j + 1, j + 1) = t11;
        w.H(j, j) = hb[0]; w.H(j + 1, j) = hb[1]; w.H(j, j + 1) = hb[2]; w.H(j + 1, j + 1) = hb[3];
        w.H(j, j - 1) = r; w.H(j + 1, j - 1) = 0.0;
      }
      x.sync();
    }
  }
}

// ---------------------------------------------------------------------------
// Pipelined double-shift sweep: the same transformations as
// cta_ds_sweep_sync, in the same order on every element, without barriers
// between steps.
//
// The core (warp 0, every lane computing the same values) carries the bulge
// in registers from step to step: the bulge column H(s..s+2, s-1), the T
// block T(s..s+2, s..s+2), the H block H(s..s+3, s..s+2) and column s+3 of
// both matrices (rows s..s+2), which the next block needs with PL_s
// applied.  Per step it forms PL_s and PR_s, stores the block row that
// leaves it (row s) and the new zeros, writes both reflectors to a ring in
// shared memory and posts the step.  The far threads (threads 32..nt-1,
// index t owned by far thread t mod nfar) apply the posted reflectors to
// the rest, behind the core:
//   PL_s  to H, T rows s..s+2 of columns t >= s+4 and to Q columns s..s+2,
//   PR_s  to H, T columns s..s+2 of rows t < s and to Z columns s..s+2.
// Ordering, all through release/acquire flags and one barrier of the far
// threads per step:
//   * core step s reads column s+3 after its owner applied PL_{s-1} (each
//     far warp posts prog after the PL part of a step);
//   * far step s reads block rows < s that the core stored before posting
//     step s, and far columns that other far threads transformed in
//     earlier PL parts (the far barrier at the end of every step);
//   * a ring slot is rewritten after every far thread finished the step
//     that used it (far_done).
// The final 2x2 step of the sweep runs the same way with rotations.  Every
// wait is bounded: on time-out a thread sets err and all threads leave the
// sweep at the next wait (the far threads together, through a voting
// barrier), and the sweep returns false.  An executor of one thread runs
// core step s and then far step s, which meets every dependency in program
// order and checks the split of the work on the host.
// ---------------------------------------------------------------------------
constexpr int kPipeSlots = 32;  // a power of two
constexpr int kPipeMaxFarWarps = 8;
struct PipeBuf {
  double ring[kPipeSlots][8];  // step s: PL (s, u0, u1, u2; rotation c, s), then PR
  int ready, far_done, err, pad;
  int prog[kPipeMaxFarWarps];
};
constexpr int kPipeDoubles = (int)((sizeof(PipeBuf) + 7) / 8);

QZ_HD int pipe_ld(const int* p) {
#ifdef __CUDA_ARCH__
  int v;
  asm volatile("ld.acquire.cta.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
#else
  return *(const volatile int*)p;
#endif
}
QZ_HD void pipe_st(int* p, int v) {
#ifdef __CUDA_ARCH__
  asm volatile("st.release.cta.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
#else
  *(volatile int*)p = v;
#endif
}
constexpr int kPipeSpin = 1 << 22;  // polls before a wait gives up
// wait for *p >= v; false once err is set or after kPipeSpin polls (then
// this thread sets err)
QZ_HD bool pipe_wait(PipeBuf* pb, const int* p, int v) {
  for (int it = 0; it < kPipeSpin; ++it) {
    if (pipe_ld(p) >= v) return true;
    if ((it & 31) == 31 && pipe_ld(&pb->err) != 0) return false;
  }
  pipe_st(&pb->err, 1);
  return false;
}
// barrier of the nfar far threads (named barrier 1) returning the OR of v
QZ_HD bool far_vote(int nfar, bool v) {
#ifdef __CUDA_ARCH__
  int r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.s32 p, %1, 0;\n bar.red.or.pred q, 1, %2, p;\n selp.s32 %0, 1, 0, q;\n}"
      : "=r"(r)
      : "r"((int)v), "r"(nfar)
      : "memory");
  return r != 0;
#else
  (void)nfar;
  return v;
#endif
}
QZ_HD void warp_bar() {
#ifdef __CUDA_ARCH__
  __syncwarp();
#endif
}

// the core's registers and its two kinds of step
struct DsCore {
  int f, l, nfar;
  double c2, c1, c0;
  int64_t ld;
  double* hd;  // &H(s, s)
  double* td;  // &T(s, s)
  int own;     // far thread that owns column s+3
  double a0, a1, a2;  // H(s..s+2, s-1) (the shift column at s == f)
  double tb[9];       // T(s..s+2, s..s+2), column-major
  double hb[12];      // H(s..s+3, s..s+2), column-major, rows past l zero

  QZ_HD void init(WinState& w) {
    ld = w.H.ld;
    hd = &w.H(f, f);
    td = &w.T(f, f);
    own = (f + 3) % nfar;
    for (int cc = 0; cc < 3; ++cc)
      for (int rr = 0; rr < 3; ++rr) tb[rr + 3 * cc] = td[rr + cc * ld];
    const int nr = (f + 3 <= l) ? 4 : 3;
    for (int cc = 0; cc < 3; ++cc)
      for (int rr = 0; rr < 4; ++rr) hb[rr + 4 * cc] = (rr < nr) ? hd[rr + cc * ld] : 0.0;
    a0 = a1 = a2 = 0.0;
  }
  QZ_HD double* slot_for(PipeBuf* pb, int s) const {
    if (s - f >= kPipeSlots && !pipe_wait(pb, &pb->far_done, s - kPipeSlots + 1)) return nullptr;
    return pb->ring[(s - f) & (kPipeSlots - 1)];
  }

  // 3x3 step at rows/cols s..s+2 (s <= l - 2)
  QZ_HD bool step3(PipeBuf* pb, int n, int s) {
    const int64_t l1 = ld, l2 = 2 * ld, l3 = 3 * ld;
    // entries of the next block that no transformation touches before
    // step s+1: T(s+3, s+3), H(s+3, s+3), H(s+4, s+3)
    double nt33 = 0.0, nh33 = 0.0, nh43 = 0.0;
    if (s + 1 <= l - 2) {
      nt33 = td[3 + l3];
      nh33 = hd[3 + l3];
      if (s + 4 <= l) nh43 = hd[4 + l3];
    }
    if (s == f)
      shift_column(hb[0], hb[1], hb[4], hb[5], hb[6], tb[0], tb[3], tb[4], c2, c1, c0, a0, a1, a2);
    House3 PL, PR;
    double beta;
    house3(a0, a1, a2, PL, beta);
    for (int cc = 0; cc < 3; ++cc) house3_apply(PL, tb[3 * cc], tb[3 * cc + 1], tb[3 * cc + 2]);
    for (int cc = 0; cc < 3; ++cc) house3_apply(PL, hb[4 * cc], hb[4 * cc + 1], hb[4 * cc + 2]);
    opposite_house3(tb, PR);
    for (int rr = 0; rr < 3; ++rr) house3_apply(PR, tb[rr], tb[rr + 3], tb[rr + 6]);
    tb[1] = 0.0; tb[2] = 0.0;
    for (int rr = 0; rr < 4; ++rr) house3_apply(PR, hb[rr], hb[rr + 4], hb[rr + 8]);
    double* slot = slot_for(pb, s);
    if (!slot) return false;
    slot[0] = PL.s; slot[1] = PL.u0; slot[2] = PL.u1; slot[3] = PL.u2;
    slot[4] = PR.s; slot[5] = PR.u0; slot[6] = PR.u1; slot[7] = PR.u2;
    // column s+3, rows s..s+2, once its owner has applied PL_{s-1}
    const int c3 = s + 3;
    double bh0 = 0.0, bh1 = 0.0, bh2 = 0.0, bt0 = 0.0, bt1 = 0.0, bt2 = 0.0;
    if (c3 < n) {
      if (s > f && !pipe_wait(pb, &pb->prog[own >> 5], s)) return false;
      bh0 = hd[l3]; bh1 = hd[1 + l3]; bh2 = hd[2 + l3];
      bt0 = td[l3]; bt1 = td[1 + l3]; bt2 = td[2 + l3];
    }
    house3_apply(PL, bh0, bh1, bh2);
    house3_apply(PL, bt0, bt1, bt2);
    // row s leaves the block; the bulge column becomes (beta, 0, 0)
    td[0] = tb[0]; td[l1] = tb[3]; td[l2] = tb[6];
    td[1] = 0.0; td[2] = 0.0;
    hd[0] = hb[0]; hd[l1] = hb[4]; hd[l2] = hb[8];
    if (s > f) { hd[-l1] = beta; hd[1 - l1] = 0.0; hd[2 - l1] = 0.0; }
    if (c3 < n) {
      hd[l3] = bh0; td[l3] = bt0;
      if (s == l - 2) {  // the last 3x3 step: column l+1 is the rotation step's far part
        hd[1 + l3] = bh1; hd[2 + l3] = bh2;
        td[1 + l3] = bt1; td[2 + l3] = bt2;
      }
    }
    pipe_st(&pb->ready, s + 1);
    // the next step's block
    a0 = hb[1]; a1 = hb[2]; a2 = hb[3];
    const double t11 = tb[4], t21 = tb[5], t12 = tb[7], t22 = tb[8];
    tb[0] = t11; tb[1] = t21; tb[2] = 0.0;
    tb[3] = t12; tb[4] = t22; tb[5] = 0.0;
    tb[6] = bt1; tb[7] = bt2; tb[8] = nt33;
    const double h11 = hb[5], h21 = hb[6], h31 = hb[7], h12 = hb[9], h22 = hb[10], h32 = hb[11];
    hb[0] = h11; hb[1] = h21; hb[2] = h31; hb[3] = 0.0;
    hb[4] = h12; hb[5] = h22; hb[6] = h32; hb[7] = 0.0;
    hb[8] = bh1; hb[9] = bh2; hb[10] = nh33; hb[11] = nh43;
    hd += ld + 1;
    td += ld + 1;
    if (++own == nfar) own = 0;
    return true;
  }

  // final 2x2 step at rows/cols l-1, l (the block carried from step l-2)
  QZ_HD bool step2(PipeBuf* pb) {
    const int j = l - 1;
    const int64_t l1 = ld;
    double c, sn, r;
    lartg(a0, a1, c, sn, r);
    double t00 = tb[0], t10 = tb[1], t01 = tb[3], t11 = tb[4];
    rot2(c, sn, t00, t10);
    rot2(c, sn, t01, t11);
    double cr, sr;
    opposite_rot2(t10, t11, cr, sr);
    rot2(cr, sr, t00, t01);
    rot2(cr, sr, t10, t11);
    double h00 = hb[0], h10 = hb[1], h01 = hb[4], h11 = hb[5];
    rot2(c, sn, h00, h10);
    rot2(c, sn, h01, h11);
    rot2(cr, sr, h00, h01);
    rot2(cr, sr, h10, h11);
    double* slot = slot_for(pb, j);
    if (!slot) return false;
    slot[0] = c; slot[1] = sn; slot[4] = cr; slot[5] = sr;
    td[0] = t00; td[1] = 0.0; td[l1] = t01; td[1 + l1] = t11;
    hd[0] = h00; hd[1] = h10; hd[l1] = h01; hd[1 + l1] = h11;
    hd[-l1] = r; hd[1 - l1] = 0.0;
    pipe_st(&pb->ready, j + 1);
    return true;
  }
};

// far step s of far thread fid (of nfar; lane and warp within the far
// threads).  Returns false when the sweep is abandoned (same on every far
// thread).
QZ_HD bool ds_far_step(WinState& w, PipeBuf* pb, int f, int l, int s, int fid, int nfar, int lane, int warp) {
  const int n = w.n;
  const double* slot = pb->ring[(s - f) & (kPipeSlots - 1)];
  const bool ok = pipe_wait(pb, &pb->ready, s + 1);
  if (ok) {
    if (s < l - 1) {
      const House3 PL{slot[0], slot[1], slot[2], slot[3]};
      for (int t = fid; t < n; t += nfar) {
        if (t >= s + 4) {
          house3_vec(PL, &w.H(s, t), 1);
          house3_vec(PL, &w.T(s, t), 1);
        }
        if (w.wantq) house3_vec(PL, &w.Q(t, s), w.Q.ld);
      }
    } else {
      const double c = slot[0], sn = slot[1];
      for (int t = fid; t < n; t += nfar) {
        if (t >= s + 2) {
          rot_vec(c, sn, &w.H(s, t), 1);
          rot_vec(c, sn, &w.T(s, t), 1);
        }
        if (w.wantq) rot_vec(c, sn, &w.Q(t, s), w.Q.ld);
      }
    }
  }
  warp_bar();
  if (lane == 0) pipe_st(&pb->prog[warp], s + 1);
  if (ok) {
    if (s < l - 1) {
      const House3 PR{slot[4], slot[5], slot[6], slot[7]};
      for (int t = fid; t < n; t += nfar) {
        if (t < s) {
          house3_vec(PR, &w.H(t, s), w.H.ld);
          house3_vec(PR, &w.T(t, s), w.T.ld);
        }
        if (w.wantz) house3_vec(PR, &w.Z(t, s), w.Z.ld);
      }
    } else {
      const double cr = slot[4], sr = slot[5];
      for (int t = fid; t < n; t += nfar) {
        if (t < s) {
          rot_vec(cr, sr, &w.H(t, s), w.H.ld);
          rot_vec(cr, sr, &w.T(t, s), w.T.ld);
        }
        if (w.wantz) rot_vec(cr, sr, &w.Z(t, s), w.Z.ld);
      }
    }
  }
  const bool stop = far_vote(nfar, pipe_ld(&pb->err) != 0);
  if (fid == 0) pipe_st(&pb->far_done, s + 1);
  return !stop;
}

template <class X>
QZ_HD bool cta_ds_sweep_pipe(X& x, PipeBuf* pb, WinState& w, int f, int l, double c2, double c1, double c0) {
  if (x.tid == 0) {
    pb->ready = f; pb->far_done = f; pb->err = 0;
    for (int k = 0; k < kPipeMaxFarWarps; ++k) pb->prog[k] = f;
  }
  x.sync();
  const int nfar = (x.nt == 1) ? 1 : x.nt - 32;
  if (x.tid < 32) {
    DsCore core{f, l, nfar, c2, c1, c0};
    core.init(w);
    for (int s = f; s < l; ++s) {
      x.count(0);
      const bool ok = (s < l - 1) ? core.step3(pb, w.n, s) : core.step2(pb);
      if (!ok) break;
      if (x.nt == 1 && !ds_far_step(w, pb, f, l, s, 0, 1, 0, 0)) break;
    }
  } else {
    const int fid = x.tid - 32;
    for (int s = f; s < l; ++s)
      if (!ds_far_step(w, pb, f, l, s, fid, nfar, fid & 31, fid >> 5)) break;
  }
  x.sync();
  return pb->err == 0;
}

// the executor's pipeline buffer, if it has one
template <class X>
QZ_HD auto pipe_of(X& x, int) -> decltype(x.pipe) {
  return x.pipe;
}
template <class X>
QZ_HD PipeBuf* pipe_of(X&, long) {
  return nullptr;
}

// One double-shift sweep: pipelined when the executor provides a pipeline
// buffer (one thread, or 64 or more threads in whole warps), otherwise with
// two barriers per step.  False if a pipelined sweep gave up waiting.
template <class X>
QZ_HD bool cta_ds_sweep(X& x, WinState& w, int f, int l, double c2, double c1, double c0) {
  PipeBuf* pb = pipe_of(x, 0);
  if (pb && (x.nt == 1 || (x.nt >= 64 && x.nt % 32 == 0 && x.nt - 32 <= 32 * kPipeMaxFarWarps)))
    return cta_ds_sweep_pipe(x, pb, w, f, l, c2, c1, c0);
  cta_ds_sweep_sync(x, w, f, l, c2, c1, c0);
  return true;
}

// negligible-subdiagonal test shared by all deflation scans
QZ_HD bool negligible_sub(double hsub, double hkm1, double hkk, const Tol& t) {
  double tst = fabs(hkm1) + fabs(hkk);
  return fabs(hsub) <= dmax(t.smlnum, t.ulp * tst);
}

// ---------------------------------------------------------------------------
// Small QZ: reduce the whole window (n x n) to generalized real Schur form.
// Returns 0 on success, or ilast+1 (1-based index of the last unconverged
// row) if maxit iterations did not suffice.
// ---------------------------------------------------------------------------
template <class X>
QZ_HD int cta_small_qz(X& x, WinState& w, int maxit) {
  int n = w.n;
  int ilast = n - 1;
  int iiter = 0, jiter = 0;
  while (ilast >= 0) {
    if (x.tid == 0) {
      int ifirst = 0;
      for (int j = ilast; j >= 1; --j) {
        double tst = fabs(w.H(j - 1, j - 1)) + fabs(w.H(j, j));
        if (tst == 0.0) tst = fabs(w.H(j - 1, j)) + fabs(w.H(j, j - 1));
        if (fabs(w.H(j, j - 1)) <= dmax(w.tol.smlnum, w.tol.ulp * tst)) {
          w.H(j, j - 1) = 0.0;
          ifirst = j;
          break;
        }
      }
      int jz = -1;
      for (int j = ilast; j >= ifirst; --j) {
        if (fabs(w.T(j, j)) <= w.tol.ttol) { w.T(j, j) = 0.0; jz = j; break; }
      }
      x.si[0] = ifirst;
      x.si[1] = jz;
    }
    x.sync();
    int ifirst = x.si[0], jz = x.si[1];
    x.sync();
    if (ifirst == ilast) { ilast -= 1; iiter = 0; continue; }
    if (jz >= 0) {
      if (jz == ifirst) {
        cta_inf_top(x, w, ifirst);
      } else {
        if (jz < ilast) cta_inf_chase_down(x, w, ifirst, jz, ilast);
        cta_inf_bottom(x, w, ilast);
        ilast -= 1;
      }
      iiter = 0;
      continue;
    }
    if (ifirst + 1 == ilast) {
      cta_std2x2(x, w, ifirst);
      ilast -= 2;
      iiter = 0;
      continue;
    }
    ++iiter;
    ++jiter;
    if (jiter > maxit) return ilast + 1;
    double c2, c1, c0;
    int l = ilast;
    if (iiter % 10 == 0) {
      // exceptional shift from the bottom subdiagonals
      double sc = fabs(w.H(l, l - 1) / w.T(l - 1, l - 1)) + fabs(w.H(l - 1, l - 2) / w.T(l - 2, l - 2));
      double h11 = 0.75 * sc + w.H(l, l) / w.T(l, l);
      c2 = 1.0;
      c1 = 2.0 * h11;
      c0 = h11 * h11 + 0.4375 * sc * sc;
    } else {
      pencil2_poly(w.H(l - 1, l - 1), w.H(l, l - 1), w.H(l - 1, l), w.H(l, l),
                   w.T(l - 1, l - 1), w.T(l - 1, l), w.T(l, l), c2, c1, c0);
    }
    if (!cta_ds_sweep(x, w, ifirst, ilast, c2, c1, c0)) return ilast + 1;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Block swapping (reordering) of a generalized real Schur form.
// ---------------------------------------------------------------------------
// Small dense helpers on M x M (M <= 4) column-major arrays.  Every loop
// bound is a compile-time constant so the arrays stay in registers.
template <int M, bool TA, bool TB>
QZ_HD void small_mm(const double* A, const double* B, double* C) {
#pragma unroll
  for (int i = 0; i < M; ++i)
#pragma unroll
    for (int j = 0; j < M; ++j) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < M; ++k) {
        double a = TA ? A[k + M * i] : A[i + M * k];
        double b = TB ? B[j + M * k] : B[k + M * j];
        acc += a * b;
      }
      C[i + M * j] = acc;
    }
}

// Full orthogonal Q (M x M) from Householder QR of the M x K matrix X
// (column-major, ld M); the first K columns of Q span range(X).
template <int M, int K>
QZ_HD void small_qr_q(double* X, double* Q) {
#pragma unroll
  for (int i = 0; i < M * M; ++i) Q[i] = (i % (M + 1) == 0) ? 1.0 : 0.0;
#pragma unroll
  for (int c = 0; c < K; ++c) {
    double mx = 0.0;
#pragma unroll
    for (int i = c; i < M; ++i) mx = dmax(mx, fabs(X[i + M * c]));
    if (mx == 0.0) continue;
    double nrm = 0.0;
    const double rmx = 1.0 / mx;
#pragma unroll
    for (int i = c; i < M; ++i) { double t = X[i + M * c] * rmx; nrm += t * t; }
    nrm = sqrt(nrm) * mx;
    double alpha = X[c + M * c];
    double beta = -dsign(nrm, alpha);
    double v[M];
    v[0] = 1.0;
    double sc = 1.0 / (alpha - beta);
#pragma unroll
    for (int i = c + 1; i < M; ++i) v[i - c] = X[i + M * c] * sc;
    double tau = (beta - alpha) / beta;
#pragma unroll
    for (int j = c; j < K; ++j) {
      double t = 0.0;
#pragma unroll
      for (int i = c; i < M; ++i) t += v[i - c] * X[i + M * j];
      t *= tau;
#pragma unroll
      for (int i = c; i < M; ++i) X[i + M * j] -= t * v[i - c];
    }
#pragma unroll
    for (int i = 0; i < M; ++i) {
      double t = 0.0;
#pragma unroll
      for (int r = c; r < M; ++r) t += Q[i + M * r] * v[r - c];
      t *= tau;
#pragma unroll
      for (int r = c; r < M; ++r) Q[i + M * r] -= t * v[r - c];
    }
  }
}

// Double-double arithmetic (a value is hi + lo with |lo| <= ulp(hi)/2),
// built from the error-free transformations TwoSum (Knuth) and TwoProd by
// FMA (Dekker's product in its FMA form).  Used only where a swap of
// nearby eigenvalues needs its orthogonal factors to more than working
// precision.
struct DD {
  double hi, lo;
};
QZ_HD DD dd_from(double a) { return DD{a, 0.0}; }
QZ_HD DD dd_add(DD a, DD b) {
  const double s = a.hi + b.hi, z = s - a.hi;
  const double e = (a.hi - (s - z)) + (b.hi - z) + a.lo + b.lo;
  const double h = s + e;
  return DD{h, e - (h - s)};
}
QZ_HD DD dd_neg(DD a) { return DD{-a.hi, -a.lo}; }
QZ_HD DD dd_mul(DD a, DD b) {
  const double p = a.hi * b.hi;
  const double e = fma(a.hi, b.hi, -p) + (a.hi * b.lo + a.lo * b.hi);
  const double h = p + e;
  return DD{h, e - (h - p)};
}
// quotient: the double quotient corrected by one Newton step on the residual
QZ_HD DD dd_div(DD a, DD b) {
  const double q = a.hi / b.hi;
  const DD r = dd_add(a, dd_neg(dd_mul(b, dd_from(q))));
  const double q2 = r.hi / b.hi;
  const double h = q + q2;
  return DD{h, q2 - (h - q)};
}
QZ_HD DD dd_sqrt(DD a) {
  if (!(a.hi > 0.0)) return DD{0.0, 0.0};
  const double x = sqrt(a.hi);
  const DD r = dd_add(a, dd_neg(dd_mul(dd_from(x), dd_from(x))));
  const double c = r.hi / (2.0 * x);
  const double h = x + c;
  return DD{h, c - (h - x)};
}

// small_qr_q in double-double: Householder QR of the M x K matrix X
// (double input), Q (M x M) accumulated in double-double and rounded.
template <int M, int K>
QZ_HD void small_qr_q_dd(const double* X0, double* Qout) {
  DD X[M * K], Q[M * M];
#pragma unroll
  for (int i = 0; i < M * K; ++i) X[i] = dd_from(X0[i]);
#pragma unroll
  for (int i = 0; i < M * M; ++i) Q[i] = dd_from((i % (M + 1) == 0) ? 1.0 : 0.0);
#pragma unroll
  for (int c = 0; c < K; ++c) {
    DD nrm2 = dd_from(0.0);
#pragma unroll
    for (int i = c; i < M; ++i) nrm2 = dd_add(nrm2, dd_mul(X[i + M * c], X[i + M * c]));
    if (nrm2.hi == 0.0) continue;
    const DD nrm = dd_sqrt(nrm2);
    const DD alpha = X[c + M * c];
    const DD beta = (alpha.hi >= 0.0) ? dd_neg(nrm) : nrm;
    const DD am = dd_add(alpha, dd_neg(beta));
    DD v[M];
    v[0] = dd_from(1.0);
#pragma unroll
    for (int i = c + 1; i < M; ++i) v[i - c] = dd_div(X[i + M * c], am);
    const DD tau = dd_div(dd_add(beta, dd_neg(alpha)), beta);
#pragma unroll
    for (int j = c; j < K; ++j) {
      DD t = dd_from(0.0);
#pragma unroll
      for (int i = c; i < M; ++i) t = dd_add(t, dd_mul(v[i - c], X[i + M * j]));
      t = dd_mul(t, tau);
#pragma unroll
      for (int i = c; i < M; ++i) X[i + M * j] = dd_add(X[i + M * j], dd_neg(dd_mul(t, v[i - c])));
    }
#pragma unroll
    for (int i = 0; i < M; ++i) {
      DD t = dd_from(0.0);
#pragma unroll
      for (int r = c; r < M; ++r) t = dd_add(t, dd_mul(Q[i + M * r], v[r - c]));
      t = dd_mul(t, tau);
#pragma unroll
      for (int r = c; r < M; ++r) Q[i + M * r] = dd_add(Q[i + M * r], dd_neg(dd_mul(t, v[r - c])));
    }
  }
#pragma unroll
  for (int i = 0; i < M * M; ++i) Qout[i] = Q[i].hi + Q[i].lo;
}

// Gaussian elimination with row pivoting on an S x S system (S <= 8,
// column-major, ld S): the pivot of column k is the largest entry of that
// column at or below the diagonal, so the search is S - k compares (complete
// pivoting searches (S - k)^2 entries, which made the serial solve the
// longest part of a block swap).  The elimination steps are unrolled by
// template recursion and row exchanges are selects, so every index is a
// compile-time constant and the system stays in registers.  Tiny pivots are
// replaced by smin (the DGETC2 device); an inaccurate solution is caught by
// the swap's stability test, which then rejects the swap.
template <int S, int K>
struct SmallElim {
  static QZ_HD void run(double* A, double* rhs, double* rpv, double smin, bool& exact) {
    if constexpr (K < S) {
      int pi = K;
      double best = fabs(A[K + S * K]);
#pragma unroll
      for (int i = K + 1; i < S; ++i) {
        const double v = fabs(A[i + S * K]);
        if (v > best) { best = v; pi = i; }
      }
#pragma unroll
      for (int i = K + 1; i < S; ++i) {
        const bool sw = (pi == i);
#pragma unroll
        for (int j = K; j < S; ++j) {
          const double a = A[K + S * j], b = A[i + S * j];
          A[K + S * j] = sw ? b : a;
          A[i + S * j] = sw ? a : b;
        }
        const double a = rhs[K], b = rhs[i];
        rhs[K] = sw ? b : a;
        rhs[i] = sw ? a : b;
      }
      if (fabs(A[K + S * K]) < smin) { A[K + S * K] = smin; exact = false; }
      const double rpiv = 1.0 / A[K + S * K];
      rpv[K] = rpiv;
#pragma unroll
      for (int i = K + 1; i < S; ++i) {
        const double f = A[i + S * K] * rpiv;
#pragma unroll
        for (int j = K + 1; j < S; ++j) A[i + S * j] -= f * A[K + S * j];
        rhs[i] -= f * rhs[K];
      }
      SmallElim<S, K + 1>::run(A, rhs, rpv, smin, exact);
    }
  }
};
template <int S>
QZ_HD bool small_solve_cp(double* A, double* rhs, double smin) {
  bool exact = true;
  double rpv[S];  // reciprocal pivots, reused by the back substitution
  SmallElim<S, 0>::run(A, rhs, rpv, smin, exact);
#pragma unroll
  for (int k = S - 1; k >= 0; --k) {
    double acc = rhs[k];
#pragma unroll
    for (int j = k + 1; j < S; ++j) acc -= A[k + S * j] * rhs[j];
    rhs[k] = acc * rpv[k];
  }
  return exact;
}

// Compute the orthogonal Qs, Zs (M x M, M = N1+N2) that swap the diagonal
// blocks of the M x M pencil block (Hb, Tb) (upper block triangular, read
// from the window) by the generalized Sylvester equation
//   A11 R - L A22 = -A12,  B11 R - L B22 = -B12
// (the DTGEX2 method, dtgex2.f).  On success S2, T2 receive
// Qs^T (Hb, Tb) Zs with the new lower-left N1 x N2 block exactly zero.
// Returns false if the swap fails the weak stability test (then nothing
// is applied).
// The Kronecker form of the swap's Sylvester system: unknowns vec(R),
// vec(L) (N1 x N2 each), rows of the A- then the B-equations.
template <int N1, int N2>
QZ_HD void swap_system(MatV Hb, MatV Tb, double* A, double* rhs) {
  constexpr int NQ = N1 * N2, NS = 2 * NQ;
#pragma unroll
  for (int i = 0; i < NS * NS; ++i) A[i] = 0.0;
#pragma unroll
  for (int j = 0; j < N2; ++j)
#pragma unroll
    for (int i = 0; i < N1; ++i) {
      const int row = i + N1 * j;
#pragma unroll
      for (int k = 0; k < N1; ++k) {
        A[row + NS * (k + N1 * j)] += Hb(i, k);
        A[(row + NQ) + NS * (k + N1 * j)] += Tb(i, k);
      }
#pragma unroll
      for (int k = 0; k < N2; ++k) {
        A[row + NS * (NQ + i + N1 * k)] -= Hb(N1 + k, N1 + j);
        A[(row + NQ) + NS * (NQ + i + N1 * k)] -= Tb(N1 + k, N1 + j);
      }
      rhs[row] = -Hb(i, N1 + j);
      rhs[row + NQ] = -Tb(i, N1 + j);
    }
}

// From the solution x = [vec R; vec L]: Zs, Qs (orthogonal factors of [R; I]
// and [L; I]) and S2 = Qs^T Hb Zs, T2 = Qs^T Tb Zs; returns the squared
// Frobenius norm of the new lower-left N1 x N2 blocks.
template <int N1, int N2>
QZ_HD double swap_apply(MatV Hb, MatV Tb, const double* x, double* S2, double* T2, double* Qs, double* Zs,
                        bool dd = false) {
  constexpr int M = N1 + N2, NQ = N1 * N2;
  double XR[M * N2], XL[M * N2];
#pragma unroll
  for (int j = 0; j < N2; ++j) {
#pragma unroll
    for (int i = 0; i < N1; ++i) {
      XR[i + M * j] = x[i + N1 * j];
      XL[i + M * j] = x[NQ + i + N1 * j];
    }
#pragma unroll
    for (int i = 0; i < N2; ++i) {
      XR[N1 + i + M * j] = (i == j) ? 1.0 : 0.0;
      XL[N1 + i + M * j] = (i == j) ? 1.0 : 0.0;
    }
  }
  if (dd) {
    small_qr_q_dd<M, N2>(XR, Zs);
    small_qr_q_dd<M, N2>(XL, Qs);
  } else {
    small_qr_q<M, N2>(XR, Zs);
    small_qr_q<M, N2>(XL, Qs);
  }
  double blk[M * M], tmp[M * M];
#pragma unroll
  for (int c = 0; c < M; ++c)
#pragma unroll
    for (int r = 0; r < M; ++r) blk[r + M * c] = Hb(r, c);
  small_mm<M, false, false>(blk, Zs, tmp);
  small_mm<M, true, false>(Qs, tmp, S2);
#pragma unroll
  for (int c = 0; c < M; ++c)
#pragma unroll
    for (int r = 0; r < M; ++r) blk[r + M * c] = Tb(r, c);
  small_mm<M, false, false>(blk, Zs, tmp);
  small_mm<M, true, false>(Qs, tmp, T2);
  double ll = 0.0;
#pragma unroll
  for (int j = 0; j < N2; ++j)
#pragma unroll
    for (int i = N2; i < M; ++i) ll += S2[i + M * j] * S2[i + M * j] + T2[i + M * j] * T2[i + M * j];
  return ll;
}

// The retry of a swap that failed the weak stability test (rare), from
// the block itself: the Sylvester solution refined once with its residual
// b - K x in twice the working precision (exact products by FMA,
// compensated summation: the Dot2 algorithm of Ogita, Rump and Oishi,
// SIAM J. Sci. Comput. 26 (2005)), and the orthogonal factors formed in
// double-double.  For nearby eigenvalues |x| is large: in working
// precision the residual cannot fall below eps |K| |x|, and a Householder
// QR of [R; I] loses the subspace by about eps |R|, either of which can
// push an acceptable swap over the threshold.  Not inlined, and its
// outputs go straight to the caller's (shared) arrays, so its temporaries
// do not weigh on the registers of the kernels that swap.
template <int N1, int N2>
QZ_NOINLINE bool swap_retry(MatV Hb, MatV Tb, double* S2, double* T2, double* Qs, double* Zs, double ulp,
                            double smlnum) {
  constexpr int M = N1 + N2, NQ = N1 * N2, NS = 2 * NQ;
  double fn = 0.0;
  for (int c = 0; c < M; ++c)
    for (int r = 0; r < M; ++r) fn += Hb(r, c) * Hb(r, c) + Tb(r, c) * Tb(r, c);
  fn = sqrt(fn);
  const double thresh = dmax(20.0 * ulp * fn, smlnum);
  const double smin = dmax(ulp * fn * 1e-3, smlnum);
  double x[NS], A[NS * NS], r[NS];
  swap_system<N1, N2>(Hb, Tb, A, x);
  small_solve_cp<NS>(A, x, smin);
  swap_system<N1, N2>(Hb, Tb, A, r);
  for (int i = 0; i < NS; ++i) {
    double sum = r[i], comp = 0.0;
    for (int j = 0; j < NS; ++j) {
      const double p = -A[i + NS * j] * x[j];
      const double q = fma(-A[i + NS * j], x[j], -p);
      const double t = sum + p, z = t - sum;
      comp += ((sum - (t - z)) + (p - z)) + q;
      sum = t;
    }
    r[i] = sum + comp;
  }
  small_solve_cp<NS>(A, r, smin);
  for (int i = 0; i < NS; ++i) {
    x[i] += r[i];
    if (!isfinite(x[i])) return false;
  }
  const double ll = swap_apply<N1, N2>(Hb, Tb, x, S2, T2, Qs, Zs, true);
  if (!(sqrt(ll) <= thresh)) return false;
  for (int j = 0; j < N2; ++j)
    for (int i = N2; i < M; ++i) { S2[i + M * j] = 0.0; T2[i + M * j] = 0.0; }
  return true;
}

// 1: accepted; 0: rejected; -1: failed the stability test in working
// precision (swap_retry may still accept it)
template <int N1, int N2>
QZ_HD int swap_compute_try(MatV Hb, MatV Tb, double* S2, double* T2, double* Qs, double* Zs, double ulp,
                           double smlnum) {
  constexpr int M = N1 + N2, NQ = N1 * N2, NS = 2 * NQ;
  double fn = 0.0;
#pragma unroll
  for (int c = 0; c < M; ++c)
#pragma unroll
    for (int r = 0; r < M; ++r) fn += Hb(r, c) * Hb(r, c) + Tb(r, c) * Tb(r, c);
  fn = sqrt(fn);
  const double thresh = dmax(20.0 * ulp * fn, smlnum);
  const double smin = dmax(ulp * fn * 1e-3, smlnum);
  double x[NS];
  {
    double A[NS * NS];
    swap_system<N1, N2>(Hb, Tb, A, x);
    small_solve_cp<NS>(A, x, smin);
  }
#pragma unroll
  for (int i = 0; i < NS; ++i)
    if (!isfinite(x[i])) return 0;
  double ll = swap_apply<N1, N2>(Hb, Tb, x, S2, T2, Qs, Zs);
  if (!(sqrt(ll) <= thresh)) return -1;
#pragma unroll
  for (int j = 0; j < N2; ++j)
#pragma unroll
    for (int i = N2; i < M; ++i) { S2[i + M * j] = 0.0; T2[i + M * j] = 0.0; }
  return 1;
}

template <int N1, int N2>
QZ_HD bool swap_compute(MatV Hb, MatV Tb, double* S2, double* T2, double* Qs, double* Zs, double ulp,
                        double smlnum) {
  const int r = swap_compute_try<N1, N2>(Hb, Tb, S2, T2, Qs, Zs, ulp, smlnum);
  if (r < 0) return swap_retry<N1, N2>(Hb, Tb, S2, T2, Qs, Zs, ulp, smlnum);
  return r > 0;
}

// Swap of two 1x1 blocks by two rotations (the direct 1x1 case of
// Kagstrom and Poromaa's swapping): for the block pencil ([a b; 0 c],
// [d e; 0 f]) the right rotation's first column is the eigenvector of the
// trailing eigenvalue, (f S - c T) z = 0, i.e. z ~ (f b - c e, -(f a - c d));
// S z and T z are then parallel and the left rotation maps the larger
// (relative to its matrix) onto e1.  The weak stability test of the
// general path decides acceptance; close eigenvalues make z inaccurate, and
// the caller then takes the generalized Sylvester path.  Same outputs as
// swap_compute<1, 1>.
QZ_HD bool swap_compute11(MatV Hb, MatV Tb, double* S2, double* T2, double* Qs, double* Zs, double ulp,
                          double smlnum) {
  const double a = Hb(0, 0), b = Hb(0, 1), c = Hb(1, 1), d = Tb(0, 0), e = Tb(0, 1), f = Tb(1, 1);
  const double fn = sqrt(a * a + b * b + c * c + Hb(1, 0) * Hb(1, 0) + d * d + e * e + f * f + Tb(1, 0) * Tb(1, 0));
  const double thresh = dmax(20.0 * ulp * fn, smlnum);
  double hm = dmax(fabs(a), dmax(fabs(b), fabs(c))), tm = dmax(fabs(d), dmax(fabs(e), fabs(f)));
  hm = (hm > 0.0 && isfinite(hm)) ? 1.0 / hm : 1.0;
  tm = (tm > 0.0 && isfinite(tm)) ? 1.0 / tm : 1.0;
  const double as = a * hm, bs = b * hm, cs = c * hm, ds = d * tm, es = e * tm, fs = f * tm;
  const double F = fs * as - cs * ds, G = fs * bs - cs * es;
  double cz, sz, rr;
  lartg(G, -F, cz, sz, rr);
  // S z, T z (scaled)
  const double s0 = as * cz + bs * sz, s1 = cs * sz, t0 = ds * cz + es * sz, t1 = fs * sz;
  const bool use_s = s0 * s0 + s1 * s1 >= t0 * t0 + t1 * t1;
  double cq, sq, rq;
  lartg(use_s ? s0 : t0, use_s ? s1 : t1, cq, sq, rq);
  Zs[0] = cz; Zs[1] = sz; Zs[2] = -sz; Zs[3] = cz;
  Qs[0] = cq; Qs[1] = sq; Qs[2] = -sq; Qs[3] = cq;
  // S2 = Q^T S Z, T2 = Q^T T Z (S, T upper triangular 2x2 blocks)
  const double sz0 = a * cz + b * sz, sz1 = c * sz, sz2 = -a * sz + b * cz, sz3 = c * cz;  // S Z columns
  const double tz0 = d * cz + e * sz, tz1 = f * sz, tz2 = -d * sz + e * cz, tz3 = f * cz;
  S2[0] = cq * sz0 + sq * sz1; S2[1] = -sq * sz0 + cq * sz1;
  S2[2] = cq * sz2 + sq * sz3; S2[3] = -sq * sz2 + cq * sz3;
  T2[0] = cq * tz0 + sq * tz1; T2[1] = -sq * tz0 + cq * tz1;
  T2[2] = cq * tz2 + sq * tz3; T2[3] = -sq * tz2 + cq * tz3;
  const double ll = S2[1] * S2[1] + T2[1] * T2[1];
  if (!(sqrt(ll) <= thresh)) return false;
  S2[1] = 0.0;
  T2[1] = 0.0;
  return true;
}

// Swap the blocks at j1 (size N1) and j1+N1 (size N2) of the window.
// Thread 0 computes, everyone applies.  Returns false (nothing changed)
// if the swap was rejected.
template <int N1, int N2, class X>
QZ_HD bool cta_swap_t(X& x, WinState& w, int j1, bool restd) {
  constexpr int M = N1 + N2;
  double* sQ = x.sd;       // 16
  double* sZ = x.sd + 16;  // 16
  double* sS = x.sd + 32;  // 16
  double* sT = x.sd + 48;  // 16
  x.count(1);
  if (x.tid == 0) {
    double S2[M * M], T2[M * M], Qs[M * M], Zs[M * M];
    const MatV hb{&w.H(j1, j1), w.H.ld}, tb{&w.T(j1, j1), w.T.ld};
    int res;
    if constexpr (N1 == 1 && N2 == 1)
      // two rotations; the Sylvester path where they fail the stability test
      res = swap_compute11(hb, tb, S2, T2, Qs, Zs, w.tol.ulp, w.tol.smlnum)
                ? 1
                : swap_compute_try<1, 1>(hb, tb, S2, T2, Qs, Zs, w.tol.ulp, w.tol.smlnum);
    else
      res = swap_compute_try<N1, N2>(hb, tb, S2, T2, Qs, Zs, w.tol.ulp, w.tol.smlnum);
    bool ok = res > 0;
    if (ok) {
#pragma unroll
      for (int i = 0; i < M * M; ++i) { sQ[i] = Qs[i]; sZ[i] = Zs[i]; sS[i] = S2[i]; sT[i] = T2[i]; }
    } else if (res < 0) {
      ok = swap_retry<N1, N2>(hb, tb, sS, sT, sQ, sZ, w.tol.ulp, w.tol.smlnum);
    }
    x.si[2] = ok ? 1 : 0;
  }
  x.sync();
  const bool ok = x.si[2] != 0;
  if (!ok) { x.sync(); return false; }
  double q[M * M], z[M * M];
#pragma unroll
  for (int i = 0; i < M * M; ++i) { q[i] = sQ[i]; z[i] = sZ[i]; }
  const int n = w.n;
  // rows j1..j1+M-1, cols j1+M..n-1 : Qs^T * rows
  for (int j = j1 + M + x.tid; j < n; j += x.nt) {
    double hv[M], tv[M];
#pragma unroll
    for (int r = 0; r < M; ++r) { hv[r] = w.H(j1 + r, j); tv[r] = w.T(j1 + r, j); }
#pragma unroll
    for (int r = 0; r < M; ++r) {
      double ah = 0.0, at = 0.0;
#pragma unroll
      for (int k = 0; k < M; ++k) { ah += q[k + M * r] * hv[k]; at += q[k + M * r] * tv[k]; }
      w.H(j1 + r, j) = ah; w.T(j1 + r, j) = at;
    }
  }
  // cols j1..j1+M-1, rows 0..j1-1 : cols * Zs
  for (int i = x.tid; i < j1; i += x.nt) {
    double hv[M], tv[M];
#pragma unroll
    for (int c = 0; c < M; ++c) { hv[c] = w.H(i, j1 + c); tv[c] = w.T(i, j1 + c); }
#pragma unroll
    for (int c = 0; c < M; ++c) {
      double ah = 0.0, at = 0.0;
#pragma unroll
      for (int k = 0; k < M; ++k) { ah += hv[k] * z[k + M * c]; at += tv[k] * z[k + M * c]; }
      w.H(i, j1 + c) = ah; w.T(i, j1 + c) = at;
    }
  }
  if (w.wantq)
    for (int i = x.tid; i < n; i += x.nt) {
      double v[M];
#pragma unroll
      for (int c = 0; c < M; ++c) v[c] = w.Q(i, j1 + c);
#pragma unroll
      for (int c = 0; c < M; ++c) {
        double a = 0.0;
#pragma unroll
        for (int k = 0; k < M; ++k) a += v[k] * q[k + M * c];
        w.Q(i, j1 + c) = a;
      }
    }
  if (w.wantz)
    for (int i = x.tid; i < n; i += x.nt) {
      double v[M];
#pragma unroll
      for (int c = 0; c < M; ++c) v[c] = w.Z(i, j1 + c);
#pragma unroll
      for (int c = 0; c < M; ++c) {
        double a = 0.0;
#pragma unroll
        for (int k = 0; k < M; ++k) a += v[k] * z[k + M * c];
        w.Z(i, j1 + c) = a;
      }
    }
  // the block itself: M*M entries of H and T from the computed S2, T2
  for (int i = x.tid; i < M * M; i += x.nt) {
    w.H(j1 + i % M, j1 + i / M) = sS[i];
    w.T(j1 + i % M, j1 + i / M) = sT[i];
  }
  x.sync();
  // re-standardise the new diagonal blocks (moved block first, size N2);
  // without restd they stay general 2x2 blocks (T's block not triangular)
  // until a later cta_std_all
  if (restd && N2 == 2) cta_std2x2(x, w, j1);
  if (restd && N1 == 2) cta_std2x2(x, w, j1 + N2);
  return true;
}

template <class X>
QZ_HD bool cta_swap(X& x, WinState& w, int j1, int n1, int n2, bool restd = true) {
  if (n1 == 1 && n2 == 1) return cta_swap_t<1, 1>(x, w, j1, restd);
  if (n1 == 1) return cta_swap_t<1, 2>(x, w, j1, restd);
  if (n2 == 1) return cta_swap_t<2, 1>(x, w, j1, restd);
  return cta_swap_t<2, 2>(x, w, j1, restd);
}

// Move the block starting at ifst (size nb) up to position ilst
// (DTGEXC semantics for ifst > ilst).  Returns false on a rejected swap.
// restd = false leaves the 2x2 blocks it touches unstandardised (the
// caller standardises the window afterwards, cta_std_all).
template <class X>
QZ_HD bool cta_move_block(X& x, WinState& w, int ifst, int nb, int ilst, bool restd = true) {
  // reads of the block structure need no barrier of their own: every swap
  // starts (after these reads) and ends with one
  int here = ifst;
  while (here > ilst) {
    int nbn = 1;
    if (here - 2 >= ilst && w.H(here - 1, here - 2) != 0.0) nbn = 2;
    if (!cta_swap(x, w, here - nbn, nbn, nb, restd)) return false;
    here -= nbn;
    // the moved block must keep its size (a complex pair stays 2x2)
    int nbnow = (nb == 2 && w.H(here + 1, here) != 0.0) ? 2 : 1;
    if (nbnow != nb) return false;
  }
  return true;
}

}  // namespace qz

namespace qz {

// ---------------------------------------------------------------------------
// Finalisation of a Schur form held in one window: beta >= 0 for 1x1
// blocks (negate the column of H, T and Z, as DHGEQZ does) and the
// eigenvalues (alphar, alphai, beta) of every block.  2x2 blocks are
// already standardised by cta_small_qz (B diagonal, positive).
// ---------------------------------------------------------------------------
template <class X>
QZ_HD void cta_finalize(X& x, WinState& w, double* ar, double* ai, double* be) {
  int n = w.n;
  // column signs: columns are independent
  for (int j = 0; j < n; ++j) {
    bool below = (j + 1 < n) && w.H(j + 1, j) != 0.0;
    bool above = (j > 0) && w.H(j, j - 1) != 0.0;
    if (below || above) continue;
    if (!(w.T(j, j) < 0.0)) continue;
    x.sync();
    for (int i = x.tid; i <= j; i += x.nt) {
      w.H(i, j) = -w.H(i, j);
      w.T(i, j) = -w.T(i, j);
    }
    if (w.wantz)
      for (int i = x.tid; i < n; i += x.nt) w.Z(i, j) = -w.Z(i, j);
  }
  x.sync();
  for (int j = x.tid; j < n; j += x.nt) {
    bool below = (j + 1 < n) && w.H(j + 1, j) != 0.0;
    bool above = (j > 0) && w.H(j, j - 1) != 0.0;
    if (!below && !above) {
      ar[j] = w.H(j, j);
      ai[j] = 0.0;
      be[j] = w.T(j, j);
      continue;
    }
    int f = below ? j : j - 1;
    double a[4] = {w.H(f, f), w.H(f + 1, f), w.H(f, f + 1), w.H(f + 1, f + 1)};
    double o_ar[2], o_ai[2], o_be[2];
    eig2_complex(a, w.T(f, f), w.T(f + 1, f + 1), o_ar, o_ai, o_be);
    const bool second = j > f;  // selects keep the pair in registers
    ar[j] = second ? o_ar[1] : o_ar[0];
    ai[j] = second ? o_ai[1] : o_ai[0];
    be[j] = second ? o_be[1] : o_be[0];
  }
  x.sync();
}

}  // namespace qz
