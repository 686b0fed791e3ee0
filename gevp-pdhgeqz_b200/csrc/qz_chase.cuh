// CTA-level chase of a chain of 3x3 bulges through one diagonal window.
//
// Role in the reference: PDHGEQZA (bulge introduction, PDHGEQZA.f:325-420),
// PDHGEQZB + DHGEQZ5 (chase inside a window, DHGEQZ5.f:128-250) and the
// push-off at the bottom edge (PDHGEQZA.f:382-417), with the window's
// orthogonal factors U (left) and V (right) accumulated for the
// off-diagonal updates (PDHGEQZ6.f:276-380).
//
// B200 design: the whole chain advances in lockstep.  At chain step tau
// every active bulge b does one step at window row j_b = base_b + tau:
//   phase A  thread b computes the left reflector (from H(j:j+2, j-1), or
//            from the shift polynomial when the bulge is introduced), the
//            left-updated 3x3 block of T, the opposite (right) reflector
//            that clears T(j+1:j+2, j), and the final 3x3 block of T;
//   phase B  every left reflector is applied to its three rows of H and T
//            and to three columns of U (one warp per bulge, lanes over
//            the bulge's items);
//   phase C  every right reflector is applied to its three columns of H
//            and T and to three columns of V; thread b stores its T block
//            (the finished column j-1 of H is stored in phase B).
// Bulges are packed 3 rows apart: the rows touched by different left
// reflectors and the columns touched by different right reflectors are
// disjoint, and phase A reads only entries no other bulge changes in the
// same step, so the lockstep schedule equals the sequential
// bottom-bulge-first chase.
#pragma once
#include "qz_cta.cuh"

namespace qz {

struct Bulge {
  int base;   // window row of the bulge's step at tau = 0 (may be < 0)
  int tlo;    // first active chain step
  int thi;    // one past the last active chain step
  int intro;  // 1: the step at tau = tlo introduces the bulge
  double c2, c1, c0;  // shift polynomial c2 M^2 - c1 M + c0 I
};

// per-step record produced in phase A
struct BulgeRec {
  int kind;  // 0 inactive, 1: 3x3 step, 2: terminal 2x2 step
  int j;
  int writecol;  // 1: store H(j:j+2, j-1) in phase B
  House3 L;      // left reflector (kind 1); kind 2: rotation c, s in L.s, L.u0
  House3 R;      // right reflector (kind 1); kind 2: rotation c, s in R.s, R.u0
  double beta;   // new H(j, j-1)
  double tb[9];  // final T block
};

// Compute the step of one bulge at window row j.  last = last active row
// of the window (rows > last are outside the active block).
QZ_HD void bulge_step_compute(MatV H, MatV T, int j, int last, bool intro,
                              double c2, double c1, double c0, BulgeRec& r) {
  r.j = j;
  if (j + 2 <= last) {
    r.kind = 1;
    double a0, a1, a2;
    if (intro) {
      shift_column(H(j, j), H(j + 1, j), H(j, j + 1), H(j + 1, j + 1), H(j + 2, j + 1),
                   T(j, j), T(j, j + 1), T(j + 1, j + 1), c2, c1, c0, a0, a1, a2);
      r.writecol = 0;
    } else {
      a0 = H(j, j - 1); a1 = H(j + 1, j - 1); a2 = H(j + 2, j - 1);
      r.writecol = 1;
    }
    house3(a0, a1, a2, r.L, r.beta);
    double* tb = r.tb;
    for (int cc = 0; cc < 3; ++cc)
      for (int rr = 0; rr < 3; ++rr) tb[rr + 3 * cc] = T(j + rr, j + cc);
    for (int cc = 0; cc < 3; ++cc) house3_apply(r.L, tb[3 * cc], tb[3 * cc + 1], tb[3 * cc + 2]);
    opposite_house3(tb, r.R);
    for (int rr = 0; rr < 3; ++rr) house3_apply(r.R, tb[rr], tb[rr + 3], tb[rr + 6]);
    tb[1] = 0.0;
    tb[2] = 0.0;
  } else {
    // terminal 2x2 step at rows j, j+1 = last
    r.kind = 2;
    r.writecol = 1;
    double c, s, rr;
    lartg(H(j, j - 1), H(j + 1, j - 1), c, s, rr);
    double t00 = T(j, j), t01 = T(j, j + 1), t10 = T(j + 1, j), t11 = T(j + 1, j + 1);
    rot2(c, s, t00, t10);
    rot2(c, s, t01, t11);
    double cr, sr;
    opposite_rot2(t10, t11, cr, sr);
    rot2(cr, sr, t00, t01);
    rot2(cr, sr, t10, t11);
    r.L.s = c; r.L.u0 = s; r.beta = rr;
    r.R.s = cr; r.R.u0 = sr;
    r.tb[0] = t00; r.tb[1] = 0.0; r.tb[3] = t01; r.tb[4] = t11;
  }
}

// Chase a chain through a window of size wk held in H, T (wk x wk), while
// accumulating U, V (wk x wk, identity on entry).  last = last row of the
// active block inside the window (wk-1 if the block continues below).
// bl[0..nb) describe the bulges, rec is shared scratch for nb records.
template <class X>
QZ_HD void cta_chase_window(X& x, int wk, int last, MatV H, MatV T, MatV U, MatV V,
                            const Bulge* bl, int nb, int tmax, BulgeRec* rec) {
  for (int tau = 0; tau < tmax; ++tau) {
    // ---- phase A: per-bulge computations ----
    for (int b = x.tid; b < nb; b += x.nt) {
      const Bulge& g = bl[b];
      if (tau >= g.tlo && tau < g.thi) {
        bool intro = g.intro && tau == g.tlo;
        bulge_step_compute(H, T, g.base + tau, last, intro, g.c2, g.c1, g.c0, rec[b]);
      } else {
        rec[b].kind = 0;
      }
    }
    x.sync();
    // ---- phase B: left transformations ----
    // The finished column j-1 of H is stored here, before phase C: the
    // right reflector of the bulge above (rows <= j, cols j-3..j-1) must
    // see it, as in the sequential bottom-first order.
    for (int b = x.tid; b < nb; b += x.nt) {
      const BulgeRec& r = rec[b];
      if (r.kind == 0 || !r.writecol) continue;
      int j = r.j;
      H(j, j - 1) = r.beta;
      H(j + 1, j - 1) = 0.0;
      if (r.kind == 1) H(j + 2, j - 1) = 0.0;
    }
    // Items of different bulges, and different items of one bulge, touch
    // disjoint entries.  Index ownership: thread tid takes index t = tid %
    // wk of bulges b = tid / wk, tid / wk + nt / wk, ...: column t of the
    // bulge's three H rows (t >= j) and T rows (t past the T block), row t
    // of U; a reflector kept in registers per bulge, no per-item dispatch.
    const int tix = (x.nt >= wk) ? x.tid % wk : x.tid;
    const int bix = (x.nt >= wk) ? x.tid / wk : 0;
    const int bstep = (x.nt >= wk) ? x.nt / wk : 1;
    const int tstep = (x.nt >= wk) ? wk : x.nt;  // threads per bulge index set
    const bool active = bix < bstep;             // the last partial group idles
    if (active)
      for (int b = bix; b < nb; b += bstep) {
        const BulgeRec& r = rec[b];
        if (r.kind == 0) continue;
        const int j = r.j;
        const int t0 = (r.kind == 1) ? j + 3 : j + 2;
        const House3 L = r.L;
        for (int t = tix; t < wk; t += tstep) {
          if (r.kind == 1) {
            if (t >= j) house3_vec(L, &H(j, t), 1);
            if (t >= t0) house3_vec(L, &T(j, t), 1);
            house3_vec(L, &U(t, j), U.ld);
          } else {
            if (t >= j) rot_vec(L.s, L.u0, &H(j, t), 1);
            if (t >= t0) rot_vec(L.s, L.u0, &T(j, t), 1);
            rot_vec(L.s, L.u0, &U(t, j), U.ld);
          }
        }
      }
    x.sync();
    // ---- phase C: right transformations: H columns j.. (rows 0..hr-1),
    // T columns j.. above the T block, V columns j.. (all rows) ----
    if (active)
      for (int b = bix; b < nb; b += bstep) {
        const BulgeRec& r = rec[b];
        if (r.kind == 0) continue;
        const int j = r.j;
        const int hr = (r.kind == 1) ? ((j + 4 < last + 1) ? j + 4 : last + 1) : last + 1;
        const House3 R = r.R;
        for (int t = tix; t < wk; t += tstep) {
          if (r.kind == 1) {
            if (t < hr) house3_vec(R, &H(t, j), H.ld);
            if (t < j) house3_vec(R, &T(t, j), T.ld);
            house3_vec(R, &V(t, j), V.ld);
          } else {
            if (t < hr) rot_vec(R.s, R.u0, &H(t, j), H.ld);
            if (t < j) rot_vec(R.s, R.u0, &T(t, j), T.ld);
            rot_vec(R.s, R.u0, &V(t, j), V.ld);
          }
        }
      }
    // deferred stores owned by the bulge's thread
    for (int b = x.tid; b < nb; b += x.nt) {
      const BulgeRec& r = rec[b];
      if (r.kind == 1) {
        int j = r.j;
        for (int cc = 0; cc < 3; ++cc)
          for (int rr = 0; rr < 3; ++rr) T(j + rr, j + cc) = r.tb[rr + 3 * cc];
      } else if (r.kind == 2) {
        int j = r.j;
        T(j, j) = r.tb[0]; T(j + 1, j) = 0.0; T(j, j + 1) = r.tb[3]; T(j + 1, j + 1) = r.tb[4];
      }
    }
    x.sync();
  }
}

// Chase a zero diagonal entry of T from window row jz down to window row
// stop (<= last) inside a window, accumulating U and V.  If stop == last
// and deflate is set, finish with the column rotation that zeros
// H(last, last-1) (an infinite eigenvalue deflates at the bottom).
// top = first row of the active block inside the window (-1 if the block
// starts above the window).  The zero-chasing steps are those of the
// Moler-Stewart QZ (cf. PDHGEQZ8/DHGEQZ7 for the windowed form).
template <class X>
QZ_HD void cta_inf_window(X& x, int wk, int top, int jz, int stop, bool deflate,
                          MatV H, MatV T, MatV U, MatV V) {
  for (int j = jz; j < stop; ++j) {
    double c, s, r;
    lartg(T(j, j + 1), T(j + 1, j + 1), c, s, r);
    x.sync();
    int hc0 = (j > top) ? j - 1 : j;
    par_rot_rows(x, H, j, j + 1, c, s, hc0, wk);
    par_rot_rows(x, T, j, j + 1, c, s, j + 2, wk);
    par_rot_cols(x, U, j, j + 1, c, s, 0, wk);
    if (x.tid == 0) { T(j, j + 1) = r; T(j + 1, j + 1) = 0.0; }
    x.sync();
    if (j > top) {
      lartg(H(j + 1, j), H(j + 1, j - 1), c, s, r);
      x.sync();
      par_rot_cols(x, H, j, j - 1, c, s, 0, j + 1);
      par_rot_cols(x, T, j, j - 1, c, s, 0, j);
      par_rot_cols(x, V, j, j - 1, c, s, 0, wk);
      if (x.tid == 0) { H(j + 1, j) = r; H(j + 1, j - 1) = 0.0; }
      x.sync();
    }
  }
  if (deflate) {
    int l = stop;
    double c, s, r;
    lartg(H(l, l), H(l, l - 1), c, s, r);
    x.sync();
    par_rot_cols(x, H, l, l - 1, c, s, 0, l);
    par_rot_cols(x, T, l, l - 1, c, s, 0, l);
    par_rot_cols(x, V, l, l - 1, c, s, 0, wk);
    if (x.tid == 0) { H(l, l) = r; H(l, l - 1) = 0.0; }
    x.sync();
  }
}

}  // namespace qz
