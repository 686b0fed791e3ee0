// AED on a window held by one CTA: window Schur form, spike test,
// reordering, spike reflector, RQ update of T and Givens Hessenberg-
// triangular re-reduction -- the role of QZEARLY (qzearly.f:229-449) inside
// PDHGEQZ2 (PDHGEQZ2.f:315-389), and with the window equal to the whole
// small block the role of PDHGEQZ4 -> KKQZ (PDHGEQZ4.f:329-372).
//
// The window's Schur form comes from cta_small_qz_ms: a small-bulge
// multishift QZ inside the window.  Each sweep chases a chain of up to
// kMsMaxBulges bulges through the active block in lockstep
// (cta_chase_window, the same code as the sweeps of the whole pencil), with
// shifts from the eigenvalues of the active block's trailing 2*nb x 2*nb
// part, which one thread computes alone (a small double-shift QZ on a copy,
// eigenvalues only).  Blocks too short for a chain, and every tenth
// iteration without deflation (exceptional shift), take one double-shift
// sweep instead.  The lockstep chain advances every bulge one row per step,
// so a sweep of 2*nb shifts costs (L + 3 nb) steps instead of nb*L.
#pragma once
#include "qz_chase.cuh"

namespace qz {

constexpr int kMsMaxBulges = 6;       // bulges per sweep of the window QZ
constexpr int kMsMinBlock = 28;       // shorter active blocks use double shifts
// shared scratch of cta_small_qz_ms: bulge records, bulge descriptions and
// two (2*kMsMaxBulges)^2 copies of the trailing block, in doubles
constexpr int kMsScratch = kMsMaxBulges * ((int)(sizeof(BulgeRec) + sizeof(Bulge)) / 8 + 2) +
                           2 * (2 * kMsMaxBulges) * (2 * kMsMaxBulges) + 16;

// Executor for code one thread runs alone while the others wait at a
// barrier of the enclosing executor.
struct SoloExec {
  int tid, nt;
  int* si;
  double* sd;
  QZ_HD void sync() {}
  QZ_HD void stamp(int) {}
  QZ_HD void count(int) {}
};

// Shift polynomials of a chain from the Schur form (Hs, Ts) of a k x k
// block: a 2x2 block gives its own real quadratic, real eigenvalues pair in
// order.  Returns the number of polynomials written (at most nbmax).
QZ_HD int shifts_from_schur(MatV Hs, MatV Ts, int k, Bulge* bl, int nbmax) {
  int nbu = 0;
  int j = k - 1;
  double ra = 0.0, rb = 0.0;
  bool have = false;
  while (j >= 0 && nbu < nbmax) {
    double c2, c1, c0;
    if (j > 0 && Hs(j, j - 1) != 0.0) {
      pencil2_poly(Hs(j - 1, j - 1), Hs(j, j - 1), Hs(j - 1, j), Hs(j, j), Ts(j - 1, j - 1), Ts(j - 1, j), Ts(j, j),
                   c2, c1, c0);
      j -= 2;
    } else {
      const double a = Hs(j, j), b = Ts(j, j);
      j -= 1;
      if (!have) { ra = a; rb = b; have = true; continue; }
      have = false;
      c2 = rb * b; c1 = ra * b + a * rb; c0 = ra * a;
    }
    const double mx = dmax(fabs(c2), dmax(fabs(c1), fabs(c0)));
    if (!(mx > 0.0) || !isfinite(mx)) continue;
    bl[nbu].c2 = c2 / mx; bl[nbu].c1 = c1 / mx; bl[nbu].c0 = c0 / mx;
    ++nbu;
  }
  return nbu;
}

// ---------------------------------------------------------------------------
// Small QZ by small-bulge multishift sweeps: reduce the whole window to
// generalized real Schur form.  Returns 0, or ilast+1 if maxit iterations
// did not suffice.  scr: kMsScratch doubles of shared scratch.
// ---------------------------------------------------------------------------
template <class X>
QZ_HD int cta_small_qz_ms(X& x, WinState& w, int maxit, double* scr) {
  const int n = w.n;
  BulgeRec* rec = (BulgeRec*)scr;
  Bulge* bl = (Bulge*)(rec + kMsMaxBulges);
  double* tcopy = scr + kMsMaxBulges * ((int)(sizeof(BulgeRec) + sizeof(Bulge)) / 8 + 2);
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
    const int ifirst = x.si[0], jz = x.si[1];
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
    const int L = ilast - ifirst + 1;
    int nb = (L - 4) / 6;
    nb = nb < kMsMaxBulges ? nb : kMsMaxBulges;
    int nbu = 0;
    if (L >= kMsMinBlock && nb >= 2 && iiter % 10 != 0) {
      // shifts: eigenvalues of the trailing 2nb x 2nb block, one thread
      if (x.tid == 0) {
        const int k = 2 * nb, a = ilast - k + 1;
        MatV Hc{tcopy, k}, Tc{tcopy + k * k, k};
        for (int c = 0; c < k; ++c)
          for (int r = 0; r < k; ++r) {
            Hc(r, c) = (r <= c + 1) ? w.H(a + r, a + c) : 0.0;
            Tc(r, c) = (r <= c) ? w.T(a + r, a + c) : 0.0;
          }
        WinState ws;
        ws.n = k; ws.H = Hc; ws.T = Tc; ws.Q = Hc; ws.Z = Hc;
        ws.wantq = false; ws.wantz = false;
        ws.tol = w.tol;
        SoloExec solo{0, 1, x.si + 16, nullptr};  // si[16..17]: free during the window QZ
        const int inf = cta_small_qz(solo, ws, 30 * k);
        int got = (inf == 0) ? shifts_from_schur(Hc, Tc, k, bl, nb) : 0;
        for (int b = 0; b < got; ++b) {
          bl[b].base = ifirst - 3 * b;
          bl[b].tlo = 3 * b;
          bl[b].thi = ilast - bl[b].base;
          bl[b].intro = 1;
        }
        x.si[2] = got;
      }
      x.sync();
      nbu = x.si[2];
    }
    if (nbu >= 1) {
      x.count(3);
      const int tmax = ilast - (ifirst - 3 * (nbu - 1));
      cta_chase_window(x, n, ilast, w.H, w.T, w.Q, w.Z, bl, nbu, tmax, rec);
      continue;
    }
    double c2, c1, c0;
    const int l = ilast;
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
// Aggressive early deflation on a window (already copied into w, with
// w.Q = w.Z = I).  s is the spike H(kwtop, kwtop-1) (0 at the top of the
// active block).  swapfail makes every block swap report failure (a test
// hook for the failure branch).  On return:
//   si[8]  = number of undeflated eigenvalues m (positions 0..m-1)
//   si[9]  = status (0 ok, >0 small QZ failed)
//   si[10] = 1 if the window was transformed (nd > 0 or full solve)
//   sd[128..] unused
// shifts (alphar, alphai, beta) of the undeflated eigenvalues are written
// to sr/si_/sb (length >= m) by thread 0 before the spike reflector is
// applied.  When nothing deflates the window is left in Schur form but the
// caller discards it (the pencil is unchanged).
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Hessenberg-triangular re-reduction of the leading m x m block of a window
// whose T is upper triangular and whose H is full in that block, by Givens
// rotations (the job of DGGHRD at qzearly.f:449).  Pair (jc, jr): the row
// rotation G on rows jr-1, jr zeros H(jr, jc); the T(jr, jr-1) it creates
// is removed by the column rotation Z on columns jr, jr-1.
//
// One barrier per pair, with one pair of lookahead: in the phase of pair
// k, every thread applies pair k-1 to its indices of the far parts while
// the block thread (a) applies pair k-1 to the few entries pair k reads --
// row jr-2 at columns jr-1, jr (Z) and column jr-2 at rows jr-1, jr (G) --
// (b) stores pair k-1's 2x2 blocks of H and T, except the entries pair k
// recomputes, and (c) forms pair k's rotations and 2x2 blocks from them
// and publishes the rotations.  The far parts of pair k-1 exclude exactly
// the entries of (a) and (b), so each entry sees the same rotations in the
// same order as with a barrier between compute and apply.  A column ends
// with a phase that applies its last pair; the next column's first pair
// reads everything from memory.
// ---------------------------------------------------------------------------
struct HrPair {
  int jc, jr;             // pair; jr < 0: none
  double c, sn, cz, sz;   // G and Z
  double r, rz;           // new H(jr-1, jc), T(jr, jr)
  double h00, h10, h01, h11, t00, t01;  // 2x2 blocks of H and T(jr-1, .) after the pair
};

template <class X>
QZ_HD void cta_hessred(X& x, WinState& w, int m) {
  const int n = w.n;
  const bool bt = block_thread(x);
  double* slot = x.sd;  // two slots of 4 rotation values (the far threads' copy)
  HrPair p;             // pending pair (block thread: all fields; others: jc, jr)
  p.jc = -1; p.jr = -1;
  int phase = 0;
  // one phase: far parts of the pending pair p, and on the block thread its
  // stores and the next pair (kjc, kjr) (kjr < 0: none)
  auto run_phase = [&](int kjc, int kjr) {
    const bool nextsame = p.jr >= 0 && kjr >= 0 && kjc == p.jc;
    if (p.jr >= 0) {
      const int J = p.jr, jc = p.jc;
      const double* sl = slot + 4 * ((phase - 1) & 1);
      const double c = sl[0], sn = sl[1], cz = sl[2], sz = sl[3];
      for (int t = x.tid; t < n; t += x.nt) {
        if ((t >= jc + 1 && t <= J - 3) || t >= J + 1) rot_vec(c, sn, &w.H(J - 1, t), 1);
        if (t >= J + 1) rot_vec(c, sn, &w.T(J - 1, t), 1);
        if (w.wantq) rot_vec(c, sn, &w.Q(t, J - 1), w.Q.ld);
        if (t <= J - 3 || (t >= J + 1 && t < m)) rot_vec(cz, sz, &w.H(t, J), -(int64_t)w.H.ld);
        if (t <= J - 3) rot_vec(cz, sz, &w.T(t, J), -(int64_t)w.T.ld);
        if (w.wantz) rot_vec(cz, sz, &w.Z(t, J), -(int64_t)w.Z.ld);
      }
    }
    if (bt) {
      // (a) pair p on row J-2 (Z) and column J-2 (G); (b) p's stores
      double a_h01 = 0.0, a_t01 = 0.0, a_h10 = 0.0;
      if (p.jr >= 0) {
        const int J = p.jr, R = J - 2;
        double hJ = w.H(R, J), hJm = w.H(R, J - 1), tJ = w.T(R, J), tJm = w.T(R, J - 1);
        rot2(p.cz, p.sz, hJ, hJm);
        rot2(p.cz, p.sz, tJ, tJm);
        w.H(R, J) = hJ;
        w.T(R, J) = tJ;
        w.H(J, p.jc) = 0.0;
        if (R == p.jc) {
          // the column's last pair: H(J-2, J-1), T(J-2, J-1) final; column jc done
          w.H(R, J - 1) = hJm;
          w.T(R, J - 1) = tJm;
          w.H(J - 1, p.jc) = p.r;
        } else {
          double x0 = w.H(J - 1, R), x1 = w.H(J, R);
          rot2(p.c, p.sn, x0, x1);
          w.H(J, R) = x1;
          a_h01 = hJm; a_t01 = tJm; a_h10 = x0;  // entries of the next pair's blocks
        }
        if (!nextsame) { w.H(J - 1, J - 1) = p.h00; w.T(J - 1, J - 1) = p.t00; }
        w.H(J, J - 1) = p.h10; w.H(J - 1, J) = p.h01; w.H(J, J) = p.h11;
        w.T(J - 1, J) = p.t01; w.T(J, J - 1) = 0.0; w.T(J, J) = p.rz;
      }
      // (c) the next pair
      if (kjr >= 0) {
        const int J = kjr, jc = kjc;
        double a0, b0, t00, t01, t11, h00, h10, h01, h11;
        a0 = w.H(J - 1, jc);
        t00 = w.T(J - 1, J - 1);
        h00 = w.H(J - 1, J - 1);
        if (nextsame) {
          b0 = p.r; t01 = a_t01; t11 = p.t00; h10 = a_h10; h01 = a_h01; h11 = p.h00;
        } else {
          b0 = w.H(J, jc); t01 = w.T(J - 1, J); t11 = w.T(J, J);
          h10 = w.H(J, J - 1); h01 = w.H(J - 1, J); h11 = w.H(J, J);
        }
        HrPair q;
        q.jc = jc; q.jr = J;
        lartg(a0, b0, q.c, q.sn, q.r);
        const double u10 = -q.sn * t00, u11 = -q.sn * t01 + q.c * t11;
        lartg(u11, u10, q.cz, q.sz, q.rz);
        rot2(q.c, q.sn, h00, h10);
        rot2(q.c, q.sn, h01, h11);
        rot2(q.cz, q.sz, h01, h00);
        rot2(q.cz, q.sz, h11, h10);
        q.h00 = h00; q.h10 = h10; q.h01 = h01; q.h11 = h11;
        double u00 = q.c * t00, u01 = q.c * t01 + q.sn * t11;
        rot2(q.cz, q.sz, u01, u00);
        q.t00 = u00; q.t01 = u01;
        double* sl = slot + 4 * (phase & 1);
        sl[0] = q.c; sl[1] = q.sn; sl[2] = q.cz; sl[3] = q.sz;
        p = q;
      }
    }
    if (kjr >= 0) { p.jc = kjc; p.jr = kjr; x.count(2); } else { p.jc = -1; p.jr = -1; }
    x.sync();
    ++phase;
  };
  for (int jc = 0; jc < m - 2; ++jc) {
    for (int jr = m - 1; jr >= jc + 2; --jr) run_phase(jc, jr);
    run_phase(-1, -1);  // the column's last pair
  }
}

template <class X>
QZ_HD void cta_aed(X& x, WinState& w, double s, double* sr, double* si_, double* sb, int maxit, int nskip = 0,
                   bool swapfail = false, double* msscr = nullptr) {
  const bool ms = msscr != nullptr;
  int n = w.n;
  x.stamp(0);
  int info = ms ? cta_small_qz_ms(x, w, maxit, msscr) : cta_small_qz(x, w, maxit);
  x.stamp(1);
  if (info != 0) {
    // window QZ did not converge: deflate nothing, hand the diagonal
    // ratios of the (equivalent) partly reduced window over as shifts
    // (qzearly.f:237-248); the caller discards the window itself
    if (x.tid == 0) {
      for (int i = 0; i < n; ++i) { sr[i] = w.H(i, i); si_[i] = 0.0; sb[i] = w.T(i, i); }
      x.si[8] = n; x.si[9] = info; x.si[10] = 0;
    }
    x.sync();
    return;
  }
  // ---- spike test with reordering (qzearly.f:253-365) ----
  int kb = n - 1, ilst = 0;
  bool failed = false;
  int fails = 0;  // consecutive undeflatable blocks
  while (kb >= ilst) {
    // optional early stop: after nskip consecutive undeflatable blocks the
    // rest of the window is left undeflated (bounds the O(n^2) swaps)
    if (nskip > 0 && fails >= nskip) break;
    bool bulge = (kb > ilst) && (w.H(kb, kb - 1) != 0.0);
    bool dfl;
    if (!bulge) {
      double temp = fabs(s) + fabs(w.H(kb, kb));
      dfl = fabs(s * w.Q(0, kb)) <= dmax(w.tol.ulp * temp, w.tol.smlnum);
    } else {
      double h11 = w.H(kb - 1, kb - 1), h21 = w.H(kb, kb - 1), h12 = w.H(kb - 1, kb), h22 = w.H(kb, kb);
      double rtdet;
      if (h11 == 0.0 && h21 == 0.0) rtdet = 0.0;
      else if (fabs(h11) >= fabs(h21)) rtdet = sqrt(fabs(h11)) * sqrt(fabs(h22 - (h21 / h11) * h12));
      else rtdet = sqrt(fabs(h21)) * sqrt(fabs(h12 - (h11 / h21) * h22));
      double temp = fabs(s) + rtdet;
      dfl = dmax(fabs(s * w.Q(0, kb)), fabs(s * w.Q(0, kb - 1))) <= dmax(w.tol.ulp * temp, w.tol.smlnum);
    }
    int nb = bulge ? 2 : 1;
    if (dfl) {
      kb -= nb;
      fails = 0;
    } else {
      // a rejected swap ends the test: the window is re-reduced with the
      // deflations found so far (qzearly.f:321-326); swapfail forces it
      if (swapfail || !cta_move_block(x, w, kb - nb + 1, nb, ilst, false)) { failed = true; break; }
      ilst += nb;
      ++fails;
    }
  }
  (void)failed;
  // the swaps left the 2x2 blocks they touched general: standardise every
  // block of the window at once (T upper triangular again, complex pairs
  // with a positive diagonal block of T)
  cta_std_all(x, w, x.sd + 64);
  x.stamp(2);
  int m = kb + 1;  // undeflated eigenvalues at 0..m-1
  // ---- shifts: eigenvalues of the undeflated Schur blocks ----
  if (x.tid == 0) {
    int j = 0;
    while (j < m) {
      if (j + 1 < m && w.H(j + 1, j) != 0.0) {
        double c2, c1, c0;
        pencil2_poly(w.H(j, j), w.H(j + 1, j), w.H(j, j + 1), w.H(j + 1, j + 1),
                     w.T(j, j), w.T(j, j + 1), w.T(j + 1, j + 1), c2, c1, c0);
        // complex pair (or real pair if rounding says so): store as
        // lambda = (c1 +- sqrt(disc)) / (2 c2)
        double disc = c1 * c1 - 4.0 * c2 * c0;
        if (disc < 0.0) {
          sr[j] = c1; si_[j] = sqrt(-disc); sb[j] = 2.0 * c2;
          sr[j + 1] = c1; si_[j + 1] = -sqrt(-disc); sb[j + 1] = 2.0 * c2;
        } else {
          double sq = sqrt(disc);
          sr[j] = c1 + sq; si_[j] = 0.0; sb[j] = 2.0 * c2;
          sr[j + 1] = c1 - sq; si_[j + 1] = 0.0; sb[j + 1] = 2.0 * c2;
        }
        j += 2;
      } else {
        sr[j] = w.H(j, j); si_[j] = 0.0; sb[j] = w.T(j, j);
        j += 1;
      }
    }
    x.si[8] = m;
    x.si[9] = 0;
    x.si[10] = (m < n) ? 1 : 0;
  }
  x.sync();
  if (m == n || m <= 1 || s == 0.0) {
    // nothing deflated (caller discards), or nothing left to re-reduce
    x.sync();
    return;
  }
  // ---- spike reflector from Q(0, 0:m-1) (qzearly.f:371-381) ----
  double* v = x.sd + 64;  // length m (<= n); caller guarantees room
  if (x.tid == 0) {
    double alpha = w.Q(0, 0);
    double mx = 0.0;
    for (int i = 1; i < m; ++i) mx = dmax(mx, fabs(w.Q(0, i)));
    double tau = 0.0;
    v[0] = 1.0;
    if (mx > 0.0) {
      double ma = dmax(mx, fabs(alpha));
      double nrm = 0.0;
      nrm += (alpha / ma) * (alpha / ma);
      for (int i = 1; i < m; ++i) { double t = w.Q(0, i) / ma; nrm += t * t; }
      nrm = sqrt(nrm) * ma;
      double beta = -dsign(nrm, alpha);
      tau = (beta - alpha) / beta;
      double sc = 1.0 / (alpha - beta);
      for (int i = 1; i < m; ++i) v[i] = w.Q(0, i) * sc;
    } else {
      for (int i = 1; i < m; ++i) v[i] = 0.0;
    }
    x.sd[63] = tau;
  }
  x.sync();
  double tau = x.sd[63];
  if (tau != 0.0) {
    // H(0:m, :) <- P H ; T(0:m, m:n) <- P T ; Q(:, 0:m) <- Q P
    for (int j = x.tid; j < n; j += x.nt) {
      double t = 0.0;
      for (int i = 0; i < m; ++i) t += v[i] * w.H(i, j);
      t *= tau;
      for (int i = 0; i < m; ++i) w.H(i, j) -= t * v[i];
      if (j >= m) {
        double u = 0.0;
        for (int i = 0; i < m; ++i) u += v[i] * w.T(i, j);
        u *= tau;
        for (int i = 0; i < m; ++i) w.T(i, j) -= u * v[i];
      }
    }
    if (w.wantq)
      for (int r = x.tid; r < n; r += x.nt) {
        double t = 0.0;
        for (int i = 0; i < m; ++i) t += w.Q(r, i) * v[i];
        t *= tau;
        for (int i = 0; i < m; ++i) w.Q(r, i) -= t * v[i];
      }
    // RQ update of the leading m x m block of T:  T' = T + v*wv^T with
    // wv = -tau T^T v  (qzearly.f:396-446)
    double* wv = x.sd + 64 + n;  // length m
    for (int j = x.tid; j < m; j += x.nt) {
      double t = 0.0;
      for (int i = 0; i <= j; ++i) t += w.T(i, j) * v[i];
      wv[j] = -tau * t;
    }
    x.sync();
    // pass 1 rotations (depend on wv only): zero wv(i) into wv(i+1)
    double* rc = x.sd + 64 + 2 * n;      // length m
    double* rs = x.sd + 64 + 3 * n;      // length m
    if (x.tid == 0) {
      double wl = wv[0];
      for (int i = 0; i < m - 1; ++i) {
        double c, sn, r;
        lartg(wv[i + 1], wl, c, sn, r);
        // column op on (col i, col i+1): col_i' = c col_i - sn col_{i+1}
        //                                col_{i+1}' = sn col_i + c col_{i+1}
        rc[i] = c; rs[i] = sn;
        wl = r;
      }
      x.sd[62] = wl;  // final wv(m-1)
    }
    x.sync();
    // apply pass 1 row by row to T (rows 0..m-1), H (rows 0..m-1), Z (all rows)
    for (int r = x.tid; r < n; r += x.nt) {
      if (r < m) {
        for (int i = (r > 0 ? r - 1 : 0); i < m - 1; ++i) {
          double a = w.T(r, i), b = w.T(r, i + 1);
          w.T(r, i) = rc[i] * a - rs[i] * b;
          w.T(r, i + 1) = rs[i] * a + rc[i] * b;
        }
        for (int i = 0; i < m - 1; ++i) {
          double a = w.H(r, i), b = w.H(r, i + 1);
          w.H(r, i) = rc[i] * a - rs[i] * b;
          w.H(r, i + 1) = rs[i] * a + rc[i] * b;
        }
      }
      if (w.wantz)
        for (int i = 0; i < m - 1; ++i) {
          double a = w.Z(r, i), b = w.Z(r, i + 1);
          w.Z(r, i) = rc[i] * a - rs[i] * b;
          w.Z(r, i + 1) = rs[i] * a + rc[i] * b;
        }
    }
    x.sync();
    double wl = x.sd[62];
    for (int i = x.tid; i < m; i += x.nt) w.T(i, m - 1) += wl * v[i];
    x.sync();
    // pass 2: zero the subdiagonal of T from the bottom
    for (int i = m - 2; i >= 0; --i) {
      double c, sn, r;
      lartg(w.T(i + 1, i + 1), w.T(i + 1, i), c, sn, r);
      x.sync();
      for (int rr = x.tid; rr <= i; rr += x.nt) {
        double a = w.T(rr, i), b = w.T(rr, i + 1);
        w.T(rr, i) = c * a - sn * b;
        w.T(rr, i + 1) = sn * a + c * b;
      }
      if (x.tid == 0) { w.T(i + 1, i + 1) = r; w.T(i + 1, i) = 0.0; rc[i] = c; rs[i] = sn; }
      x.sync();
    }
    for (int r = x.tid; r < n; r += x.nt) {
      if (r < m)
        for (int i = m - 2; i >= 0; --i) {
          double a = w.H(r, i), b = w.H(r, i + 1);
          w.H(r, i) = rc[i] * a - rs[i] * b;
          w.H(r, i + 1) = rs[i] * a + rc[i] * b;
        }
      if (w.wantz)
        for (int i = m - 2; i >= 0; --i) {
          double a = w.Z(r, i), b = w.Z(r, i + 1);
          w.Z(r, i) = rc[i] * a - rs[i] * b;
          w.Z(r, i + 1) = rs[i] * a + rc[i] * b;
        }
    }
    x.sync();
  }
  x.stamp(3);
  cta_hessred(x, w, m);
  x.stamp(4);
}

}  // namespace qz
