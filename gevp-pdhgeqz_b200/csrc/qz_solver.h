// Host-side control of the multishift QZ iteration.
//
// Mirrors the iteration of PDHGEQZ1 / PDHGEQZ0 on a 1x1 grid
// (src/pdhgeqz/PDHGEQZ1.f:466-763, PDHGEQZ0.f:505-1202): deflation scan
// (PDLASMSUB), infinite-eigenvalue deflation (PDHGEQZ7), aggressive early
// deflation (PDHGEQZ2/3 + QZEARLY), the nibble gate, shift selection and
// the multishift sweep (PDHGEQZ5 -> PDHGEQZA/B -> DHGEQZ5 -> PDHGEQZ6).
// The numerical work is done by the backend (device kernels); this file
// only decides what runs next from a handful of integers read back from the
// device.  The control code holds no global state (reentrant).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "qz_window.cuh"

namespace qz {

// Tunables (defaults follow the reference's PIPARMQ table where the GPU
// window limits allow; see piparmq.f:438-535).
struct SolveParams {
  int nw_max = 48;       // AED window (one CTA, shared memory; up to 80)
  int w_chase = 80;      // chase window
  int nmin = 80;         // active blocks this small are solved by one CTA
  int nibble = -1;       // -1: table (14 in PDHGEQZ1 regime, 335*nh^-0.44 above)
  int ns_max = -1;       // -1: table
  int maxit_factor = 30; // MAXIT = 30*NH
  int chain_max = -1;    // bulges per chain, -1: from w_chase
  int verbose = 0;       // progress lines on stderr (B200QZ_VERBOSE=1)
  int aed_nskip = -1;    // AED spike test stops after this many consecutive
                         // undeflatable blocks (0: test the whole window;
                         // -1: whole window for n >= 6000, else 4)
  int max_wave = 8;      // chains chased concurrently (one CTA each)
  int stall_limit = 300; // iterations without deflation before giving up
  int aed_threads = 128; // threads of the AED / endgame window kernel (32: one warp)
  int split = 0;         // 7 or 8: off-diagonal updates through that many INT8
                         // Ozaki slices on the tensor cores (windows up to 80)
  int upd_persist = 1;   // 1: persistent, prefetching DMMA update kernels
  int aed_limit = -1;    // >= 0: stop before the AED after this many AEDs
                         // (tuning traces; the solve then returns -2)
  int aed_ms = 0;        // window QZ of the AED kernel: 1 small-bulge multishift
                         // (lockstep chains), 0 double shift
  int aed_swap_fail = 0; // 1: every block swap inside the AED reports failure
                         // (exercises the swap-failure branch, qzearly.f:321-326)
};

struct SolveStats {
  int64_t iters = 0, aeds = 0, aed_defl = 0, sweeps = 0, chains = 0, windows = 0;
  int64_t endgames = 0, infs = 0, shifts = 0;
  double upd_flops = 0.0;  // FP64-equivalent flops of the off-diagonal updates
  double win_bytes = 0.0;  // algorithmic bytes of window kernels (load+store)
  int64_t launches = 0;    // kernel launches issued by the solve
  int64_t aed_fail = 0;    // AED windows whose small QZ did not converge
  int64_t exceptional = 0; // sweeps with exceptional shifts
  int64_t remaining = 0;   // rows of the active part left at exit (0: converged)
  int stop_ktop = -1, stop_kbot = -1;  // active block where an AED limit stopped the solve
  double last_frac = 0.0;  // deflated fraction of the last AED window
  int64_t policy_calls = 0;  // AED decisions taken by the learned policy
  // algorithmic bytes and launches per window kernel (roofline accounting):
  // a window of order w moves 6*8*w^2 bytes (H, T in; H, T, and both
  // factors out)
  double aed_bytes = 0.0, chase_bytes = 0.0;
  int64_t aed_launches = 0, chase_launches = 0;
};

// reference shift-count table (piparmq.f:504-533)
inline int ns_table(int nh) {
  int ns = 2;
  if (nh >= 30) ns = 4;
  if (nh >= 60) ns = 10;
  if (nh >= 150) ns = std::max(10, (int)(nh / std::lround(std::log((double)nh) / std::log(2.0))));
  if (nh >= 590) ns = 64;
  if (nh >= 3000) ns = 128;
  if (nh >= 6000) ns = 256;
  if (nh >= 12000) ns = 512;
  return std::max(2, ns - ns % 2);
}
inline int nibble_table(int nh) {
  if (nh <= 6000) return 14;  // PDHGEQZ1 regime (piparmq.f:495-496)
  return std::min(100, (int)std::ceil(335.0 * std::pow((double)nh, -0.44)));
}

// Power of two applied to T before the iteration when T's magnitude is far
// from H's (more than 2^30 apart), so that shift polynomials, whose
// coefficients grow like the square of the eigenvalues' magnitude, stay in
// the floating-point range; undone on T (and hence beta) at the end.  The
// scaling is exact and commutes with the orthogonal transformations.
// Arguments are the largest absolute entries of the two active blocks.
inline int balance_exponent(double hmax, double tmax) {
  if (!(hmax > 0.0) || !(tmax > 0.0) || !std::isfinite(hmax) || !std::isfinite(tmax)) return 0;
  const double l2 = std::log2(hmax) - std::log2(tmax);
  if (std::fabs(l2) <= 30.0) return 0;
  return (int)std::lround(l2);
}

struct ShiftPair { double c2, c1, c0; };

// Pair the shifts (alphar, alphai, beta) into real quadratics: complex
// conjugates pair with each other, real shifts pair in order (the role of
// the shuffle at PDHGEQZ1.f:608-629 / PDHGEQZ0.f:1111-1126).
inline void pair_shifts(const double* sr, const double* si, const double* sb, int m, int ns,
                        std::vector<ShiftPair>& out) {
  out.clear();
  // use the shifts closest to the bottom of the undeflated part
  std::vector<int> reals;
  std::vector<std::pair<int, int>> cplx;
  for (int j = m - 1; j >= 0; --j) {
    if (si[j] != 0.0 && j > 0 && si[j - 1] == -si[j]) {
      cplx.push_back({j - 1, j});
      --j;
    } else if (si[j] == 0.0) {
      reals.push_back(j);
    }
  }
  size_t ir = 0, ic = 0;
  while ((int)out.size() * 2 < ns) {
    // alternate by position: take whichever unused candidate is lower
    int next_r = (ir + 1 < reals.size()) ? reals[ir] : -1;
    int next_c = (ic < cplx.size()) ? cplx[ic].second : -1;
    if (next_r < 0 && next_c < 0) break;
    ShiftPair p;
    if (next_c >= next_r) {
      int a = cplx[ic].first;
      double b = sb[a];
      // lambda = (sr + i si)/b: c2 = b^2, c1 = 2 sr b, c0 = sr^2 + si^2
      p.c2 = b * b; p.c1 = 2.0 * sr[a] * b; p.c0 = sr[a] * sr[a] + si[a] * si[a];
      ++ic;
    } else {
      int a = reals[ir], b = reals[ir + 1];
      p.c2 = sb[a] * sb[b]; p.c1 = sr[a] * sb[b] + sr[b] * sb[a]; p.c0 = sr[a] * sr[b];
      ir += 2;
    }
    double mx = std::max(std::fabs(p.c2), std::max(std::fabs(p.c1), std::fabs(p.c0)));
    if (!(mx > 0.0) || !std::isfinite(mx)) continue;
    p.c2 /= mx; p.c1 /= mx; p.c0 /= mx;
    out.push_back(p);
  }
}

// One chase window of one chain.
struct WinPlan {
  int w, wk, last, tmax, nb;
  std::vector<Bulge> bl;
};
struct ChainPlan {
  std::vector<WinPlan> wins;
};

// Window sequence of one chain of nb bulges over the active block
// [ktop, kbot] (the PDHGEQZ5 schedule with windows of size W): the first
// window introduces the bulges at ktop, the following ones start one row
// above the topmost bulge, the last one pushes every bulge off at kbot.
// Every window advances the chain by exactly adv rows (adv must not exceed
// W - 4 - 3*(nb-1), the most a chain of nb bulges can move), so chains of
// different lengths launched with the same lag never catch up.
inline void plan_chain(int ktop, int kbot, int W, int nb, const ShiftPair* sp, int adv, ChainPlan& cp) {
  std::vector<int> pos(nb);
  bool first = true;
  while (true) {
    WinPlan wp;
    wp.w = first ? ktop : pos[nb - 1] - 1;
    wp.wk = std::min(W, kbot - wp.w + 1);
    bool fin = (wp.w + wp.wk - 1 >= kbot);
    wp.last = fin ? (kbot - wp.w) : (wp.wk - 1);
    wp.nb = nb;
    wp.bl.resize(nb);
    wp.tmax = 0;
    for (int k = 0; k < nb; ++k) {
      Bulge& g = wp.bl[k];
      g.c2 = sp[k].c2; g.c1 = sp[k].c1; g.c0 = sp[k].c0;
      if (first) {
        g.base = -3 * k;
        g.tlo = 3 * k;
        g.intro = 1;
      } else {
        g.base = pos[k] - wp.w;
        g.tlo = 0;
        g.intro = 0;
      }
      if (fin) {
        // push-off: each bulge ends with its 2x2 step at row kbot-1
        g.thi = (kbot - wp.w) - g.base;
      } else {
        // lockstep: every bulge moves adv rows; in the first window bulge
        // k starts at step 3k, so the topmost one also advances adv
        g.thi = first ? (adv + 3 * nb - 2) : adv;
      }
      wp.tmax = std::max(wp.tmax, g.thi);
    }
    for (int k = 0; k < nb; ++k) pos[k] = wp.w + wp.bl[k].base + wp.bl[k].thi;
    cp.wins.push_back(std::move(wp));
    if (fin) break;
    first = false;
  }
}

// Backend interface (implemented by the GPU backend):
//   void scan(int ifirst, int kbot, int* out5)          // ktop, ninf, jmax, jmin, nonfinite
//   void aed(int ktop, int kwtop, int kbot, int* info3, double* shifts) // m, status, transformed
//   void update(int w, int wk, int which)               // which 0: AED factors, 1: zero-chase U,V
//   void chase_wave(const WinPlan* const* wins, int n)  // one CTA per window
//   void update_wave(const WinPlan* const* wins, int n) // far updates of those windows
//   void inf_window(int w, int wk, int top, int jz, int stop, bool deflate)
//   void inf_top(int ktop)
//   bool policy(int ktop, int kbot, double lastfrac, int* nw, int* ns)
//                                                       // learned (nw, ns); false: use the table
//   void active(int ktop, int kbot)                     // the active block of the next steps
//                                                       // (bounds the far updates when only
//                                                       // eigenvalues are wanted)
template <class BK>
int qz_iterate(BK& bk, int n, int ilo, int ihi, const SolveParams& P, SolveStats& S) {
  int ifirst = ilo, kbot = ihi;
  int nh0 = ihi - ilo + 1;
  int64_t maxit = (int64_t)P.maxit_factor * std::max(1, nh0);
  std::vector<double> sh(3 * std::max(P.nw_max, P.nmin) + 8);
  std::vector<ShiftPair> pairs;
  std::vector<const WinPlan*> wave;
  int scan_out[5];
  int info3[3];
  int stall = 0;             // iterations since the last deflation
  int last_kbot = kbot, last_ktop = -1;
  auto done = [&](int r) {
    S.remaining = (kbot >= ifirst) ? kbot - ifirst + 1 : 0;
    return r;
  };
  for (int64_t it = 0; it < maxit; ++it) {
    if (kbot < ifirst) return done(0);
    ++S.iters;
    bk.scan(ifirst, kbot, scan_out);
    int ktop = scan_out[0];
    int ninf = scan_out[1];
    if (scan_out[4]) return done(-1);  // non-finite entry in the active block
    if (kbot != last_kbot || ktop != last_ktop) stall = 0; else ++stall;
    last_kbot = kbot;
    last_ktop = ktop;
    if (stall > P.stall_limit) return done(kbot + 1);
    if (P.verbose)
      std::fprintf(stderr, "[b200qz] it=%lld ktop=%d kbot=%d ninf=%d\n", (long long)it, ktop, kbot, ninf);
    bk.active(ktop, kbot);
    if (ktop == kbot) {
      // a 1x1 block has converged (finite or infinite eigenvalue)
      kbot -= 1;
      continue;
    }
    if (ninf > 0) {
      ++S.infs;
      int jz = scan_out[2];  // lowest zero
      if (jz == ktop && ktop < kbot) {
        bk.inf_top(ktop);
        continue;
      }
      // chase down to kbot in windows of w_chase, then deflate
      int W = P.w_chase;
      while (true) {
        int w = std::max(ktop, jz - 1);
        int wk = std::min(W, kbot - w + 1);
        int stop = std::min(w + wk - 1, kbot);
        bool defl = (stop == kbot);
        int top = (ktop >= w) ? ktop - w : -1;
        bk.inf_window(w, wk, top, jz - w, stop - w, defl);
        bk.update(w, wk, 1);
        ++S.windows;
        if (defl) break;
        jz = stop;
      }
      kbot -= 1;
      continue;
    }
    int nh = kbot - ktop + 1;
    if (nh <= P.nmin) {
      // small block: one CTA solves it (PDHGEQZ4 -> KKQZ role)
      ++S.endgames;
      bk.aed(ktop, ktop, kbot, info3, sh.data());
      if (info3[1] != 0) return done(kbot + 1);
      bk.update(ktop, nh, 0);
      kbot = ktop - 1;
      continue;
    }
    // ---- aggressive early deflation ----
    if (P.aed_limit >= 0 && S.aeds >= P.aed_limit) {
      S.stop_ktop = ktop;
      S.stop_kbot = kbot;
      return done(-2);
    }
    int nw = std::min(P.nw_max, nh);
    int ns_pol = -1;
    {
      int pnw = 0, pns = 0;
      if (bk.policy(ktop, kbot, S.last_frac, &pnw, &pns)) {
        // the network's window, up to the window kernel's limit (which the
        // decoded output already respects) rather than the table's nw_max
        nw = std::max(std::min(4, nh), std::min(pnw, nh));
        ns_pol = pns;
        ++S.policy_calls;
      }
    }
    int kwtop = kbot - nw + 1;
    ++S.aeds;
    bk.aed(ktop, kwtop, kbot, info3, sh.data());
    if (P.verbose)
      std::fprintf(stderr, "[b200qz]   aed kwtop=%d nw=%d m=%d status=%d tr=%d\n", kwtop, nw, info3[0], info3[1], info3[2]);
    int m = info3[0];
    int nd = 0;
    if (info3[1] == 0 && info3[2] != 0) {
      nd = nw - m;
      bk.update(kwtop, nw, 0);
    }
    // a failed window QZ deflates nothing but still supplies shifts (the
    // diagonal ratios of the window), so the sweep changes the pencil and
    // the next AED sees a different window (PDHGEQZ0.f:944-949)
    if (info3[1] != 0) ++S.aed_fail;
    S.aed_defl += nd;
    S.last_frac = (double)nd / (double)nw;
    kbot -= nd;
    if (kbot < ktop) continue;
    int nib = (P.nibble >= 0) ? P.nibble : nibble_table(nh);
    if (info3[1] == 0 && 100 * nd > nib * nw) continue;
    // ---- multishift sweep ----
    int nsmax = (P.ns_max > 0) ? P.ns_max : ns_table(nh);
    if (ns_pol > 0) nsmax = ns_pol;
    int ns = std::min(nsmax, m - (m % 2));
    if (ns < 2) continue;
    pair_shifts(sh.data(), sh.data() + m, sh.data() + 2 * m, m, ns, pairs);
    if (stall > 0 && stall % 40 == 0) {
      // no deflation for a while: exceptional shifts (scaled pseudo-random
      // real pairs spread over the spectrum's magnitude) break the cycle
      double mag = 0.0;
      for (int i = 0; i < m; ++i)
        if (sh[2 * m + i] != 0.0) mag = std::max(mag, std::fabs(sh[i] / sh[2 * m + i]));
      if (!(mag > 0.0) || !std::isfinite(mag)) mag = 1.0;
      for (size_t k = 0; k < pairs.size(); ++k) {
        double a = mag * std::sin(1.0 + 2.0 * k + 0.37 * stall), b = mag * std::cos(0.5 + 3.0 * k);
        pairs[k].c2 = 1.0; pairs[k].c1 = a + b; pairs[k].c0 = a * b;
        double mx = std::max(1.0, std::max(std::fabs(pairs[k].c1), std::fabs(pairs[k].c0)));
        pairs[k].c2 /= mx; pairs[k].c1 /= mx; pairs[k].c0 /= mx;
      }
      ++S.exceptional;
    }
    int npairs = (int)pairs.size();
    if (npairs == 0) continue;
    int nh2 = kbot - ktop + 1;
    if (nh2 < 3) continue;
    ++S.sweeps;
    S.shifts += 2 * npairs;
    int W = P.w_chase;
    int cmax = (P.chain_max > 0) ? P.chain_max : std::max(1, (W - 4) / 6);
    cmax = std::min(cmax, std::max(1, (W - 4) / 3 - 1));
    // ---- plan every chain's windows (positions do not depend on data) ----
    int nbig = std::min(cmax, npairs);
    int adv = W - 4 - 3 * (nbig - 1);  // common advance per window
    std::vector<ChainPlan> plans;
    for (int p0 = 0; p0 < npairs; p0 += cmax) {
      ChainPlan cp;
      int nb = std::min(cmax, npairs - p0);
      plan_chain(ktop, kbot, W, nb, pairs.data() + p0, adv, cp);
      plans.push_back(std::move(cp));
      ++S.chains;
    }
    // ---- waves: chain c trails chain c-1 by lag windows with
    // lag*adv >= W, so the windows of one wave are disjoint; the far
    // updates of a wave run as one left batch then one right batch, and
    // a left update of one window only meets a right update of another
    // (commuting transformations, never in the same launch) ----
    const int lag = (W + adv - 1) / adv;
    const int G = std::max(1, std::min(P.max_wave, (int)plans.size()));
    for (size_t g0 = 0; g0 < plans.size(); g0 += G) {
      size_t g1 = std::min(plans.size(), g0 + G);
      int tmax_wave = 0;
      for (size_t c = g0; c < g1; ++c)
        tmax_wave = std::max(tmax_wave, (int)(lag * (c - g0)) + (int)plans[c].wins.size());
      for (int t = 0; t < tmax_wave; ++t) {
        wave.clear();
        for (size_t c = g0; c < g1; ++c) {
          int i = t - lag * (int)(c - g0);
          if (i < 0 || i >= (int)plans[c].wins.size()) continue;
          wave.push_back(&plans[c].wins[i]);
        }
        if (wave.empty()) continue;
        bk.chase_wave(wave.data(), (int)wave.size());
        bk.update_wave(wave.data(), (int)wave.size());
        S.windows += (int64_t)wave.size();
      }
    }
  }
  return done(kbot + 1);
}

}  // namespace qz
