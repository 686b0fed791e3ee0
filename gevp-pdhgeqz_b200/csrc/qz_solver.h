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

#include "qz_chase.cuh"

namespace qz {

// Tunables (defaults follow the reference's PIPARMQ table where the GPU
// window limits allow; see piparmq.f:438-535).
struct SolveParams {
  int nw_max = 80;       // AED window (one CTA, shared memory)
  int w_chase = 80;      // chase window
  int nmin = 80;         // active blocks this small are solved by one CTA
  int nibble = -1;       // -1: table (14 in PDHGEQZ1 regime, 335*nh^-0.44 above)
  int ns_max = -1;       // -1: table
  int maxit_factor = 30; // MAXIT = 30*NH
  int chain_max = -1;    // bulges per chain, -1: from w_chase
  int verbose = 0;       // progress lines on stderr (B200QZ_VERBOSE=1)
  int aed_nskip = 0;     // AED spike test stops after this many consecutive
                         // undeflatable blocks (0: test the whole window)
};

struct SolveStats {
  int64_t iters = 0, aeds = 0, aed_defl = 0, sweeps = 0, chains = 0, windows = 0;
  int64_t endgames = 0, infs = 0, shifts = 0;
  double upd_flops = 0.0;  // FP64-equivalent flops of the off-diagonal updates
  double win_bytes = 0.0;  // algorithmic bytes of window kernels (load+store)
  int64_t launches = 0;    // kernel launches issued by the solve
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

// Backend interface (implemented by the GPU backend):
//   void scan(int ifirst, int kbot, int* out4)          // ktop, ninf, jmax, jmin
//   void aed(int ktop, int kwtop, int kbot, int* info3, double* shifts) // m, status, transformed
//   void update(int w, int wk, int which)               // which 0: AED factors, 1: chase U,V
//   void chase(int w, int wk, int last, const Bulge* bl, int nb, int tmax)
//   void inf_window(int w, int wk, int top, int jz, int stop, bool deflate)
//   void inf_top(int ktop)
template <class BK>
int qz_iterate(BK& bk, int n, int ilo, int ihi, const SolveParams& P, SolveStats& S) {
  int ifirst = ilo, kbot = ihi;
  int nh0 = ihi - ilo + 1;
  int64_t maxit = (int64_t)P.maxit_factor * std::max(1, nh0);
  std::vector<double> sh(3 * std::max(P.nw_max, P.nmin) + 8);
  std::vector<ShiftPair> pairs;
  std::vector<Bulge> bl;
  int scan_out[4];
  int info3[3];
  for (int64_t it = 0; it < maxit; ++it) {
    if (kbot < ifirst) return 0;
    ++S.iters;
    bk.scan(ifirst, kbot, scan_out);
    int ktop = scan_out[0];
    int ninf = scan_out[1];
    if (P.verbose)
      std::fprintf(stderr, "[b200qz] it=%lld ktop=%d kbot=%d ninf=%d\n", (long long)it, ktop, kbot, ninf);
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
      if (info3[1] != 0) return kbot + 1;
      bk.update(ktop, nh, 0);
      kbot = ktop - 1;
      continue;
    }
    // ---- aggressive early deflation ----
    int nw = std::min(P.nw_max, nh);
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
    if (info3[1] != 0) m = 0;  // failed window QZ: no deflation, no shifts
    S.aed_defl += nd;
    kbot -= nd;
    if (kbot < ktop) continue;
    int nib = (P.nibble >= 0) ? P.nibble : nibble_table(nh);
    if (100 * nd > nib * nw) continue;
    // ---- multishift sweep ----
    int nsmax = (P.ns_max > 0) ? P.ns_max : ns_table(nh);
    int ns = std::min(nsmax, m - (m % 2));
    if (ns < 2) continue;
    pair_shifts(sh.data(), sh.data() + m, sh.data() + 2 * m, m, ns, pairs);
    int npairs = (int)pairs.size();
    if (npairs == 0) continue;
    int nh2 = kbot - ktop + 1;
    if (nh2 < 3) continue;
    ++S.sweeps;
    S.shifts += 2 * npairs;
    int W = P.w_chase;
    int cmax = (P.chain_max > 0) ? P.chain_max : std::max(1, (W - 4) / 6);
    for (int p0 = 0; p0 < npairs; p0 += cmax) {
      int nb = std::min(cmax, npairs - p0);
      ++S.chains;
      // next-step positions (global) of each bulge; bulge 0 is the deepest
      std::vector<int> pos(nb);
      bool first = true;
      while (true) {
        int w, wk;
        if (first) {
          w = ktop;
        } else {
          w = pos[nb - 1] - 1;
        }
        wk = std::min(W, kbot - w + 1);
        bool fin = (w + wk - 1 >= kbot);
        int last = fin ? (kbot - w) : (wk - 1);
        bl.resize(nb);
        int tmax = 0;
        for (int k = 0; k < nb; ++k) {
          Bulge& g = bl[k];
          const ShiftPair& sp = pairs[p0 + k];
          g.c2 = sp.c2; g.c1 = sp.c1; g.c0 = sp.c0;
          if (first) {
            g.base = -3 * k;
            g.tlo = 3 * k;
            g.intro = 1;
          } else {
            g.base = pos[k] - w;
            g.tlo = 0;
            g.intro = 0;
          }
          if (fin) {
            // push-off: each bulge ends with its 2x2 step at row kbot-1
            g.thi = (kbot - w) - g.base;
          } else {
            // lockstep: every bulge moves as far as the deepest one can
            // (its last 3x3 step at window row wk-4)
            g.thi = first ? (wk - 3) : (wk - 3 - (pos[0] - w));
          }
          tmax = std::max(tmax, g.thi);
        }
        bk.chase(w, wk, last, bl.data(), nb, tmax);
        bk.update(w, wk, 1);
        ++S.windows;
        if (fin) break;
        for (int k = 0; k < nb; ++k) pos[k] = w + bl[k].base + bl[k].thi;
        first = false;
      }
    }
  }
  return kbot + 1;
}

}  // namespace qz
