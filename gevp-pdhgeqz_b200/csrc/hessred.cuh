// Hessenberg-triangular reduction of a pencil (A, B) with B upper
// triangular, by Givens rotations: the semantics of LAPACK DGGHRD, in the
// role of the reference's PDGGHRD (src/ab2ht/PDGGHRD.f:13, called by the
// examples after a QR factorisation of B, examples/EXRAND2.f:296-336).
//
// The rotations are LAPACK's: for column jc = ilo..ihi-2 and pair
// J = ihi..jc+2 (0-based), the row rotation G on rows (J-1, J) zeros
// A(J, jc) (lartg(A(J-1, jc), A(J, jc))), and the column rotation Z on
// columns (J, J-1) zeros the entry B(J, J-1) that G created
// (lartg(B(J, J), B(J, J-1))).  G acts on A(.., jc+1:n) and B(.., J-1:n),
// Z on A(0:ihi, ..) and B(0:J-1, ..); Q accumulates G and Z accumulates Z.
//
// Device form.  The pairs of one column form a dependent chain through the
// 2x2 diagonal blocks of B; everything else is a rotation applied to a row
// or a column "walk".  A column's chain runs in windows of at most W pairs
// from the bottom up.  One CTA holds the window's diagonal block of B in
// shared memory with the column's entries of A: one thread computes the
// row rotations from the column of A (hr_g_chain, which does not depend on
// B) ahead of the others, which run the column rotations through the block
// (cta_hr_zchain: one barrier per pair, the block thread one pair ahead of
// the threads applying the previous pair inside the block).  The rest of a
// window's rotations is applied by the launch of the next window (or by the
// column's last launch) as walks:
//   (a) its Z on the rows of B the next window's block holds (CTA 0),
//   (e) its Z on the rows of B above those,
//   (f) its G on the columns of B right of the window,
//   (g) its Z on rows 0..ihi of A;
// after the column, its G on the columns of A right of jc and both factors
// on Q and Z.  Every entry sees the rotations in LAPACK's order: the right
// and left transformations commute, and the walks of one window come after
// those of the window before on every entry they share.
#pragma once
#include "qz_prims.cuh"

namespace qz {

// Rotation record of pair J: rot[4J .. 4J+3] = (c, s, cz, sz).

// Z rotations of pairs Jhi, Jhi-1, .., Jlo on one row (element j at
// row[j * st]): columns (J, J-1), x = column J.
QZ_HD void hr_walk_z(double* __restrict__ row, int64_t st, int Jhi, int Jlo, const double* __restrict__ rot) {
  constexpr int kChunk = 8;
  double x = row[Jhi * st];
  int J = Jhi;
  while (J >= Jlo) {
    const int k = (J - Jlo + 1) < kChunk ? (J - Jlo + 1) : kChunk;
    double y[kChunk], cz[kChunk], sz[kChunk];
#pragma unroll
    for (int i = 0; i < kChunk; ++i)
      if (i < k) {
        y[i] = row[(int64_t)(J - 1 - i) * st];
        cz[i] = rot[4 * (J - i) + 2];
        sz[i] = rot[4 * (J - i) + 3];
      }
#pragma unroll
    for (int i = 0; i < kChunk; ++i)
      if (i < k) {
        const double xn = cz[i] * x + sz[i] * y[i];
        x = -sz[i] * x + cz[i] * y[i];
        row[(int64_t)(J - i) * st] = xn;
      }
    J -= k;
  }
  row[(int64_t)(Jlo - 1) * st] = x;
}

// G rotations of pairs Jhi, .., Jlo along one line (element i at
// v[i * st]): entries (J-1, J), x = entry J-1.  A column of A or B, a
// column of the transposed Q, or a row of Q (Q <- Q G^T).
QZ_HD void hr_walk_g(double* __restrict__ v, int64_t st, int Jhi, int Jlo, const double* __restrict__ rot) {
  constexpr int kChunk = 8;
  double y = v[Jhi * st];
  int J = Jhi;
  while (J >= Jlo) {
    const int k = (J - Jlo + 1) < kChunk ? (J - Jlo + 1) : kChunk;
    double x[kChunk], c[kChunk], s[kChunk];
#pragma unroll
    for (int i = 0; i < kChunk; ++i)
      if (i < k) {
        x[i] = v[(int64_t)(J - 1 - i) * st];
        c[i] = rot[4 * (J - i)];
        s[i] = rot[4 * (J - i) + 1];
      }
#pragma unroll
    for (int i = 0; i < kChunk; ++i)
      if (i < k) {
        const double yn = -s[i] * x[i] + c[i] * y;
        y = c[i] * x[i] + s[i] * y;
        v[(int64_t)(J - i) * st] = yn;
      }
    J -= k;
  }
  v[(int64_t)(Jlo - 1) * st] = y;
}

// Leading dimension of the window block in shared memory (odd, so that a
// row of the block spreads over the banks).
QZ_HD int hr_ldw(int m) { return (m & 1) ? m : m + 1; }

QZ_HD double hr_rsqrt(double q) {
#ifdef __CUDA_ARCH__
  return rsqrt(q);
#else
  return 1.0 / sqrt(q);
#endif
}

// Givens rotation with lartg's convention (c*f + s*g = r, -s*f + c*g = 0,
// c >= 0, r with the sign of f), one reciprocal square root in the range
// where the squares neither overflow nor underflow (the chain's latency is
// two of these per pair).
QZ_HD void hr_lartg(double f, double g, double& c, double& s, double& r) {
  const double af = fabs(f), ag = fabs(g), mx = af > ag ? af : ag;
  if (mx > kSafeLo && mx < kSafeHi) {
    // in range: selects instead of branches for the exact cases g = 0
    // (identity) and f = 0 (a swap), as LAPACK returns them
    const double q = f * f + g * g, inv = hr_rsqrt(q);
    const double sg = f < 0.0 ? -1.0 : 1.0;
    const bool g0 = g == 0.0, f0 = f == 0.0;
    c = g0 ? 1.0 : (f0 ? 0.0 : af * inv);
    s = g0 ? 0.0 : (f0 ? (g > 0.0 ? 1.0 : -1.0) : sg * g * inv);
    r = g0 ? f : (f0 ? ag : sg * (q * inv));
  } else if (mx == 0.0) {
    c = 1.0; s = 0.0; r = f;
  } else {
    const double fs = f / mx, gs = g / mx, q = fs * fs + gs * gs, inv = hr_rsqrt(q);
    if (g == 0.0) {
      c = 1.0; s = 0.0; r = f;
    } else if (f == 0.0) {
      c = 0.0; s = (g > 0.0) ? 1.0 : -1.0; r = ag;
    } else {
      const double sg = f < 0.0 ? -1.0 : 1.0;
      c = fabs(fs) * inv;
      s = sg * gs * inv;
      r = sg * (q * inv * mx);
    }
  }
}

QZ_HD int hr_ld_acq(const int* p) {
#ifdef __CUDA_ARCH__
  int v;
  asm volatile("ld.acquire.cta.shared.b32 %0, [%1];" : "=r"(v) : "r"((unsigned)__cvta_generic_to_shared(p)) : "memory");
  return v;
#else
  return *(const volatile int*)p;
#endif
}
QZ_HD void hr_st_rel(int* p, int v) {
#ifdef __CUDA_ARCH__
  asm volatile("st.release.cta.shared.b32 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(p)), "r"(v) : "memory");
#else
  *(volatile int*)p = v;
#endif
}

// Shared memory of a window CTA for windows of up to wmax pairs: the block
// (m x hr_ldw(m), m <= wmax+1), the column entries of A, the rotations by
// pair (c, s, cz, sz; copied to the global record after the chain, so
// that no global store is in flight at the chain's barriers), the far
// threads' rotation slots and the producer's count.
struct HrSmem {
  double* Tw;
  double* acol;
  double* gbuf;
  double* slot;
  int* gready;
};
QZ_HD size_t hr_smem_doubles(int wmax) {
  const int m = wmax + 1;
  return (size_t)m * hr_ldw(m) + 5 * (size_t)m + 8 + 2;
}
QZ_HD HrSmem hr_layout(double* sm, int wmax) {
  const int m = wmax + 1;
  HrSmem L;
  L.Tw = sm;
  L.acol = sm + (size_t)m * hr_ldw(m);
  L.gbuf = L.acol + m;
  L.slot = L.gbuf + 4 * m;
  L.gready = (int*)(L.slot + 8);
  return L;
}

// The row rotations of one window (the producer): pairs J = m-1 .. 1
// (window-local) from the column entries acol of A; acol[m-1] holds the
// value carried in from the window below (or A(ihi, jc)).  Publishes pair
// J's (c, s) in gbuf[4J..4J+1] and then m-J in *gready; leaves acol[0] =
// the value carried out (H(lo-1, jc) at the column's top), acol[1..] = 0.
QZ_HD void hr_g_chain(int m, double* acol, double* gbuf, int* gready) {
  double y = acol[m - 1];
  for (int J = m - 1; J >= 1; --J) {
    double c, s, r;
    hr_lartg(acol[J - 1], y, c, s, r);
    gbuf[4 * J] = c;
    gbuf[4 * J + 1] = s;
    y = r;
    hr_st_rel(gready, m - J);
  }
  acol[0] = y;
  for (int J = 1; J < m; ++J) acol[J] = 0.0;
}

// The column rotations of one window (the chain threads): pairs J = m-1
// .. 1 on the diagonal block Tw (m x m, ld ldw, upper triangular), pair
// J's row rotation read from gbuf once *gready >= m-J (x.wait).  On return
// Tw is the block after the window's rotations and gbuf[4J+2..4J+3] holds
// pair J's (cz, sz).  slot: 8 doubles of shared scratch.
//
// Phase k computes pair J = m-1-k on the block thread while the far
// threads apply the pending pair P = J+1 to their entries of the block: G
// on rows P-1, P at columns >= P+1 and Z on columns P, P-1 at rows <= P-3.
// The block thread applies P's Z to row P-2 (which pair J reads) and
// stores P's 2x2 block, so each entry sees the rotations in the order of
// the sequential algorithm.  The entries pair J reads that no thread
// changes before it (its diagonal entry of the block, the original
// T(J-1, J), its row rotation once published) are loaded one phase
// ahead, so that after the barrier the block thread waits on one shared
// load, T(J-1, J+1).  On the device the block thread is lane 0 of the last
// warp (x.nt - 32 far threads before it, the rest of its warp idle); with
// one host thread (x.nt == 1) that thread does both parts.
template <class X>
QZ_HD void cta_hr_zchain(X& x, double* Tw, int ldw, int m, double* gbuf, const int* gready, double* slot) {
  auto T = [&](int i, int j) -> double& { return Tw[i + j * ldw]; };
  const int nfar = x.nt > 32 ? x.nt - 32 : x.nt;
  const bool bt = x.nt > 32 ? x.tid == nfar : true;
  const int np = m - 1;
  double pcz = 0.0, psz = 0.0, pt00 = 0.0, pt01 = 0.0, prz = 0.0;
  // block thread: the next pair's entries loaded ahead, and the count of
  // published row rotations last seen
  double nt00 = 0.0, nv = 0.0, nc = 0.0, ns = 0.0;
  int avail = 0;
  if (bt && np >= 1) {
    const int J = m - 1;
    nt00 = T(J - 1, J - 1);
    while (avail < 1) avail = x.wait(gready, 1) ? hr_ld_acq(gready) : 1;
    nc = gbuf[4 * J];
    ns = gbuf[4 * J + 1];
  }
  for (int k = 0; k <= np; ++k) {
    const int J = m - 1 - k, P = J + 1;
    if (k >= 1 && x.tid < nfar) {
      const double* sl = slot + 4 * ((k - 1) & 1);
      const double c = sl[0], s = sl[1], cz = sl[2], sz = sl[3];
      for (int t = x.tid; t < m; t += nfar) {
        if (t >= P + 1) rot2(c, s, T(P - 1, t), T(P, t));
        else if (t <= P - 3) rot2(cz, sz, T(t, P), T(t, P - 1));
      }
    }
    if (bt) {
      double a_t01 = 0.0;
      if (k >= 1) {
        if (P >= 2) {
          double u = T(P - 2, P), v = nv;
          rot2(pcz, psz, u, v);
          T(P - 2, P) = u;
          a_t01 = v;
        }
        T(P - 1, P) = pt01;
        T(P, P) = prz;
        T(P, P - 1) = 0.0;
        if (k == np) T(P - 1, P - 1) = pt00;
      }
      if (k < np) {
        const double t00 = nt00;
        const double t01 = (k == 0) ? T(J - 1, J) : a_t01;
        const double t11 = (k == 0) ? T(J, J) : pt00;
        const double c = nc, s = ns;
        double cz, sz, rz;
        const double u10 = -s * t00, u11 = -s * t01 + c * t11;
        double u00 = c * t00, u01 = c * t01 + s * t11;
        const double af = fabs(u11), ag = fabs(u10), mx = af > ag ? af : ag;
        if (u10 != 0.0 && u11 != 0.0 && mx > kSafeLo && mx < kSafeHi) {
          // the column rotation and its action on row J-1 of the block:
          // cz u01 + sz u00 = sg (u11 u01 + u10 u00) / d and -sz u01 + cz u00
          // = sg (u11 u00 - u10 u01) / d, whose numerators are formed while
          // the reciprocal square root of d^2 runs
          const double q = u11 * u11 + u10 * u10;
          const double n0 = u11 * u00 - u10 * u01, n1 = u11 * u01 + u10 * u00;
          const double inv = hr_rsqrt(q), si = (u11 < 0.0 ? -inv : inv);
          cz = af * inv;
          sz = u10 * si;
          rz = q * si;
          u00 = n0 * si;
          u01 = n1 * si;
        } else {
          hr_lartg(u11, u10, cz, sz, rz);
          rot2(cz, sz, u01, u00);
        }
        pcz = cz; psz = sz; pt00 = u00; pt01 = u01; prz = rz;
        double* sl = slot + 4 * (k & 1);
        sl[0] = c; sl[1] = s; sl[2] = cz; sl[3] = sz;
        gbuf[4 * J + 2] = cz;
        gbuf[4 * J + 3] = sz;
        // ahead: what pair J-1 reads and nobody changes before it
        if (J >= 2) {
          nt00 = T(J - 2, J - 2);
          nv = T(J - 2, J - 1);
          if (avail < k + 2) avail = x.wait(gready, k + 2) ? hr_ld_acq(gready) : k + 2;
          nc = gbuf[4 * (J - 1)];
          ns = gbuf[4 * (J - 1) + 1];
        }
      }
    }
    x.sync();
  }
}

// Operands of one reduction (device or host pointers, 0-based ihi).
struct HrArgs {
  double* A; int64_t lda;
  double* B; int64_t ldb;
  double* Q; int64_t ldq;
  double* Z; int64_t ldz;
  double* rot;  // 4 n
  int* err;     // device flag: a wait gave up
  int n, ihi;
  bool wantq, wantz, qrows;  // qrows: Q <- G Q (the transposed Q of PDGGHRD)
};

// Walk items of a window's rotations (pairs phi..plo) outside the blocks:
// (e) rows [0, e_end) of B, (f) columns phi+1..n-1 of B, (g) rows 0..ihi
// of A.  Item i of hr_win_items(..).
QZ_HD int hr_win_items(const HrArgs& a, int e_end, int phi) { return e_end + (a.n - 1 - phi) + (a.ihi + 1); }
QZ_HD void hr_win_item(const HrArgs& a, int i, int e_end, int plo, int phi) {
  const int nf = a.n - 1 - phi;
  if (i < e_end) hr_walk_z(a.B + i, a.ldb, phi, plo, a.rot);
  else if (i < e_end + nf) hr_walk_g(a.B + (int64_t)(phi + 1 + i - e_end) * a.ldb, 1, phi, plo, a.rot);
  else hr_walk_z(a.A + (i - e_end - nf), a.lda, phi, plo, a.rot);
}

// Column-end items of column jc (pairs ihi..jc+2): G on the columns
// jc+1..n-1 of A, G on Q, Z on the rows of Z.
QZ_HD int hr_col_items(const HrArgs& a, int jc) {
  return (a.n - 1 - jc) + (a.wantq ? a.n : 0) + (a.wantz ? a.n : 0);
}
QZ_HD void hr_col_item(const HrArgs& a, int i, int jc) {
  const int na = a.n - 1 - jc, nq = a.wantq ? a.n : 0;
  if (i < na) {
    hr_walk_g(a.A + (int64_t)(jc + 1 + i) * a.lda, 1, a.ihi, jc + 2, a.rot);
  } else if (i < na + nq) {
    const int r = i - na;
    if (a.qrows) hr_walk_g(a.Q + (int64_t)r * a.ldq, 1, a.ihi, jc + 2, a.rot);
    else hr_walk_g(a.Q + r, a.ldq, a.ihi, jc + 2, a.rot);
  } else {
    hr_walk_z(a.Z + (i - na - nq), a.ldz, a.ihi, jc + 2, a.rot);
  }
}

// Windows of column jc from the bottom: the first covers pairs
// [max(jc+2, ihi-W+1), ihi], each next one ends below the last.
QZ_HD int hr_win_lo(int jc, int hi, int W) { return (hi - W + 1) > (jc + 2) ? (hi - W + 1) : (jc + 2); }

}  // namespace qz
