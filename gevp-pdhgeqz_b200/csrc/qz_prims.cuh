// Scalar FP64 primitives shared by the CTA-level QZ algorithms.
//
// Every routine here is written from the mathematics (Givens rotations,
// 3-element Householder reflectors, 2x2 generalized Schur forms) and is
// usable from device and host code.  Storage is column-major.
//
// Rotation convention used throughout: a rotation (c, s) maps a pair
// (x, y) to (c*x + s*y, -s*x + c*y).  Applied to two ROWS of H and T it is
// accumulated into Q by applying the same (c, s) to the two COLUMNS of Q;
// applied to two COLUMNS of H and T it is accumulated into Z the same way.
// With that convention H_in = Q * H_out * Z^T holds at every step.
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define QZ_HD __host__ __device__ __forceinline__
#define QZ_NOINLINE __host__ __device__ __noinline__
#else
#define QZ_HD inline
#define QZ_NOINLINE inline
#endif

namespace qz {

// Column-major matrix view.
struct MatV {
  double* p;
  int ld;
  QZ_HD double& operator()(int i, int j) const { return p[i + (int64_t)j * ld]; }
};

struct Tol {
  double ulp;     // relative machine precision (DLAMCH('P') = eps*base)
  double smlnum;  // safe minimum * (n / ulp)
  double safmin;  // underflow threshold
  double ttol;    // |t(k,k)| <= ttol  => infinite eigenvalue
  double htol;    // max(unfl, ulp*||H||_F)
};

QZ_HD double dmax(double a, double b) { return a > b ? a : b; }
QZ_HD double dmin(double a, double b) { return a < b ? a : b; }
QZ_HD double dsign(double a, double b) { return b >= 0.0 ? fabs(a) : -fabs(a); }

// Givens rotation: c*f + s*g = r, -s*f + c*g = 0, c >= 0 when f != 0.
// In the range where squares cannot over/underflow the rotation costs one
// square root and one division; outside it the operands are rescaled.
constexpr double kSafeLo = 1e-140, kSafeHi = 1e140;
QZ_HD void lartg(double f, double g, double& c, double& s, double& r) {
  if (g == 0.0) {
    c = 1.0; s = 0.0; r = f;
  } else if (f == 0.0) {
    c = 0.0; s = (g > 0.0) ? 1.0 : -1.0; r = fabs(g);
  } else {
    double af = fabs(f), ag = fabs(g);
    double m = af > ag ? af : ag;
    double d;
    if (m > kSafeLo && m < kSafeHi) {
      d = sqrt(f * f + g * g);
      double inv = 1.0 / d;
      c = af * inv;
      s = g * inv;
    } else {
      double fs = f / m, gs = g / m;
      double dd = sqrt(fs * fs + gs * gs);
      c = fabs(fs) / dd;
      s = gs / dd;
      d = dd * m;
    }
    r = dsign(d, f);
    if (f < 0.0) s = -s;
  }
}

// 3-element Householder reflector P = I - tau*[1;v1;v2][1 v1 v2] with
// P*[alpha;x1;x2] = [beta;0;0].  On return alpha = beta, x1 = v1, x2 = v2.
QZ_HD void larfg3(double& alpha, double& x1, double& x2, double& tau) {
  double m = dmax(fabs(x1), fabs(x2));
  if (m == 0.0) { tau = 0.0; x1 = 0.0; x2 = 0.0; return; }
  // norm with the entries divided by the largest one (one of them is then
  // exactly 1): keeps the reflector orthogonal to a few ulp; an unscaled sum
  // of squares or a multiplication by a rounded reciprocal measurably does not
  double ma = dmax(m, fabs(alpha));
  double a = alpha / ma, b1 = x1 / ma, b2 = x2 / ma;
  double nrm = sqrt(a * a + b1 * b1 + b2 * b2) * ma;
  double beta = -dsign(nrm, alpha);
  tau = (beta - alpha) / beta;
  double scal = 1.0 / (alpha - beta);
  x1 *= scal;
  x2 *= scal;
  alpha = beta;
}

// Apply P = I - tau*v*v^T (v = [1,v1,v2]) to a 3-vector in place.
QZ_HD void refl3(double tau, double v1, double v2, double& a0, double& a1, double& a2) {
  double t = tau * (a0 + v1 * a1 + v2 * a2);
  a0 -= t;
  a1 -= t * v1;
  a2 -= t * v2;
}

QZ_HD void rot2(double c, double s, double& x, double& y) {
  double a = c * x + s * y;
  y = -s * x + c * y;
  x = a;
}

// "Opposite" reflector for a 3x3 block M (column-major m[i+3j]): returns a
// reflector (tau, v1, v2) with (M*P) e1 = gamma*e1, i.e. P e1 is parallel
// to the first column of the orthogonal factor of M = R*Zr^T (RQ).  The
// RQ factorisation is done by three column rotations.  This is the role
// of INVHSE (src/kkqz/invhse.f:1-75, PARA_ITOPP=2 branch).
QZ_HD void opposite_reflector3(const double* m_in, double& tau, double& v1, double& v2) {
  double m[9];
  for (int i = 0; i < 9; ++i) m[i] = m_in[i];
  double zr[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  double c, s, r;
  // zero m(2,0) rotating columns (1,0): new col1 = c*col1 + s*col0, new col0 = -s*col1 + c*col0
  lartg(m[2 + 3 * 1], m[2 + 3 * 0], c, s, r);
  for (int i = 0; i < 3; ++i) {
    double x = m[i + 3], y = m[i];
    m[i + 3] = c * x + s * y; m[i] = -s * x + c * y;
    x = zr[i + 3]; y = zr[i];
    zr[i + 3] = c * x + s * y; zr[i] = -s * x + c * y;
  }
  // zero m(2,1) rotating columns (2,1)
  lartg(m[2 + 3 * 2], m[2 + 3 * 1], c, s, r);
  for (int i = 0; i < 3; ++i) {
    double x = m[i + 6], y = m[i + 3];
    m[i + 6] = c * x + s * y; m[i + 3] = -s * x + c * y;
    x = zr[i + 6]; y = zr[i + 3];
    zr[i + 6] = c * x + s * y; zr[i + 3] = -s * x + c * y;
  }
  // zero m(1,0) rotating columns (1,0)
  lartg(m[1 + 3 * 1], m[1 + 3 * 0], c, s, r);
  for (int i = 0; i < 3; ++i) {
    double x = zr[i + 3], y = zr[i];
    zr[i + 3] = c * x + s * y; zr[i] = -s * x + c * y;
  }
  double a = zr[0];
  v1 = zr[1];
  v2 = zr[2];
  larfg3(a, v1, v2, tau);
}

// Householder reflector in unnormalised form, P = I - s*u*u^T with
// P*x = beta*e1: u = x - beta*e1, s = 2/(u^T u).  P is orthogonal to
// rounding whatever the accuracy of beta, because s is formed from the
// stored u.  One square root and one division.
struct House3 {
  double s, u0, u1, u2;
};
QZ_HD void house3(double x0, double x1, double x2, House3& h, double& beta) {
  if (x1 == 0.0 && x2 == 0.0) {
    h.s = 0.0; h.u0 = 1.0; h.u1 = 0.0; h.u2 = 0.0;
    beta = x0;
    return;
  }
  // P is invariant under scaling of u: outside the safe range work with
  // x / max|x| so that u^T u can neither underflow (a collapsing bulge has
  // entries far below 1e-140) nor overflow
  double m = dmax(fabs(x0), dmax(fabs(x1), fabs(x2)));
  double sc = 1.0;
  if (!(m > kSafeLo && m < kSafeHi)) {
    sc = m;
    x0 /= m; x1 /= m; x2 /= m;
  }
  double nrm = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
  double b = -dsign(nrm, x0);
  h.u0 = x0 - b;
  h.u1 = x1;
  h.u2 = x2;
  double uu = h.u0 * h.u0 + x1 * x1 + x2 * x2;
  h.s = 2.0 / uu;
  beta = b * sc;
}
QZ_HD void house3_apply(const House3& h, double& a0, double& a1, double& a2) {
  double t = h.s * (h.u0 * a0 + h.u1 * a1 + h.u2 * a2);
  a0 -= t * h.u0;
  a1 -= t * h.u1;
  a2 -= t * h.u2;
}

// Opposite reflector in unnormalised form: (M*P) e1 = gamma*e1.  The
// direction P e1 spans the null space of rows 1 and 2 of M, i.e. their
// cross product, which costs no square root or division.  Its rounding
// error grows like 1/sin(angle between the rows); when sin < 0.1 the
// direction comes from the RQ factorisation by Givens rotations instead
// (opposite_reflector3), which is backward stable for any block.
QZ_HD void opposite_house3(const double* m, House3& h) {
  double r10 = m[1], r11 = m[4], r12 = m[7];
  double r20 = m[2], r21 = m[5], r22 = m[8];
  double w0 = r11 * r22 - r12 * r21;
  double w1 = r12 * r20 - r10 * r22;
  double w2 = r10 * r21 - r11 * r20;
  double ww = w0 * w0 + w1 * w1 + w2 * w2;
  double n1 = r10 * r10 + r11 * r11 + r12 * r12;
  double n2 = r20 * r20 + r21 * r21 + r22 * r22;
  double beta;
  if (ww >= 0.01 * n1 * n2 && ww > 0.0 && isfinite(ww) && n1 * n2 < 1e280 && n1 * n2 > 1e-280) {
    house3(w0, w1, w2, h, beta);
  } else {
    double tau, v1, v2;
    opposite_reflector3(m, tau, v1, v2);
    // I - tau*v*v^T with v = [1, v1, v2] is I - s*u*u^T with u = v, s = tau
    h.s = tau; h.u0 = 1.0; h.u1 = v1; h.u2 = v2;
  }
}

// Opposite rotation for a 2x2 block: a column rotation (c, s) on columns
// (0,1) that zeros m(1,0): new col0 = c*col0 + s*col1 ... expressed in the
// global convention (x, y) -> (c*x + s*y, -s*x + c*y) on (col0, col1).
QZ_HD void opposite_rot2(double m10, double m11, double& c, double& s) {
  // want -s*m10 + c*m11 ... choose so that new (1,0) = c*m10 + s*m11 = 0
  double r;
  lartg(m11, -m10, c, s, r);  // c*m11 - s*m10 = r, s*m11 + c*m10 = 0
  // with (x,y)->(c x + s y, -s x + c y) on (col0,col1):
  // new m10 = c*m10 + s*m11 = 0 as required.
}

// Shift-polynomial first column.  Given the leading 3x3 parts of H
// (Hessenberg) and T (upper triangular) and two shifts given in
// homogeneous form through the real polynomial
//     p(M) = c2*M^2 - c1*M + c0*I,  M = H*T^{-1},
// returns v = p(M) e1 scaled by its largest entry.  For a shift pair
// lambda_1,2 = (a1/b1, a2/b2): c2 = b1*b2, c1 = a1*b2 + a2*b1, c0 = a1*a2
// (real for a real pair and for a complex-conjugate pair).  Same role as
// QZFCOL (src/kkqz/qzfcol.f:1-116).
QZ_HD void shift_column(double h11, double h21, double h12, double h22, double h32,
                        double t11, double t12, double t22,
                        double c2, double c1, double c0,
                        double& v0, double& v1, double& v2) {
  // Scale H and T entries to at most one (M = H T^{-1} scales by k =
  // tmax/hmax, so c1 -> c1*k, c0 -> c0*k^2), then form p(M) e1 multiplied
  // by t11^2 * t22: no division by a possibly tiny T diagonal entry and no
  // overflow for graded entries.
  double hm = dmax(dmax(fabs(h11), fabs(h21)), dmax(dmax(fabs(h12), fabs(h22)), fabs(h32)));
  double tm = dmax(fabs(t11), dmax(fabs(t12), fabs(t22)));
  if (hm > 0.0 && tm > 0.0 && isfinite(hm) && isfinite(tm)) {
    h11 /= hm; h21 /= hm; h12 /= hm; h22 /= hm; h32 /= hm;
    t11 /= tm; t12 /= tm; t22 /= tm;
    double k = tm / hm;
    c1 *= k;
    c0 *= k * k;
    double cm = dmax(fabs(c2), dmax(fabs(c1), fabs(c0)));
    if (cm > 0.0 && isfinite(cm)) { c2 /= cm; c1 /= cm; c0 /= cm; }
  }
  double g = h11 * t22 - t12 * h21;
  v0 = c2 * (h11 * g + h12 * h21 * t11) - c1 * h11 * t11 * t22 + c0 * t11 * t11 * t22;
  v1 = c2 * (h21 * g + h22 * h21 * t11) - c1 * h21 * t11 * t22;
  v2 = c2 * h32 * h21 * t11;
  double m = dmax(fabs(v0), dmax(fabs(v1), fabs(v2)));
  if (m > 0.0 && isfinite(m)) {
    v0 /= m; v1 /= m; v2 /= m;
  } else {
    // degenerate polynomial column: no bulge (identity reflector)
    v0 = 1.0; v1 = 0.0; v2 = 0.0;
  }
}

// Eigenvalues of a 2x2 pencil (A, B), B upper triangular (b10 = 0), as
// the coefficients of the real quadratic c2*l^2 - c1*l + c0 with
//   c2 = b00*b11, c1 = a00*b11 + a11*b00 - a10*b01, c0 = a00*a11 - a01*a10.
QZ_HD void pencil2_poly(double a00, double a10, double a01, double a11,
                        double b00, double b01, double b11,
                        double& c2, double& c1, double& c0) {
  double sa = dmax(dmax(fabs(a00), fabs(a10)), dmax(fabs(a01), fabs(a11)));
  double sb = dmax(dmax(fabs(b00), fabs(b01)), fabs(b11));
  if (sa == 0.0) sa = 1.0;
  if (sb == 0.0) sb = 1.0;
  a00 /= sa; a10 /= sa; a01 /= sa; a11 /= sa;
  b00 /= sb; b01 /= sb; b11 /= sb;
  // lambda scales by sa/sb: c2*l^2 - c1*l + c0 with l = (sa/sb) l'
  double k = sa / sb;
  c2 = b00 * b11;
  c1 = (a00 * b11 + a11 * b00 - a10 * b01) * k;
  c0 = (a00 * a11 - a01 * a10) * k * k;
}

// Result of standardising a 2x2 pencil.
struct Std2 {
  double csl, snl;  // row rotation on (0,1)
  double csr, snr;  // column rotation on (0,1)
  double a[4];      // transformed A (column-major)
  double b[4];      // transformed B (column-major)
  int cplx;         // 1: complex-conjugate pair, 0: two real eigenvalues
  int negrow0, negrow1;  // rows to negate (complex case, to make B diagonal positive)
};

QZ_HD void apply_rows2(double* m, double c, double s) {
  // m column-major 2x2, rotate rows 0/1
  rot2(c, s, m[0], m[1]);
  rot2(c, s, m[2], m[3]);
}
QZ_HD void apply_cols2(double* m, double c, double s) {
  rot2(c, s, m[0], m[2]);
  rot2(c, s, m[1], m[3]);
}

// Generalized real Schur form of a 2x2 pencil (the job of LAPACK DLAGV2,
// called at PDHGEQZ0.f:630 and PDHGEQZ1.f:693): rotations making
//  * real eigenvalues: both A and B upper triangular;
//  * complex pair: B diagonal with b00 >= b11 > 0 (rows negated as needed).
// B may be a general 2x2 on entry.
QZ_HD void std2x2(const double* A, const double* B, Std2& o) {
  double a[4] = {A[0], A[1], A[2], A[3]};
  double b[4] = {B[0], B[1], B[2], B[3]};
  double c, s, r;
  // make B upper triangular first (row rotation)
  double csl = 1.0, snl = 0.0, csr = 1.0, snr = 0.0;
  if (b[1] != 0.0) {
    lartg(b[0], b[1], c, s, r);
    apply_rows2(a, c, s);
    apply_rows2(b, c, s);
    b[1] = 0.0;
    csl = c; snl = s;
  }
  o.negrow0 = 0; o.negrow1 = 0;
  double c2, c1, c0;
  pencil2_poly(a[0], a[1], a[2], a[3], b[0], b[2], b[3], c2, c1, c0);
  double disc = c1 * c1 - 4.0 * c2 * c0;
  bool cplx = (a[1] != 0.0) && (disc < 0.0) && (c2 != 0.0);
  double rc, rs;  // row rotation (composed later)
  if (!cplx) {
    o.cplx = 0;
    if (a[1] == 0.0) {
      rc = 1.0; rs = 0.0; c = 1.0; s = 0.0;
    } else {
      // one eigenvalue in homogeneous form (alpha, beta): beta*A - alpha*B singular
      double al, be;
      if (c2 == 0.0) {
        // infinite eigenvalue present: beta = 0, alpha = 1
        al = 1.0; be = 0.0;
      } else {
        double sq = sqrt(dmax(disc, 0.0));
        // root with larger |numerator| avoids cancellation
        double num = (c1 >= 0.0) ? (c1 + sq) : (c1 - sq);
        al = num; be = 2.0 * c2;
        double mm = dmax(fabs(al), fabs(be));
        al /= mm; be /= mm;
      }
      double sa = dmax(dmax(fabs(a[0]), fabs(a[1])), dmax(fabs(a[2]), fabs(a[3])));
      double sb = dmax(dmax(fabs(b[0]), fabs(b[2])), fabs(b[3]));
      if (sa == 0.0) sa = 1.0;
      if (sb == 0.0) sb = 1.0;
      // M = be*A - al*B is singular; (al, be) are in true units.  Divide
      // the two terms by their natural sizes before forming M.
      double ka = be / sa, kb = al / sa;
      double m00 = ka * a[0] - kb * b[0], m01 = ka * a[2] - kb * b[2];
      double m10 = ka * a[1],             m11 = ka * a[3] - kb * b[3];
      double n0 = fabs(m00) + fabs(m01), n1 = fabs(m10) + fabs(m11);
      double z0, z1;
      if (n0 >= n1) { z0 = -m01; z1 = m00; } else { z0 = -m11; z1 = m10; }
      double zn = sqrt(z0 * z0 + z1 * z1);
      if (zn == 0.0) { z0 = 1.0; z1 = 0.0; zn = 1.0; }
      c = z0 / zn; s = z1 / zn;
      if (c < 0.0) { c = -c; s = -s; }
      // new col0 = c*col0 + s*col1 = M*(c,s)
      apply_cols2(a, c, s);
      apply_cols2(b, c, s);
      // left rotation mapping the (parallel) first columns to e1
      double nb = fabs(b[0]) + fabs(b[1]);
      double na = fabs(a[0]) + fabs(a[1]);
      if (nb / sb >= na / sa) lartg(b[0], b[1], rc, rs, r);
      else lartg(a[0], a[1], rc, rs, r);
      apply_rows2(a, rc, rs);
      apply_rows2(b, rc, rs);
      a[1] = 0.0;
      b[1] = 0.0;
    }
  } else {
    o.cplx = 1;
    // one-sided Jacobi on the columns of B to make them orthogonal
    double p0 = b[0], p1 = b[1], q0 = b[2], q1 = b[3];
    double alpha = p0 * p0 + p1 * p1, beta = q0 * q0 + q1 * q1, gamma = p0 * q0 + p1 * q1;
    if (gamma == 0.0) {
      c = 1.0; s = 0.0;
    } else {
      double zeta = (beta - alpha) / (2.0 * gamma);
      double t = dsign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
      c = 1.0 / sqrt(1.0 + t * t);
      s = c * t;
      // rotation (x,y)->(c x - s y, s x + c y) on (col0,col1) orthogonalises;
      // in our convention that is (c, -s)
      s = -s;
    }
    apply_cols2(a, c, s);
    apply_cols2(b, c, s);
    // order columns so that |col0| >= |col1|
    double n0 = b[0] * b[0] + b[1] * b[1], n1 = b[2] * b[2] + b[3] * b[3];
    if (n1 > n0) {
      // extra rotation by 90 degrees: (x,y)->(y,-x) is (c=0,s=1)
      double cc = 0.0, ss = 1.0;
      apply_cols2(a, cc, ss);
      apply_cols2(b, cc, ss);
      // compose: first (c,s) then (0,1): combined angle
      double c_new = c * cc - s * ss;
      double s_new = s * cc + c * ss;
      c = c_new; s = s_new;
    }
    lartg(b[0], b[1], rc, rs, r);
    apply_rows2(a, rc, rs);
    apply_rows2(b, rc, rs);
    b[1] = 0.0;
    b[2] = 0.0;
    if (b[0] < 0.0) { o.negrow0 = 1; b[0] = -b[0]; a[0] = -a[0]; a[2] = -a[2]; }
    if (b[3] < 0.0) { o.negrow1 = 1; b[3] = -b[3]; a[1] = -a[1]; a[3] = -a[3]; }
  }
  // compose row rotations: first (csl,snl) then (rc,rs)
  double cl = rc * csl - rs * snl;
  double sl = rs * csl + rc * snl;
  o.csl = cl; o.snl = sl;
  o.csr = c;  o.snr = s;
  for (int i = 0; i < 4; ++i) { o.a[i] = a[i]; o.b[i] = b[i]; }
  csr = c; snr = s;
  (void)csr; (void)snr;
}

// Eigenvalues (LAPACK DHGEQZ conventions) of a standardised complex 2x2
// block: A full, B = diag(b0, b1) > 0.  Writes (alphar, alphai, beta) for
// both rows, alphai > 0 on the first.
QZ_HD void eig2_complex(const double* a, double b0, double b1, double* ar, double* ai, double* be) {
  double m00 = a[0] / b0, m01 = a[2] / b0, m10 = a[1] / b1, m11 = a[3] / b1;
  // M = diag(b)^-1 A scaled by a power of two to at most 1 in magnitude, so
  // that the discriminant cannot overflow for eigenvalues far from 1 in
  // magnitude; the scaling is exact and is folded back into b, so the
  // results are the unscaled formula's wherever that one does not overflow
  const double mx = dmax(dmax(fabs(m00), fabs(m01)), dmax(fabs(m10), fabs(m11)));
  int e = 0;
  if (mx > 0.0 && isfinite(mx)) frexp(mx, &e);
  m00 = ldexp(m00, -e); m01 = ldexp(m01, -e); m10 = ldexp(m10, -e); m11 = ldexp(m11, -e);
  double tr = 0.5 * (m00 + m11);
  double d = 0.5 * (m00 - m11);
  // disc = d^2 + m01 m10 (< 0 for a complex pair) with the rounding error of
  // the product added back (fma), so a nearly real pair, where the two terms
  // almost cancel, keeps its imaginary part accurate
  const double p = m01 * m10;
  const double perr = fma(m01, m10, -p);
  double disc = fma(d, d, p) + perr;
  double wr = tr;
  double wi = sqrt(fabs(dmin(disc, 0.0)));
  const double s0 = ldexp(b0, e), s1 = ldexp(b1, e);
  ar[0] = wr * s0; ai[0] = wi * s0; be[0] = b0;
  ar[1] = wr * s1; ai[1] = -wi * s1; be[1] = b1;
}

}  // namespace qz
