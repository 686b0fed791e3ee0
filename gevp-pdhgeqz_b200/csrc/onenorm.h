// Host-side 1-norm estimator of a linear operator given only by products
// (used for DTGSEN's Dif estimates; tested against LAPACK's DLACN2 by the
// host build).
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

namespace qz {

// 1-norm estimate of a linear operator Op of order n from products with Op
// and Op^T (Hager's method with Higham's refinements: the sign-vector
// iteration stops on a repeated sign vector, a non-increasing estimate or
// five iterations, and the alternating vector x_i = (-1)^i (1 + i/(n-1))
// guards the result; N. J. Higham, ACM TOMS 14 (1988) 381-396, the
// algorithm of LAPACK's DLACN2).  apply(kind, x) replaces x by Op x (kind
// 1) or Op^T x (kind 2) and returns false on a device error.
template <class F>
inline double onenorm_est(int n, F&& apply, bool& ok) {
  std::vector<double> x(n, 1.0 / n);
  std::vector<int> sgn(n);
  auto asum = [&]() { double t = 0.0; for (double v : x) t += fabs(v); return t; };
  auto imax = [&]() { int j = 0; for (int i = 1; i < n; ++i) if (fabs(x[i]) > fabs(x[j])) j = i; return j; };
  ok = apply(1, x);
  if (!ok) return 0.0;
  if (n == 1) return fabs(x[0]);
  double est = asum();
  for (int i = 0; i < n; ++i) { x[i] = x[i] >= 0.0 ? 1.0 : -1.0; sgn[i] = (int)x[i]; }
  ok = apply(2, x);
  if (!ok) return 0.0;
  int j = imax();
  for (int iter = 2;; ++iter) {
    std::fill(x.begin(), x.end(), 0.0);
    x[j] = 1.0;
    ok = apply(1, x);
    if (!ok) return 0.0;
    const double estold = est;
    est = asum();
    bool same = true;
    for (int i = 0; i < n && same; ++i) same = (x[i] >= 0.0 ? 1 : -1) == sgn[i];
    if (same || est <= estold) break;
    for (int i = 0; i < n; ++i) { x[i] = x[i] >= 0.0 ? 1.0 : -1.0; sgn[i] = (int)x[i]; }
    ok = apply(2, x);
    if (!ok) return 0.0;
    const int jlast = j;
    j = imax();
    if (!(x[jlast] != fabs(x[j]) && iter < 5)) break;
  }
  double alt = 1.0;
  for (int i = 0; i < n; ++i) { x[i] = alt * (1.0 + (double)i / (n - 1)); alt = -alt; }
  ok = apply(1, x);
  if (!ok) return 0.0;
  const double temp = 2.0 * (asum() / (3.0 * n));
  return temp > est ? temp : est;
}

}  // namespace qz
