// Host build of the library's CTA-level QZ algorithms, for the CPU tests.
//
// The window routines of the device kernels (qz_cta.cuh, qz_chase.cuh) and
// the iteration driver (qz_solver.h) are templates over an executor; here
// they run with a single host "thread" (tid 0 of 1, barriers are no-ops),
// and a host backend plays the part of the device kernels with the same
// window copies, factor updates and deflation scan.  This checks the
// algorithms and the solver's control logic against LAPACK without a GPU;
// thread-level concurrency is checked by the GPU tests.
//
// Built by tests/test_cpu_host_algorithms.py with g++ into a temporary
// directory.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "../gevp-pdhgeqz_b200/csrc/qz_solver.h"
#include "../gevp-pdhgeqz_b200/csrc/hessred.cuh"
#include "../gevp-pdhgeqz_b200/csrc/onenorm.h"

using namespace qz;

namespace {

// Barrier counts by AED phase (the latency model of the device kernels:
// each barrier separates two dependent steps): [0] outside the AED kernel
// routine, [1] window QZ, [2] spike test + reordering, [3] spike reflector
// + RQ update, [4] Hessenberg-triangular re-reduction; [5] AED routine calls.
static long g_barriers[6] = {0, 0, 0, 0, 0, 0};
static int g_phase = 0;

// Pipelined double-shift sweeps (core step, then far step, per step) when
// set by host_set_pipe; the two-barrier form otherwise.
static bool g_pipe = false;
static PipeBuf g_pipebuf;

struct HostExec {
  int tid = 0, nt = 1;
  int si[64];
  double* sd;
  std::vector<double> sdv;
  PipeBuf* pipe = nullptr;
  HostExec() : sdv(16384, 0.0) { sd = sdv.data(); }
  void use_pipe() { pipe = g_pipe ? &g_pipebuf : nullptr; }
  void sync() { ++g_barriers[g_phase]; }
  void stamp(int k) {
    g_phase = (k < 4) ? k + 1 : 0;
    if (k == 0) ++g_barriers[5];
  }
  void count(int) {}
  bool wait(const int*, int) { return true; }
};

Tol make_tol(const double* H, const double* T, int ld, int o, int nh) {
  double hn = 0.0, tn = 0.0;
  for (int j = 0; j < nh; ++j)
    for (int i = 0; i < nh; ++i) {
      const double a = H[(o + i) + (size_t)(o + j) * ld], b = T[(o + i) + (size_t)(o + j) * ld];
      hn += a * a;
      tn += b * b;
    }
  Tol t;
  t.safmin = DBL_MIN;
  t.ulp = DBL_EPSILON;
  t.smlnum = DBL_MIN * ((double)nh / DBL_EPSILON);
  t.htol = dmax(DBL_MIN, DBL_EPSILON * sqrt(hn));
  t.ttol = dmax(DBL_MIN, DBL_EPSILON * sqrt(tn));
  return t;
}

int balance_exponent(const double* H, const double* T, int ld, int o, int nh) {
  double hm = 0.0, tm = 0.0;
  for (int j = 0; j < nh; ++j)
    for (int i = 0; i < nh; ++i) {
      hm = dmax(hm, fabs(H[(o + i) + (size_t)(o + j) * ld]));
      tm = dmax(tm, fabs(T[(o + i) + (size_t)(o + j) * ld]));
    }
  return qz::balance_exponent(hm, tm);
}

struct HostBK {
  int n, ld;
  double *H, *T, *Q, *Z;
  bool wantq = true, wantz = true;
  int nskip = 4;
  int swapfail = 0;
  int ms = 1;  // multishift window QZ
  // JOB = 'E': far updates of H and T stop at the active block (as in the
  // device backend)
  bool schur = true;
  int act_top = 0, act_bot = 0;
  int far_col_end() const { return schur ? n : act_bot + 1; }
  int far_row_begin() const { return schur ? 0 : act_top; }
  Tol tol;
  HostExec x;
  std::vector<double> Ua, Va;                 // last AED window factors
  std::vector<std::vector<double>> Uc, Vc;    // chase / zero-chase factors per window of a wave
  double& h(int i, int j) { return H[i + (size_t)j * ld]; }
  double& t(int i, int j) { return T[i + (size_t)j * ld]; }

  void scan(int ifirst, int kbot, int* out) {
    int bad = 0;
    for (int j = ifirst; j <= kbot; ++j) {
      const double a = h(j, j), b = t(j, j), c = (j > ifirst) ? h(j, j - 1) : 0.0;
      if (!std::isfinite(a) || !std::isfinite(b) || !std::isfinite(c)) bad = 1;
    }
    int ktop = ifirst;
    for (int k = kbot; k > ifirst; --k)
      if (negligible_sub(h(k, k - 1), h(k - 1, k - 1), h(k, k), tol)) { ktop = k; break; }
    if (ktop > ifirst) h(ktop, ktop - 1) = 0.0;
    int cnt = 0, jmax = -1, jmin = -1;
    for (int j = ktop; j <= kbot; ++j)
      if (fabs(t(j, j)) <= tol.ttol) {
        t(j, j) = 0.0;
        ++cnt;
        jmax = j;
        if (jmin < 0) jmin = j;
      }
    out[0] = ktop; out[1] = cnt; out[2] = jmax; out[3] = jmin; out[4] = bad;
  }

  void load(int w, int wk, std::vector<double>& Hs, std::vector<double>& Ts, std::vector<double>& Us,
            std::vector<double>& Vs) {
    Hs.assign((size_t)wk * wk, 0.0); Ts = Hs; Us = Hs; Vs = Hs;
    for (int j = 0; j < wk; ++j) {
      for (int i = 0; i < wk; ++i) { Hs[i + (size_t)j * wk] = h(w + i, w + j); Ts[i + (size_t)j * wk] = t(w + i, w + j); }
      Us[j + (size_t)j * wk] = 1.0;
      Vs[j + (size_t)j * wk] = 1.0;
    }
  }
  void store(int w, int wk, const std::vector<double>& Hs, const std::vector<double>& Ts) {
    for (int j = 0; j < wk; ++j)
      for (int i = 0; i < wk; ++i) { h(w + i, w + j) = Hs[i + (size_t)j * wk]; t(w + i, w + j) = Ts[i + (size_t)j * wk]; }
  }

  void aed(int ktop, int kwtop, int kbot, int* info3, double* sh) {
    const int nw = kbot - kwtop + 1;
    std::vector<double> Hs, Ts, Us, Vs, s3(3 * (size_t)nw);
    load(kwtop, nw, Hs, Ts, Us, Vs);
    const double s = (kwtop > ktop) ? h(kwtop, kwtop - 1) : 0.0;
    WinState w;
    w.n = nw; w.H = MatV{Hs.data(), nw}; w.T = MatV{Ts.data(), nw}; w.Q = MatV{Us.data(), nw};
    w.Z = MatV{Vs.data(), nw}; w.wantq = true; w.wantz = true; w.tol = tol;
    cta_aed(x, w, s, s3.data(), s3.data() + nw, s3.data() + 2 * nw, 30 * nw, (kwtop > ktop) ? nskip : 0,
            swapfail != 0, ms ? x.sd + 64 + 4 * nw : nullptr);
    const int m = x.si[8], st = x.si[9], tr = x.si[10];
    if (st == 0 && tr) {
      store(kwtop, nw, Hs, Ts);
      if (kwtop > ktop) h(kwtop, kwtop - 1) = s * Us[0];
      Ua = Us;
      Va = Vs;
    }
    info3[0] = m; info3[1] = st; info3[2] = tr;
    const int mm = m < nw ? m : nw;
    for (int i = 0; i < mm; ++i) { sh[i] = s3[i]; sh[mm + i] = s3[nw + i]; sh[2 * mm + i] = s3[2 * nw + i]; }
  }

  // off-diagonal updates with a window's factors, left part or right part
  void apply_left(int w, int wk, const std::vector<double>& U) {
    std::vector<double> col(wk);
    for (double* M : {H, T})
      for (int c = w + wk; c < far_col_end(); ++c) {
        for (int i = 0; i < wk; ++i) {
          double a = 0.0;
          for (int k = 0; k < wk; ++k) a += U[k + (size_t)i * wk] * M[(w + k) + (size_t)c * ld];
          col[i] = a;
        }
        for (int i = 0; i < wk; ++i) M[(w + i) + (size_t)c * ld] = col[i];
      }
  }
  void apply_right(int w, int wk, const std::vector<double>& U, const std::vector<double>& V) {
    std::vector<double> row(wk);
    auto right = [&](double* M, int r0, int rows, const std::vector<double>& W) {
      for (int r = r0; r < rows; ++r) {
        for (int j = 0; j < wk; ++j) {
          double a = 0.0;
          for (int k = 0; k < wk; ++k) a += M[r + (size_t)(w + k) * ld] * W[k + (size_t)j * wk];
          row[j] = a;
        }
        for (int j = 0; j < wk; ++j) M[r + (size_t)(w + j) * ld] = row[j];
      }
    };
    right(H, far_row_begin(), w, V);
    right(T, far_row_begin(), w, V);
    if (wantq) right(Q, 0, n, U);
    if (wantz) right(Z, 0, n, V);
  }
  void update(int w, int wk, int which) {
    const std::vector<double>& U = which == 0 ? Ua : Uc[0];
    const std::vector<double>& V = which == 0 ? Va : Vc[0];
    apply_left(w, wk, U);
    apply_right(w, wk, U, V);
  }

  void chase_wave(const WinPlan* const* wins, int nw) {
    Uc.assign(nw, {});
    Vc.assign(nw, {});
    for (int i = 0; i < nw; ++i) {
      const WinPlan& p = *wins[i];
      std::vector<double> Hs, Ts, Us, Vs;
      load(p.w, p.wk, Hs, Ts, Us, Vs);
      std::vector<BulgeRec> rec(p.nb);
      cta_chase_window(x, p.wk, p.last, MatV{Hs.data(), p.wk}, MatV{Ts.data(), p.wk}, MatV{Us.data(), p.wk},
                       MatV{Vs.data(), p.wk}, p.bl.data(), p.nb, p.tmax, rec.data());
      store(p.w, p.wk, Hs, Ts);
      Uc[i] = Us;
      Vc[i] = Vs;
    }
  }
  // as on the device: every left update of the wave, then every right one
  void update_wave(const WinPlan* const* wins, int nw) {
    for (int i = 0; i < nw; ++i) apply_left(wins[i]->w, wins[i]->wk, Uc[i]);
    for (int i = 0; i < nw; ++i) apply_right(wins[i]->w, wins[i]->wk, Uc[i], Vc[i]);
  }
  void inf_window(int w, int wk, int top, int jz, int stop, bool deflate) {
    std::vector<double> Hs, Ts, Us, Vs;
    load(w, wk, Hs, Ts, Us, Vs);
    cta_inf_window(x, wk, top, jz, stop, deflate, MatV{Hs.data(), wk}, MatV{Ts.data(), wk}, MatV{Us.data(), wk},
                   MatV{Vs.data(), wk});
    store(w, wk, Hs, Ts);
    Uc.assign(1, Us);
    Vc.assign(1, Vs);
  }
  void inf_top(int f) {
    double c, s, r;
    lartg(h(f, f), h(f + 1, f), c, s, r);
    for (int j = f + 1; j < n; ++j) {
      double a = h(f, j), b = h(f + 1, j);
      h(f, j) = c * a + s * b; h(f + 1, j) = -s * a + c * b;
      a = t(f, j); b = t(f + 1, j);
      t(f, j) = c * a + s * b; t(f + 1, j) = -s * a + c * b;
    }
    if (wantq)
      for (int i = 0; i < n; ++i) {
        double a = Q[i + (size_t)f * ld], b = Q[i + (size_t)(f + 1) * ld];
        Q[i + (size_t)f * ld] = c * a + s * b; Q[i + (size_t)(f + 1) * ld] = -s * a + c * b;
      }
    h(f, f) = r;
    h(f + 1, f) = 0.0;
  }
  bool policy(int, int, double, int*, int*) { return false; }
  void active(int ktop, int kbot) {
    act_top = ktop;
    act_bot = kbot;
  }
};

}  // namespace

extern "C" {

void host_set_pipe(int on) { g_pipe = on != 0; }

// Swap of the 1x1 blocks of the 2x2 pencil (S, T) (column-major, upper
// triangular): out = {ok, S2[4], T2[4], Q[4], Z[4]}; general = 1 takes the
// generalized Sylvester path, 0 the two-rotation path.
void host_swap11(const double* S, const double* T, int general, double* out) {
  double S2[4], T2[4], Qs[4], Zs[4];
  double s[4] = {S[0], S[1], S[2], S[3]}, t[4] = {T[0], T[1], T[2], T[3]};
  const bool ok = general ? swap_compute<1, 1>(MatV{s, 2}, MatV{t, 2}, S2, T2, Qs, Zs, DBL_EPSILON, DBL_MIN)
                          : swap_compute11(MatV{s, 2}, MatV{t, 2}, S2, T2, Qs, Zs, DBL_EPSILON, DBL_MIN);
  out[0] = ok ? 1.0 : 0.0;
  for (int i = 0; i < 4; ++i) { out[1 + i] = S2[i]; out[5 + i] = T2[i]; out[9 + i] = Qs[i]; out[13 + i] = Zs[i]; }
}
// steps of the last pipelined sweep that the far part completed (far_done)
int host_pipe_far_done() { return g_pipebuf.far_done; }

void host_barriers(long* out, int reset) {
  for (int i = 0; i < 6; ++i) out[i] = g_barriers[i];
  if (reset)
    for (int i = 0; i < 6; ++i) g_barriers[i] = 0;
}

// Window QZ of an n x n pencil (Q, Z accumulate from their input).
int host_small_qz(int n, double* H, double* T, double* Q, double* Z) {
  static HostExec x;
  x.use_pipe();
  WinState w;
  w.n = n; w.H = MatV{H, n}; w.T = MatV{T, n}; w.Q = MatV{Q, n}; w.Z = MatV{Z, n};
  w.wantq = w.wantz = true;
  w.tol = make_tol(H, T, n, 0, n);
  return cta_small_qz(x, w, 30 * n);
}

// The same with the multishift window QZ (lockstep chains of bulges).
int host_small_qz_ms(int n, double* H, double* T, double* Q, double* Z) {
  static HostExec x;
  x.use_pipe();
  WinState w;
  w.n = n; w.H = MatV{H, n}; w.T = MatV{T, n}; w.Q = MatV{Q, n}; w.Z = MatV{Z, n};
  w.wantq = w.wantz = true;
  w.tol = make_tol(H, T, n, 0, n);
  return cta_small_qz_ms(x, w, 30 * n, x.sd + 1024);
}

// AED on a whole window with spike s (Q, Z identity on entry); out3 =
// {undeflated m, status, transformed}; shifts: alphar, alphai, beta (n each).
void host_aed(int n, double* H, double* T, double* Q, double* Z, double s, int nskip, double* shifts, int* out3) {
  static HostExec x;
  x.use_pipe();
  WinState w;
  w.n = n; w.H = MatV{H, n}; w.T = MatV{T, n}; w.Q = MatV{Q, n}; w.Z = MatV{Z, n};
  w.wantq = w.wantz = true;
  w.tol = make_tol(H, T, n, 0, n);
  cta_aed(x, w, s, shifts, shifts + n, shifts + 2 * n, 30 * n, nskip);
  out3[0] = x.si[8]; out3[1] = x.si[9]; out3[2] = x.si[10];
}

// Chase a chain of nb bulges through an n x n window (the whole matrix):
// bulges int[4*nb] = {base, tlo, thi, intro} per bulge, coef double[3*nb]
// = {c2, c1, c0}; U, V identity on entry accumulate the transformations.
void host_chase(int n, double* H, double* T, double* U, double* V, const int* bulges, const double* coef, int nb,
                int tmax, int last) {
  static HostExec x;
  x.use_pipe();
  std::vector<Bulge> bl(nb);
  for (int b = 0; b < nb; ++b) {
    bl[b].base = bulges[4 * b]; bl[b].tlo = bulges[4 * b + 1]; bl[b].thi = bulges[4 * b + 2];
    bl[b].intro = bulges[4 * b + 3];
    bl[b].c2 = coef[3 * b]; bl[b].c1 = coef[3 * b + 1]; bl[b].c0 = coef[3 * b + 2];
  }
  std::vector<BulgeRec> rec(nb);
  cta_chase_window(x, n, last, MatV{H, n}, MatV{T, n}, MatV{U, n}, MatV{V, n}, bl.data(), nb, tmax, rec.data());
}

// Full solve with the library's iteration driver and the host backend
// (COMPQ = COMPZ = 'I'); eigenvalues to ar, ai, be.  stats: iterations,
// AEDs, sweeps, chase windows, zero-chase steps.
int host_solve(int n, double* H, double* T, double* Q, double* Z, int nw_max, int w_chase, int nmin, int nskip,
               double* ar, double* ai, double* be, int* stats) {
  HostBK bk;
  bk.x.use_pipe();
  bk.n = n; bk.ld = n; bk.H = H; bk.T = T; bk.Q = Q; bk.Z = Z; bk.nskip = nskip;
  // as the library does: T scaled by a power of two when its norm is far
  // from H's (shifts and their polynomials stay in range), undone at the end
  const int e = balance_exponent(H, T, n, 0, n);
  if (e != 0)
    for (size_t i = 0; i < (size_t)n * n; ++i) T[i] = ldexp(T[i], e);
  bk.tol = make_tol(H, T, n, 0, n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) { Q[i + (size_t)j * n] = (i == j); Z[i + (size_t)j * n] = (i == j); }
  SolveParams P;
  P.nw_max = nw_max; P.w_chase = w_chase; P.nmin = nmin;
  SolveStats S;
  int info = (n > 0) ? qz_iterate(bk, n, 0, n - 1, P, S) : 0;
  if (e != 0)
    for (size_t i = 0; i < (size_t)n * n; ++i) T[i] = ldexp(T[i], -e);
  if (info == 0) {
    WinState w;
    w.n = n; w.H = MatV{H, n}; w.T = MatV{T, n}; w.Q = MatV{Q, n}; w.Z = MatV{Z, n};
    w.wantq = w.wantz = true;
    w.tol = bk.tol;
    cta_finalize(bk.x, w, ar, ai, be);
  }
  stats[0] = (int)S.iters; stats[1] = (int)S.aeds; stats[2] = (int)S.sweeps; stats[3] = (int)S.windows;
  stats[4] = (int)S.infs;
  return info;
}

// The same with more controls: ip = {nw_max, w_chase, nmin, nskip,
// stall_limit, aed_swap_fail, schur (1: JOB='S', 0: JOB='E'), window QZ
// (1: multishift, 0: double shift)}.  Returns
// INFO (0, or the 1-based unconverged row).  The eigenvalues are read from
// the diagonal blocks also for JOB='E'.
int host_solve_p(int n, double* H, double* T, double* Q, double* Z, const int* ip, double* ar, double* ai, double* be,
                 int* stats) {
  HostBK bk;
  bk.x.use_pipe();
  bk.n = n; bk.ld = n; bk.H = H; bk.T = T; bk.Q = Q; bk.Z = Z; bk.nskip = ip[3];
  bk.swapfail = ip[5];
  bk.schur = ip[6] != 0;
  bk.ms = ip[7];
  bk.act_top = 0;
  bk.act_bot = n - 1;
  bk.tol = make_tol(H, T, n, 0, n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) { Q[i + (size_t)j * n] = (i == j); Z[i + (size_t)j * n] = (i == j); }
  SolveParams P;
  P.nw_max = ip[0]; P.w_chase = ip[1]; P.nmin = ip[2];
  P.stall_limit = ip[4];
  P.aed_swap_fail = ip[5];
  SolveStats S;
  int info = (n > 0) ? qz_iterate(bk, n, 0, n - 1, P, S) : 0;
  if (info == 0) {
    WinState w;
    w.n = n; w.H = MatV{H, n}; w.T = MatV{T, n}; w.Q = MatV{Q, n}; w.Z = MatV{Z, n};
    w.wantq = w.wantz = true;
    w.tol = bk.tol;
    cta_finalize(bk.x, w, ar, ai, be);
  }
  stats[0] = (int)S.iters; stats[1] = (int)S.aeds; stats[2] = (int)S.sweeps; stats[3] = (int)S.windows;
  stats[4] = (int)S.infs;
  return info;
}

// Hessenberg-triangular reduction with the device's launch sequence
// (hessred.cu): per column, window launches (CTA 0 part and helper walks),
// the last window's walks, the column-end walks.  order 0 runs a launch's
// CTA 0 part before its helper items, 1 after them, 2 after them in
// reverse order: the parts touch disjoint entries, so all three give the
// same bits.  icompq/icompz 0 none, 1 update, 2 identity first.
int host_gghrd(int n, int ilo, int ihi, double* A, double* B, double* Q, double* Z, int W, int icompq, int icompz,
               int qrows, int order) {
  if (icompq == 2)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) Q[i + (size_t)j * n] = (i == j);
  if (icompz == 2)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) Z[i + (size_t)j * n] = (i == j);
  if (n <= 1) return 0;
  for (int j = 0; j < n; ++j)
    for (int i = j + 1; i < n; ++i) B[i + (size_t)j * n] = 0.0;
  std::vector<double> rot(4 * (size_t)n, 0.0), sm(hr_smem_doubles(W) + 8, 0.0);
  int err = 0;
  HrArgs a{A, n, B, n, Q, n, Z, n, rot.data(), &err, n, ihi, icompq != 0, icompz != 0, qrows != 0};
  HostExec x;
  int launches = 0;
  auto items = [&](int cnt, auto&& f) {
    if (order == 2)
      for (int i = cnt - 1; i >= 0; --i) f(i);
    else
      for (int i = 0; i < cnt; ++i) f(i);
  };
  // CTA 0 of a window launch (hessred.cu hr_window_cta), one host thread
  auto window = [&](int jc, int lo, int hi, int plo, int phi) {
    const int o = lo - 1, m = hi - lo + 2, ldw = hr_ldw(m);
    const HrSmem L = hr_layout(sm.data(), W);
    if (plo >= 0)
      for (int r = o; r <= hi - 1; ++r) hr_walk_z(B + r, n, phi, plo, rot.data());
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) L.Tw[i + j * ldw] = (i <= j) ? B[(o + i) + (size_t)(o + j) * n] : 0.0;
    for (int i = 0; i < m; ++i) L.acol[i] = A[(o + i) + (size_t)jc * n];
    *L.gready = 0;
    hr_g_chain(m, L.acol, L.gbuf, L.gready);
    cta_hr_zchain(x, L.Tw, ldw, m, L.gbuf, L.gready, L.slot);
    for (int i = 4; i < 4 * m; ++i) rot[4 * o + i] = L.gbuf[i];
    for (int j = 0; j < m; ++j)
      for (int i = 0; i <= j; ++i) B[(o + i) + (size_t)(o + j) * n] = L.Tw[i + j * ldw];
    for (int i = 0; i < m; ++i) A[(o + i) + (size_t)jc * n] = L.acol[i];
  };
  for (int jc = ilo; jc <= ihi - 2; ++jc) {
    int plo = -1, phi = -1;
    for (int hi = ihi; hi >= jc + 2;) {
      const int lo = hr_win_lo(jc, hi, W);
      auto helpers = [&]() {
        if (plo >= 0) items(hr_win_items(a, lo - 1, phi), [&](int i) { hr_win_item(a, i, lo - 1, plo, phi); });
      };
      if (order != 0) helpers();
      window(jc, lo, hi, plo, phi);
      if (order == 0) helpers();
      ++launches;
      plo = lo; phi = hi; hi = lo - 1;
    }
    items(hr_win_items(a, plo - 1, phi), [&](int i) { hr_win_item(a, i, plo - 1, plo, phi); });
    items(hr_col_items(a, jc), [&](int i) { hr_col_item(a, i, jc); });
    launches += 2;
  }
  return launches;
}

// The reduction's Givens rotation (hessred.cuh hr_lartg) for a test
// against LAPACK's DLARTG convention.
void host_hr_lartg(double f, double g, double* out) { hr_lartg(f, g, out[0], out[1], out[2]); }

// The 1-norm estimator of DTGSEN's Dif (onenorm.h) on an explicit
// column-major n x n matrix M: the estimate of ||M||_1.
double host_onenorm_est(int n, const double* M) {
  auto apply = [&](int kind, std::vector<double>& x) {
    std::vector<double> y(n, 0.0);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        if (kind == 1) y[i] += M[i + (size_t)j * n] * x[j];
        else y[j] += M[i + (size_t)j * n] * x[i];
      }
    x = y;
    return true;
  };
  bool ok = true;
  return onenorm_est(n, apply, ok);
}

}  // extern "C"

