// C-ABI of the B200 multishift QZ: context, device backend of the QZ
// iteration, and the PDHGEQZ-compatible drop-in.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include <functional>

#include "../../include/b200qz.h"
#include "balance.h"
#include "hessred.h"
#include "reorder.h"
#include "kernels.h"
#include "ozaki.h"
#include "policy.h"
#include "qz_solver.h"

using namespace qz;

namespace {
constexpr int kAedMax = 512;  // largest AED / small-solve window supported
constexpr int64_t kUslot = (int64_t)kWinSmemMax * kWinSmemMax;  // one window's factor in Uc/Vc
constexpr int kTsSlots = 16;  // AED kernel profiling: stamps 0..4, counters 5..8
}

// Phase timer: CUDA event pairs recorded around each group of launches on
// the solver stream, resolved once at the end of a solve (B200QZ_PROFILE=1).
enum Phase { kPhScan, kPhAed, kPhAedUpd, kPhChase, kPhChaseUpd, kPhInf, kPhFinal, kPhN };

struct PhaseTimer {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  std::vector<std::pair<int, size_t>> marks;  // (phase, index of start event)
  double ms[kPhN] = {0};
  cudaEvent_t next() {
    if (used == pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[used++];
  }
  void begin(int ph, cudaStream_t st) {
    if (!on) return;
    marks.push_back({ph, used});
    cudaEventRecord(next(), st);
  }
  void end(cudaStream_t st) {
    if (!on) return;
    cudaEventRecord(next(), st);
  }
  void reset() {
    used = 0;
    marks.clear();
    for (double& v : ms) v = 0.0;
  }
  void resolve() {
    if (!on) return;
    for (auto& m : marks) {
      float t = 0.f;
      if (m.second + 1 < used && cudaEventElapsedTime(&t, pool[m.second], pool[m.second + 1]) == cudaSuccess)
        ms[m.first] += t;
    }
  }
  ~PhaseTimer() {
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
  }
};

// Everything the captured batched launch depends on: a replay is valid only
// while every field is unchanged.
struct BatchKey {
  // descriptors (order, n, queue counter, moff, eoff), then h, t, q, z,
  // alphar, alphai, beta, info
  const void* ptr[13] = {};
  int count = -1, threads = 0, smem_max = 0, ctas_per_sm = 0;
  bool operator==(const BatchKey& o) const {
    for (int i = 0; i < 13; ++i)
      if (ptr[i] != o.ptr[i]) return false;
    return count == o.count && threads == o.threads && smem_max == o.smem_max && ctas_per_sm == o.ctas_per_sm;
  }
};

// Tensor maps of the split-precision update, cached by matrix and box.
struct TmapEntry {
  const double* M;
  int64_t ld;
  int n, left, k;
  CUtensorMap map;
};

struct b200qz_ctx {
  int device = 0;
  std::vector<TmapEntry> tmaps;       // split-precision update: encoded tensor maps
  cudaStream_t stream = nullptr;
  double* Ua = nullptr;  // AED window factors (kAedMax^2)
  double* Va = nullptr;
  double* Uc = nullptr;  // chase / zero-chase window factors
  double* Vc = nullptr;
  double* shifts = nullptr;    // 3*kAedMax
  double* gscratch = nullptr;  // 2*kAedMax^2 (windows above the smem limit)
  // learned (nw, ns) policy: parameters, feature vector, activations, output
  float* pol = nullptr;        // kPolicyParams + kPolicyIn + 2*kPolicyHidden + kPolicyOut floats
  float* hpol_y = nullptr;     // pinned, kPolicyOut
  bool pol_on = false;
  // split-precision updates: prepared digits of up to kOzMaxFac factors
  uint8_t* ozb = nullptr;
  int* ozerr = nullptr;        // device flag: a tensor-core wait timed out
  double* norms = nullptr;     // 2
  double* npart = nullptr;     // 592 per-block partial sums of the norm kernel
  int* dinfo = nullptr;        // 16 ints: [4..6] AED info, [8..12] scan output
  int* hinfo = nullptr;        // pinned mirror
  double* hshifts = nullptr;   // pinned 3*kAedMax
  double* hnorms = nullptr;    // pinned 2
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  SolveParams params;
  SolveStats stats;
  double seconds = 0.0;
  int ka = 0;  // size of the AED factors in Ua/Va
  int kc = 0;  // size of the chase factors in Uc/Vc
  int hr_win = 128;  // pairs per window of the Hessenberg-triangular reduction
  cudaError_t err = cudaSuccess;
  PhaseTimer timer;
  unsigned long long* dts = nullptr;  // AED phase timestamps (device)
  double* dbuf = nullptr;             // cached device copy of H, T, Q, Z, eigenvalues (host entry)
  size_t dbuf_bytes = 0;
  // batched solver
  int* bdesc = nullptr;                // device: order, n, counter, moff/eoff (int64) packed
  size_t bdesc_bytes = 0;
  int batch_threads = 128, batch_smem_max = kBatchSmemMax, batch_ctas_per_sm = 1;
  cudaGraph_t bgraph = nullptr;
  cudaGraphExec_t bexec = nullptr;
  BatchKey bkey;                       // operands and configuration of the captured launch
  int sm_count = 148;
  double batch_seconds = 0.0;
  unsigned long long* hts = nullptr;  // pinned mirror
  double aed_ms[4] = {0, 0, 0, 0};   // small QZ, reorder, spike+RQ, HT re-reduction
  double aed_counts[4] = {0, 0, 0, 0};  // small-QZ steps, block swaps, re-reduction rotation pairs,
                                        // multishift window sweeps
};

namespace {

#define QZ_CK(x)                                 \
  do {                                           \
    cudaError_t e_ = (x);                        \
    if (e_ != cudaSuccess) {                     \
      if (c->err == cudaSuccess) c->err = e_;    \
    }                                            \
  } while (0)

// Device backend of qz_iterate (see qz_solver.h for the interface).
struct GpuBackend {
  b200qz_ctx* c;
  double *H, *T, *Q, *Z;
  int64_t ld;
  int n;
  bool wantq, wantz;
  // JOB = 'S': full Schur form.  JOB = 'E' (eigenvalues only): the far
  // updates of H and T stop at the active block [act_top, act_bot], the
  // role of ILSCHR = .FALSE. (PDHGEQZ.f:132-150; LAPACK DHGEQZ's
  // IFRSTM/ILASTM), while Q and Z still accumulate when asked for.
  bool schur = true;
  int act_top = 0, act_bot = 0;
  Tol tol;

  void active(int ktop, int kbot) {
    act_top = ktop;
    act_bot = kbot;
  }
  // columns right of a window (left updates) end at this column + 1, rows
  // above a window (right updates) start at this row
  int far_col_end() const { return schur ? n : act_bot + 1; }
  int far_row_begin() const { return schur ? 0 : act_top; }

  void scan(int ifirst, int kbot, int* out) {
    c->timer.begin(kPhScan, c->stream);
    launch_scan(c->stream, H, T, ld, ifirst, kbot, tol, c->dinfo + 8);
    c->stats.launches += 1;
    c->timer.end(c->stream);
    QZ_CK(cudaMemcpyAsync(c->hinfo, c->dinfo + 8, 5 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    QZ_CK(cudaStreamSynchronize(c->stream));
    if (c->err != cudaSuccess) { out[0] = ifirst; out[1] = 0; out[2] = -1; out[3] = -1; out[4] = 1; return; }
    for (int i = 0; i < 5; ++i) out[i] = c->hinfo[i];
  }
  // consecutive undeflatable blocks after which the spike test stops
  // (0: the whole window).  Automatic: the whole window for pencils of
  // order 6000 and more (measured: -34 % time to Schur at n = 10000 against
  // stopping after 4), 4 below (-16 % at n = 2000 against the whole window)
  int aed_early_stop(int nh) const {
    (void)nh;
    if (c->params.aed_nskip >= 0) return c->params.aed_nskip;
    return n >= 6000 ? 0 : 4;
  }
  void aed(int ktop, int kwtop, int kbot, int* info3, double* sh) {
    int nw = kbot - kwtop + 1;
    c->timer.begin(kPhAed, c->stream);
    launch_aed(c->stream, H, T, ld, ktop, kwtop, nw, tol, c->Ua, c->Va, c->shifts, c->dinfo + 4, c->gscratch,
               c->timer.on ? c->dts : nullptr, (kwtop > ktop) ? aed_early_stop(kbot - ktop + 1) : 0,
               c->params.aed_threads, c->params.aed_swap_fail, c->params.aed_ms);
    c->stats.launches += 1;
    c->stats.aed_launches += 1;
    c->stats.aed_bytes += 6.0 * 8.0 * nw * nw;
    c->timer.end(c->stream);
    QZ_CK(cudaMemcpyAsync(c->hinfo + 4, c->dinfo + 4, 3 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    QZ_CK(cudaMemcpyAsync(c->hshifts, c->shifts, 3 * nw * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (c->timer.on)
      QZ_CK(cudaMemcpyAsync(c->hts, c->dts, kTsSlots * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    QZ_CK(cudaStreamSynchronize(c->stream));
    c->ka = nw;
    if (c->timer.on) {
      // stamps 0..4: start, after small QZ, after reordering, after spike+RQ, end
      unsigned long long* t = c->hts;
      if (t[1] >= t[0]) c->aed_ms[0] += (t[1] - t[0]) * 1e-6;
      if (c->hinfo[5] == 0 && t[2] >= t[1]) c->aed_ms[1] += (t[2] - t[1]) * 1e-6;
      if (c->hinfo[5] == 0 && t[3] >= t[2] && t[4] >= t[3]) {
        c->aed_ms[2] += (t[3] - t[2]) * 1e-6;
        c->aed_ms[3] += (t[4] - t[3]) * 1e-6;
      }
      c->aed_counts[0] += (double)t[5];
      c->aed_counts[1] += (double)t[6];
      c->aed_counts[2] += (double)t[7];
      c->aed_counts[3] += (double)t[8];
      for (int i = 0; i < kTsSlots; ++i) t[i] = 0;
      QZ_CK(cudaMemsetAsync(c->dts, 0, kTsSlots * sizeof(unsigned long long), c->stream));
    }
    if (c->err != cudaSuccess) { info3[0] = nw; info3[1] = 1; info3[2] = 0; return; }
    info3[0] = c->hinfo[4];
    info3[1] = c->hinfo[5];
    info3[2] = c->hinfo[6];
    int m = std::min(info3[0], nw);
    for (int i = 0; i < m; ++i) {
      sh[i] = c->hshifts[i];
      sh[m + i] = c->hshifts[nw + i];
      sh[2 * m + i] = c->hshifts[2 * nw + i];
    }
    c->stats.win_bytes += 2.0 * 2.0 * 8.0 * nw * nw + 2.0 * 8.0 * nw * nw;
  }
  // one CTA per window of the wave; window i's factors go to slot i
  void chase_wave(const WinPlan* const* wins, int nw) {
    ChaseWave wave;
    for (int i = 0; i < nw; ++i) {
      const WinPlan& p = *wins[i];
      ChaseJob& J = wave.job[i];
      J.w0 = p.w; J.wk = p.wk; J.last = p.last; J.nb = p.nb; J.tmax = p.tmax;
      for (int b = 0; b < p.nb; ++b) J.bl[b] = p.bl[b];
      c->stats.win_bytes += 2.0 * 2.0 * 8.0 * p.wk * p.wk + 2.0 * 8.0 * p.wk * p.wk;
      c->stats.chase_bytes += 6.0 * 8.0 * p.wk * p.wk;
    }
    c->stats.chase_launches += 1;
    c->timer.begin(kPhChase, c->stream);
    launch_chase_wave(c->stream, H, T, ld, wave, nw, c->Uc, c->Vc, kUslot);
    c->timer.end(c->stream);
    c->stats.launches += 1;
    c->kc = kWinSmemMax;
  }
  void update_wave(const WinPlan* const* wins, int nw) {
    std::vector<int> w(nw), wk(nw);
    for (int i = 0; i < nw; ++i) { w[i] = wins[i]->w; wk[i] = wins[i]->wk; }
    update_list(w.data(), wk.data(), nw, c->Uc, c->Vc, kUslot, kPhChaseUpd);
  }
  void inf_window(int w, int wk, int top, int jz, int stop, bool deflate) {
    c->timer.begin(kPhInf, c->stream);
    launch_inf(c->stream, H, T, ld, w, wk, top, jz, stop, deflate ? 1 : 0, c->Uc, c->Vc);
    c->stats.launches += 1;
    c->timer.end(c->stream);
    c->kc = wk;
    c->stats.win_bytes += 2.0 * 2.0 * 8.0 * wk * wk + 2.0 * 8.0 * wk * wk;
  }
  // The same updates through the split-precision (INT8 Ozaki) tensor-core
  // kernels: digits of every factor prepared once, then one launch for the
  // left updates and one for the right updates.
  void update_list_split(const int* w, const int* wk, int nwin, const double* Ub, const double* Vb, int64_t ustride,
                         int phase) {
    OzPrep P;
    P.nfac = 0;
    P.out = c->ozb;
    OzBatch L, R;
    L.njobs = 0;
    R.njobs = 0;
    L.bslices = R.bslices = c->ozb;
    L.err = R.err = c->ozerr;
    // TMA tensor map of (M, side, k) in batch B: index, or -1 (plain loads)
    auto map_for = [&](OzBatch& B, int& nmaps, const double* (&mm)[kOzMaxMaps], int (&mk)[kOzMaxMaps],
                       int (&ml)[kOzMaxMaps], const double* M, int left, int k) -> int {
      for (int i = 0; i < nmaps; ++i)
        if (mm[i] == M && mk[i] == k && ml[i] == left) return i;
      if (nmaps == kOzMaxMaps) return -1;
      const TmapEntry* hit = nullptr;
      for (const TmapEntry& e : c->tmaps)
        if (e.M == M && e.ld == ld && e.n == n && e.left == left && e.k == k) { hit = &e; break; }
      if (!hit) {
        TmapEntry e{M, ld, n, left, k, {}};
        if (!ozaki_tensor_map(&e.map, M, ld, n, n, left, k)) return -1;
        if (c->tmaps.size() >= 64) c->tmaps.erase(c->tmaps.begin());
        c->tmaps.push_back(e);
        hit = &c->tmaps.back();
      }
      B.maps[nmaps] = hit->map;
      mm[nmaps] = M; mk[nmaps] = k; ml[nmaps] = left;
      return nmaps++;
    };
    int nmL = 0, nmR = 0;
    const double* mmL[kOzMaxMaps]; int mkL[kOzMaxMaps], mlL[kOzMaxMaps];
    const double* mmR[kOzMaxMaps]; int mkR[kOzMaxMaps], mlR[kOzMaxMaps];
    auto job = [&](OzBatch& B, double* M, int r0, int c0, int len, int k, int left, int fac) {
      OzJob& j = B.job[B.njobs++];
      j.M = M; j.ld = ld; j.r0 = r0; j.c0 = c0; j.len = len; j.k = k; j.left = left; j.fac = fac;
      j.tiles = (len + 127) / 128;
      j.map = (&B == &L) ? map_for(B, nmL, mmL, mkL, mlL, M, left, k) : map_for(B, nmR, mmR, mkR, mlR, M, left, k);
    };
    for (int i = 0; i < nwin; ++i) {
      const int k = wk[i], w0 = w[i];
      const int fu = P.nfac, fv = P.nfac + 1;
      P.W[fu] = Ub + i * ustride; P.ldw[fu] = k; P.k[fu] = k;
      P.W[fv] = Vb + i * ustride; P.ldw[fv] = k; P.k[fv] = k;
      P.nfac += 2;
      const int right_len = far_col_end() - (w0 + k);
      if (right_len > 0) {
        job(L, H, w0, w0 + k, right_len, k, 1, fu);
        job(L, T, w0, w0 + k, right_len, k, 1, fu);
        c->stats.upd_flops += 2.0 * 2.0 * k * k * right_len;
      }
      const int r0 = far_row_begin();
      if (w0 > r0) {
        job(R, H, r0, w0, w0 - r0, k, 0, fv);
        job(R, T, r0, w0, w0 - r0, k, 0, fv);
        c->stats.upd_flops += 2.0 * 2.0 * k * k * (w0 - r0);
      }
      if (wantq) { job(R, Q, 0, w0, n, k, 0, fu); c->stats.upd_flops += 2.0 * k * k * n; }
      if (wantz) { job(R, Z, 0, w0, n, k, 0, fv); c->stats.upd_flops += 2.0 * k * k * n; }
    }
    c->timer.begin(phase, c->stream);
    const int sl = c->params.split;
    launch_ozaki_prep(c->stream, P, sl);
    c->stats.launches += 1;
    if (L.njobs) { launch_ozaki_update(c->stream, L, sl); c->stats.launches += 1; }
    if (R.njobs) { launch_ozaki_update(c->stream, R, sl); c->stats.launches += 1; }
    c->timer.end(c->stream);
  }
  // Learned (nw, ns) for the AED decision on the active block [ktop, kbot]
  // (features of the subdiagonal profile, then the MLP, on the device).
  bool policy(int ktop, int kbot, double lastfrac, int* nw, int* ns) {
    if (!c->pol_on) return false;
    float* P = c->pol;
    float* X = P + kPolicyParams;
    float* A1 = X + kPolicyIn;
    float* A2 = A1 + kPolicyHidden;
    float* Y = A2 + kPolicyHidden;
    launch_policy_features(c->stream, H, ld, ktop, kbot, (float)lastfrac, X);
    launch_mlp_forward(c->stream, P, X, 1, A1, A2, Y);
    c->stats.launches += 2;
    QZ_CK(cudaMemcpyAsync(c->hpol_y, Y, kPolicyOut * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    QZ_CK(cudaStreamSynchronize(c->stream));
    if (c->err != cudaSuccess) return false;
    float y0 = c->hpol_y[0], y1 = c->hpol_y[1];
    if (!std::isfinite(y0) || !std::isfinite(y1)) return false;
    y0 = std::min(1.f, std::max(0.f, y0));
    y1 = std::min(1.f, std::max(0.f, y1));
    int w = (int)std::lround(kPolicyNwMin + y0 * kPolicyNwSpan);
    w = std::min(w, (int)kWinSmemMax);
    int s = (int)std::lround(y1 * w);
    s = std::max(2, s - s % 2);
    *nw = w;
    *ns = s;
    return true;
  }
  void inf_top(int f) {
    c->timer.begin(kPhInf, c->stream);
    launch_inf_top(c->stream, H, T, Q, ld, n, f, wantq ? 1 : 0);
    c->stats.launches += 1;
    c->timer.end(c->stream);
  }
  // off-diagonal updates with the factors of the last AED (which 0) or
  // zero-chase (which 1) window kernel
  void update(int w, int wk, int which) {
    if (which == 0) update_list(&w, &wk, 1, c->Ua, c->Va, 0, kPhAedUpd);
    else update_list(&w, &wk, 1, c->Uc, c->Vc, kUslot, kPhChaseUpd);
  }
  // Far updates of a list of disjoint windows (window i's factors at
  // U + i*ustride, V + i*ustride): one batched launch for every left
  // update (rows of a window, columns to its right), then one for every
  // right update (rows above a window, its columns; Q and Z columns).
  void update_list(const int* w, const int* wk, int nwin, const double* Ub, const double* Vb, int64_t ustride,
                   int phase) {
    bool split = c->params.split != 0 && nwin <= kOzMaxFac / 2;
    for (int i = 0; i < nwin && split; ++i)
      if (wk[i] > kOzMaxK) split = false;
    if (split) {
      update_list_split(w, wk, nwin, Ub, Vb, ustride, phase);
      return;
    }
    UpdBatch L, R;
    L.njobs = 0;
    R.njobs = 0;
    for (int i = 0; i < nwin; ++i) {
      const double* U = Ub + i * ustride;
      const double* V = Vb + i * ustride;
      int k = wk[i], w0 = w[i];
      int tile = update_tile(k);
      int right_len = far_col_end() - (w0 + k);
      if (right_len > 0) {
        for (double* M : {H, T}) {
          UpdJob& j = L.job[L.njobs++];
          j.M = M; j.ld = ld; j.r0 = w0; j.c0 = w0 + k; j.len = right_len; j.W = U; j.ldw = k; j.k = k;
          j.tiles = (right_len + tile - 1) / tile;
        }
        c->stats.upd_flops += 2.0 * 2.0 * k * k * right_len;
      }
      const int r0 = far_row_begin();
      if (w0 > r0) {
        for (double* M : {H, T}) {
          UpdJob& j = R.job[R.njobs++];
          j.M = M; j.ld = ld; j.r0 = r0; j.c0 = w0; j.len = w0 - r0; j.W = V; j.ldw = k; j.k = k;
          j.tiles = (w0 - r0 + tile - 1) / tile;
        }
        c->stats.upd_flops += 2.0 * 2.0 * k * k * (w0 - r0);
      }
      if (wantq) {
        UpdJob& j = R.job[R.njobs++];
        j.M = Q; j.ld = ld; j.r0 = 0; j.c0 = w0; j.len = n; j.W = U; j.ldw = k; j.k = k;
        j.tiles = (n + tile - 1) / tile;
        c->stats.upd_flops += 2.0 * k * k * n;
      }
      if (wantz) {
        UpdJob& j = R.job[R.njobs++];
        j.M = Z; j.ld = ld; j.r0 = 0; j.c0 = w0; j.len = n; j.W = V; j.ldw = k; j.k = k;
        j.tiles = (n + tile - 1) / tile;
        c->stats.upd_flops += 2.0 * k * k * n;
      }
    }
    c->timer.begin(phase, c->stream);
    if (L.njobs) { launch_update(c->stream, L, 0, c->params.upd_persist); c->stats.launches += 1; }
    if (R.njobs) { launch_update(c->stream, R, 1, c->params.upd_persist); c->stats.launches += 1; }
    c->timer.end(c->stream);
  }
};

bool is(char a, char b) { return std::toupper((unsigned char)a) == b; }

int check_args(char job, char compq, char compz, int n, int ilo, int ihi) {
  if (!is(job, 'E') && !is(job, 'S')) return -1;
  if (!is(compq, 'N') && !is(compq, 'V') && !is(compq, 'I')) return -2;
  if (!is(compz, 'N') && !is(compz, 'V') && !is(compz, 'I')) return -3;
  if (n < 0) return -4;
  if (ilo < 1) return -5;
  if (ihi > n || ihi < ilo - 1) return -6;
  return 0;
}

int solve_dev_impl(b200qz_ctx* c, char job, char compq, char compz, int n, int ilo, int ihi, double* h, double* t,
                   double* q, double* z, int ld, double* ar, double* ai, double* be) {
  c->stats = SolveStats();
  c->seconds = 0.0;
  c->err = cudaSuccess;
  {
    const char* v = std::getenv("B200QZ_VERBOSE");
    c->params.verbose = (v && *v && *v != '0') ? 1 : 0;
    const char* p = std::getenv("B200QZ_PROFILE");
    c->timer.on = (p && *p && *p != '0');
    c->timer.reset();
    for (double& a : c->aed_ms) a = 0.0;
    for (double& a : c->aed_counts) a = 0.0;
  }
  QZ_CK(cudaSetDevice(c->device));
  bool wantq = !is(compq, 'N'), wantz = !is(compz, 'N');
  if (is(compq, 'I')) { launch_identity(c->stream, q, ld, n); c->stats.launches += 1; }
  if (is(compz, 'I')) { launch_identity(c->stream, z, ld, n); c->stats.launches += 1; }
  QZ_CK(cudaEventRecord(c->ev0, c->stream));
  int nh = ihi - ilo + 1;
  // /PREC/ constants (PDHGEQZ.f:449-458): ulp, smlnum, Frobenius norms
  QZ_CK(cudaMemsetAsync(c->norms, 0, 2 * sizeof(double), c->stream));
  launch_sumsq(c->stream, h, ld, ilo - 1, nh, c->norms, c->npart);
  launch_sumsq(c->stream, t, ld, ilo - 1, nh, c->norms + 1, c->npart);
  c->stats.launches += 2;
  QZ_CK(cudaMemcpyAsync(c->hnorms, c->norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  QZ_CK(cudaStreamSynchronize(c->stream));
  if (c->err != cudaSuccess) return 10001;
  // T far from H in magnitude (or sums of squares out of range): balance T
  // by a power of two for the iteration, undone before the finalisation
  int ebal = 0;
  {
    const double hs = c->hnorms[0], ts = c->hnorms[1];
    const bool plain = hs > 1e-280 && hs < 1e280 && ts > 1e-280 && ts < 1e280 &&
                       std::fabs(0.5 * (std::log2(hs) - std::log2(ts))) <= 28.0;
    if (!plain && nh > 0) {
      launch_maxabs(c->stream, h, ld, ilo - 1, nh, c->norms, c->npart);
      launch_maxabs(c->stream, t, ld, ilo - 1, nh, c->norms + 1, c->npart);
      c->stats.launches += 4;
      QZ_CK(cudaMemcpyAsync(c->hnorms, c->norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      QZ_CK(cudaStreamSynchronize(c->stream));
      if (c->err != cudaSuccess) return 10001;
      ebal = balance_exponent(c->hnorms[0], c->hnorms[1]);
      if (ebal != 0) {
        launch_scale_pow2(c->stream, t, ld, n, ebal);
        c->stats.launches += 1;
      }
      launch_sumsq(c->stream, h, ld, ilo - 1, nh, c->norms, c->npart);
      launch_sumsq(c->stream, t, ld, ilo - 1, nh, c->norms + 1, c->npart);
      c->stats.launches += 4;
      QZ_CK(cudaMemcpyAsync(c->hnorms, c->norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      QZ_CK(cudaStreamSynchronize(c->stream));
      if (c->err != cudaSuccess) return 10001;
    }
  }
  GpuBackend bk;
  bk.c = c;
  bk.H = h; bk.T = t; bk.Q = q; bk.Z = z;
  bk.ld = ld;
  bk.n = n;
  bk.wantq = wantq;
  bk.wantz = wantz;
  bk.schur = is(job, 'S');
  bk.act_top = ilo - 1;
  bk.act_bot = ihi - 1;
  Tol& tol = bk.tol;
  tol.safmin = DBL_MIN;
  tol.ulp = DBL_EPSILON;
  tol.smlnum = DBL_MIN * ((double)nh / DBL_EPSILON);
  tol.htol = std::max(DBL_MIN, DBL_EPSILON * std::sqrt(c->hnorms[0]));
  tol.ttol = std::max(DBL_MIN, DBL_EPSILON * std::sqrt(c->hnorms[1]));
  int info = 0;
  if (nh > 0) info = qz_iterate(bk, n, ilo - 1, ihi - 1, c->params, c->stats);
  if (ebal != 0) {
    launch_scale_pow2(c->stream, t, ld, n, -ebal);
    c->stats.launches += 1;
  }
  const bool stopped = (info == -2);  // AED limit reached (tuning traces)
  if (stopped) info = 10003;
  else if (info < 0) info = 10002;  // non-finite entries appeared (or were given)
  if (!stopped) {
    c->timer.begin(kPhFinal, c->stream);
    launch_finalize(c->stream, h, t, z, ld, n, wantz ? 1 : 0, ar, ai, be);
    c->stats.launches += 2;
    c->timer.end(c->stream);
  }
  QZ_CK(cudaGetLastError());
  QZ_CK(cudaEventRecord(c->ev1, c->stream));
  QZ_CK(cudaEventSynchronize(c->ev1));
  c->timer.resolve();
  float ms = 0.f;
  QZ_CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->seconds = ms * 1e-3;
  if (c->err != cudaSuccess) return 10001;
  return info;
}

}  // namespace

extern "C" {

int b200qz_create(b200qz_ctx** out, int device) {
  if (!out) return -1;
  *out = nullptr;
  b200qz_ctx* c = new b200qz_ctx();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = kernels_init();
  if (e == cudaSuccess) e = batch_init();
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  size_t a2 = (size_t)kAedMax * kAedMax * sizeof(double);
  size_t w2 = (size_t)kMaxWave * kUslot * sizeof(double);
  if (e == cudaSuccess) e = cudaMalloc(&c->Ua, a2);
  if (e == cudaSuccess) e = cudaMalloc(&c->Va, a2);
  if (e == cudaSuccess) e = cudaMalloc(&c->Uc, w2);
  if (e == cudaSuccess) e = cudaMalloc(&c->Vc, w2);
  if (e == cudaSuccess) e = cudaMalloc(&c->shifts, 3 * kAedMax * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&c->gscratch, 2 * a2);
  if (e == cudaSuccess)
    e = cudaMalloc(&c->pol, (kPolicyParams + kPolicyIn + 2 * kPolicyHidden + kPolicyOut) * sizeof(float));
  if (e == cudaSuccess) e = cudaMallocHost(&c->hpol_y, kPolicyOut * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&c->ozb, kOzMaxFac * kOzFacBytes);
  if (e == cudaSuccess) e = cudaMalloc(&c->ozerr, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->ozerr, 0, sizeof(int));
  if (e == cudaSuccess) e = ozaki_init();
  if (e == cudaSuccess) e = cudaMalloc(&c->norms, 2 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&c->npart, 592 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&c->dinfo, 16 * sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost(&c->hinfo, 16 * sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost(&c->hshifts, 3 * kAedMax * sizeof(double));
  if (e == cudaSuccess) e = cudaMallocHost(&c->hnorms, 2 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&c->dts, kTsSlots * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(c->dts, 0, kTsSlots * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMallocHost(&c->hts, kTsSlots * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
  if (e != cudaSuccess) {
    b200qz_destroy(c);
    return (int)e;
  }
  *out = c;
  return 0;
}

void b200qz_destroy(b200qz_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->Ua); cudaFree(c->Va); cudaFree(c->Uc); cudaFree(c->Vc);
  if (c->pol) cudaFree(c->pol);
  if (c->ozb) cudaFree(c->ozb);
  if (c->ozerr) cudaFree(c->ozerr);
  if (c->hpol_y) cudaFreeHost(c->hpol_y);
  cudaFree(c->shifts); cudaFree(c->gscratch); cudaFree(c->norms); cudaFree(c->npart); cudaFree(c->dinfo);
  if (c->hinfo) cudaFreeHost(c->hinfo);
  if (c->hshifts) cudaFreeHost(c->hshifts);
  if (c->hnorms) cudaFreeHost(c->hnorms);
  cudaFree(c->dts);
  if (c->hts) cudaFreeHost(c->hts);
  if (c->dbuf) cudaFree(c->dbuf);
  if (c->bexec) cudaGraphExecDestroy(c->bexec);
  if (c->bgraph) cudaGraphDestroy(c->bgraph);
  if (c->bdesc) cudaFree(c->bdesc);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int b200qz_set_params(b200qz_ctx* c, int nw_max, int w_chase, int nmin, int nibble, int ns_max, int maxit_factor) {
  if (!c) return -1;
  if (nw_max > kWinSmemMax) return -2;
  if (w_chase > kWinSmemMax || (w_chase >= 0 && w_chase < 12)) return -3;
  if (nmin > kAedMax) return -4;
  if (nibble > 100) return -5;
  if (nw_max >= 0) c->params.nw_max = std::max(4, nw_max);
  if (w_chase >= 0) c->params.w_chase = w_chase;
  if (nmin >= 0) c->params.nmin = std::max(4, nmin);
  if (nibble >= 0) c->params.nibble = nibble;
  if (ns_max >= 0) c->params.ns_max = ns_max;
  if (maxit_factor >= 0) c->params.maxit_factor = std::max(1, maxit_factor);
  c->params.chain_max = std::min(kMaxChain, std::max(1, (c->params.w_chase - 4) / 6));
  return 0;
}

int b200qz_set_param(b200qz_ctx* c, const char* name, double value) {
  if (!c || !name) return -1;
  std::string k(name);
  int v = (int)value;
  SolveParams& P = c->params;
  if (k == "nw_max") { if (v < 4 || v > kWinSmemMax) return -3; P.nw_max = v; }
  else if (k == "w_chase") { if (v < 12 || v > kWinSmemMax) return -3; P.w_chase = v;
    P.chain_max = std::min(kMaxChain, std::max(1, (v - 4) / 6)); }
  else if (k == "nmin") { if (v < 4 || v > kAedMax) return -3; P.nmin = v; }
  else if (k == "nibble") { if (v < 0 || v > 100) return -3; P.nibble = v; }
  else if (k == "ns_max") { if (v < 0) return -3; P.ns_max = v; }
  else if (k == "maxit_factor") { if (v < 1) return -3; P.maxit_factor = v; }
  else if (k == "chain_max") { if (v < 1 || v > kMaxChain) return -3; P.chain_max = v; }
  else if (k == "aed_nskip") { if (v < -1) return -3; P.aed_nskip = v; }
  else if (k == "max_wave") { if (v < 1 || v > kMaxWave) return -3; P.max_wave = v; }
  else if (k == "stall_limit") { if (v < 1) return -3; P.stall_limit = v; }
  else if (k == "aed_limit") { P.aed_limit = v < 0 ? -1 : v; }
  else if (k == "upd_persist") { if (v != 0 && v != 1) return -3; P.upd_persist = v; }
  else if (k == "split") { if (v != 0 && v != 7 && v != 8) return -3; P.split = v; }
  else if (k == "aed_threads") { if (v != 32 && v != 64 && v != 128) return -3; P.aed_threads = v; }
  else if (k == "aed_swap_fail") { if (v != 0 && v != 1) return -3; P.aed_swap_fail = v; }
  else if (k == "aed_ms") { if (v != 0 && v != 1) return -3; P.aed_ms = v; }
  else if (k == "hr_win") { if (v < 2 || v > qz::kHrMaxWin) return -3; c->hr_win = v; }
  else return -2;
  return 0;
}

int b200qz_solve_dev(b200qz_ctx* c, char job, char compq, char compz, int n, int ilo, int ihi, double* h, double* t,
                     double* q, double* z, int ld, double* ar, double* ai, double* be) {
  if (!c) return 10001;
  int a = check_args(job, compq, compz, n, ilo, ihi);
  if (a != 0) return a;
  if (n == 0) return 0;
  if (ld < std::max(1, n)) return -(7 * 1000 + 9);
  return solve_dev_impl(c, job, compq, compz, n, ilo, ihi, h, t, q, z, ld, ar, ai, be);
}

int b200qz_solve_host(b200qz_ctx* c, char job, char compq, char compz, int n, int ilo, int ihi, double* h, int ldh,
                      double* t, int ldt, double* q, int ldq, double* z, int ldz, double* ar, double* ai,
                      double* be) {
  if (!c) return 10001;
  int a = check_args(job, compq, compz, n, ilo, ihi);
  if (a != 0) return a;
  if (n == 0) return 0;
  if (ldh < std::max(1, n)) return -(7 * 1000 + 9);
  if (ldt < std::max(1, n)) return -(9 * 1000 + 9);
  bool wantq = !is(compq, 'N'), wantz = !is(compz, 'N');
  if (wantq && ldq < std::max(1, n)) return -(14 * 1000 + 9);
  if (wantz && ldz < std::max(1, n)) return -(16 * 1000 + 9);
  c->err = cudaSuccess;
  QZ_CK(cudaSetDevice(c->device));
  int ldd = (n + 31) & ~31;
  size_t bytes = (size_t)ldd * n * sizeof(double);
  size_t need = 4 * bytes + 3 * (size_t)n * sizeof(double);
  if (c->dbuf_bytes < need) {
    if (c->dbuf) cudaFree(c->dbuf);
    c->dbuf = nullptr;
    c->dbuf_bytes = 0;
    QZ_CK(cudaMalloc(&c->dbuf, need));
    if (c->err == cudaSuccess) c->dbuf_bytes = need;
  }
  double* dh = c->dbuf;
  double* dt = dh + bytes / sizeof(double);
  double* dq = dt + bytes / sizeof(double);
  double* dz = dq + bytes / sizeof(double);
  double* de = dz + bytes / sizeof(double);
  int info = 10001;
  if (c->err == cudaSuccess) {
    size_t w = (size_t)n * sizeof(double);
    QZ_CK(cudaMemcpy2DAsync(dh, ldd * sizeof(double), h, (size_t)ldh * sizeof(double), w, n, cudaMemcpyHostToDevice, c->stream));
    QZ_CK(cudaMemcpy2DAsync(dt, ldd * sizeof(double), t, (size_t)ldt * sizeof(double), w, n, cudaMemcpyHostToDevice, c->stream));
    if (is(compq, 'V'))
      QZ_CK(cudaMemcpy2DAsync(dq, ldd * sizeof(double), q, (size_t)ldq * sizeof(double), w, n, cudaMemcpyHostToDevice, c->stream));
    if (is(compz, 'V'))
      QZ_CK(cudaMemcpy2DAsync(dz, ldd * sizeof(double), z, (size_t)ldz * sizeof(double), w, n, cudaMemcpyHostToDevice, c->stream));
    if (c->err == cudaSuccess) {
      info = solve_dev_impl(c, job, compq, compz, n, ilo, ihi, dh, dt, dq, dz, ldd, de, de + n, de + 2 * n);
      QZ_CK(cudaMemcpy2DAsync(h, (size_t)ldh * sizeof(double), dh, ldd * sizeof(double), w, n, cudaMemcpyDeviceToHost, c->stream));
      QZ_CK(cudaMemcpy2DAsync(t, (size_t)ldt * sizeof(double), dt, ldd * sizeof(double), w, n, cudaMemcpyDeviceToHost, c->stream));
      if (wantq)
        QZ_CK(cudaMemcpy2DAsync(q, (size_t)ldq * sizeof(double), dq, ldd * sizeof(double), w, n, cudaMemcpyDeviceToHost, c->stream));
      if (wantz)
        QZ_CK(cudaMemcpy2DAsync(z, (size_t)ldz * sizeof(double), dz, ldd * sizeof(double), w, n, cudaMemcpyDeviceToHost, c->stream));
      QZ_CK(cudaMemcpyAsync(ar, de, w, cudaMemcpyDeviceToHost, c->stream));
      QZ_CK(cudaMemcpyAsync(ai, de + n, w, cudaMemcpyDeviceToHost, c->stream));
      QZ_CK(cudaMemcpyAsync(be, de + 2 * n, w, cudaMemcpyDeviceToHost, c->stream));
      QZ_CK(cudaStreamSynchronize(c->stream));
    }
  }
  if (c->err != cudaSuccess) return 10001;
  return info;
}

int b200qz_get_stats(const b200qz_ctx* c, double* out, int nout) {
  if (!c || !out) return 0;
  const SolveStats& s = c->stats;
  const double* ph = c->timer.ms;
  double v[39] = {c->seconds, (double)s.iters, (double)s.aeds, (double)s.aed_defl, (double)s.sweeps,
                  (double)s.chains, (double)s.windows, (double)s.endgames, (double)s.infs, (double)s.shifts,
                  s.upd_flops, s.win_bytes,
                  ph[kPhScan], ph[kPhAed], ph[kPhAedUpd], ph[kPhChase], ph[kPhChaseUpd], ph[kPhInf], ph[kPhFinal],
                  c->aed_ms[0], c->aed_ms[1], c->aed_ms[2], c->aed_ms[3], (double)s.launches,
                  (double)s.aed_fail, (double)s.exceptional, (double)s.remaining, (double)s.stop_ktop,
                  (double)s.stop_kbot, s.last_frac, (double)s.policy_calls, s.aed_bytes,
                  (double)s.aed_launches, s.chase_bytes, (double)s.chase_launches, c->aed_counts[0],
                  c->aed_counts[1], c->aed_counts[2], c->aed_counts[3]};
  int k = std::min(nout, 39);
  for (int i = 0; i < k; ++i) out[i] = v[i];
  return k;
}

int b200qz_aed_window(b200qz_ctx* c, double* h, double* t, int ld, int ktop, int kwtop, int kbot, double* qw,
                      double* zw, double* shifts, int* info3) {
  if (!c) return 10001;
  int nw = kbot - kwtop + 1;
  if (nw < 1 || nw > kAedMax || ktop > kwtop || kwtop < 0) return -1;
  c->err = cudaSuccess;
  QZ_CK(cudaSetDevice(c->device));
  // norms of the whole leading (kbot+1) block give the tolerances
  int nh = kbot + 1;
  QZ_CK(cudaMemsetAsync(c->norms, 0, 2 * sizeof(double), c->stream));
  launch_sumsq(c->stream, h, ld, 0, nh, c->norms, c->npart);
  launch_sumsq(c->stream, t, ld, 0, nh, c->norms + 1, c->npart);
  QZ_CK(cudaMemcpyAsync(c->hnorms, c->norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  QZ_CK(cudaStreamSynchronize(c->stream));
  Tol tol;
  tol.safmin = DBL_MIN;
  tol.ulp = DBL_EPSILON;
  tol.smlnum = DBL_MIN * ((double)nh / DBL_EPSILON);
  tol.htol = std::max(DBL_MIN, DBL_EPSILON * std::sqrt(c->hnorms[0]));
  tol.ttol = std::max(DBL_MIN, DBL_EPSILON * std::sqrt(c->hnorms[1]));
  launch_aed(c->stream, h, t, ld, ktop, kwtop, nw, tol, qw, zw, shifts, c->dinfo + 4, c->gscratch);
  QZ_CK(cudaMemcpyAsync(c->hinfo + 4, c->dinfo + 4, 3 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  QZ_CK(cudaStreamSynchronize(c->stream));
  QZ_CK(cudaGetLastError());
  if (c->err != cudaSuccess) return 10001;
  for (int i = 0; i < 3; ++i) info3[i] = c->hinfo[4 + i];
  return 0;
}

int b200qz_chase_window(b200qz_ctx* c, double* h, double* t, int ld, int w, int wk, int last, const int* bulges,
                        const double* coef, int nb, int tmax, double* u, double* v) {
  if (!c) return 10001;
  if (wk < 4 || wk > kWinSmemMax || nb < 1 || nb > kMaxChain || last >= wk) return -1;
  c->err = cudaSuccess;
  QZ_CK(cudaSetDevice(c->device));
  ChaseWave wave;
  ChaseJob& J = wave.job[0];
  J.w0 = w; J.wk = wk; J.last = last; J.nb = nb; J.tmax = tmax;
  for (int b = 0; b < nb; ++b) {
    J.bl[b].base = bulges[4 * b];
    J.bl[b].tlo = bulges[4 * b + 1];
    J.bl[b].thi = bulges[4 * b + 2];
    J.bl[b].intro = bulges[4 * b + 3];
    J.bl[b].c2 = coef[3 * b];
    J.bl[b].c1 = coef[3 * b + 1];
    J.bl[b].c0 = coef[3 * b + 2];
  }
  launch_chase_wave(c->stream, h, t, ld, wave, 1, u, v, 0);
  QZ_CK(cudaGetLastError());
  QZ_CK(cudaStreamSynchronize(c->stream));
  return c->err == cudaSuccess ? 0 : 10001;
}

int b200qz_update(b200qz_ctx* c, char side, double* m, int ldm, int r0, int c0, int len, const double* w, int ldw,
                  int k) {
  if (!c) return 10001;
  if (k < 1 || k > kAedMax || len < 0) return -1;
  c->err = cudaSuccess;
  QZ_CK(cudaSetDevice(c->device));
  UpdBatch B;
  B.k = k;
  B.njobs = 1;
  UpdJob& j = B.job[0];
  j.M = m; j.ld = ldm; j.r0 = r0; j.c0 = c0; j.len = len; j.W = w; j.ldw = ldw; j.k = k;
  int tile = update_tile(k);
  j.tiles = (len + tile - 1) / tile;
  if (is(side, 'L')) launch_update(c->stream, B, 0);
  else if (is(side, 'R')) launch_update(c->stream, B, 1);
  else return -2;
  QZ_CK(cudaGetLastError());
  QZ_CK(cudaStreamSynchronize(c->stream));
  return c->err == cudaSuccess ? 0 : 10001;
}

int b200qz_update_split(b200qz_ctx* c, char side, double* m, int ldm, int r0, int c0, int len, const double* w,
                        int ldw, int k, int slices) {
  if (!c) return 10001;
  if (k < 1 || k > kOzMaxK || len < 0 || (slices != 7 && slices != 8)) return -1;
  if (!is(side, 'L') && !is(side, 'R')) return -2;
  c->err = cudaSuccess;
  QZ_CK(cudaSetDevice(c->device));
  OzPrep P;
  P.nfac = 1; P.W[0] = w; P.ldw[0] = ldw; P.k[0] = k; P.out = c->ozb;
  OzBatch B;
  B.njobs = 1; B.bslices = c->ozb; B.err = c->ozerr;
  OzJob& j = B.job[0];
  j.M = m; j.ld = ldm; j.r0 = r0; j.c0 = c0; j.len = len; j.k = k; j.left = is(side, 'L') ? 1 : 0; j.fac = 0;
  j.tiles = (len + 127) / 128;
  // the slab as a TMA tensor map when its leading dimension allows
  j.map = -1;
  {
    // the map spans exactly the slab's rows and columns from the origin
    const int rows = r0 + (j.left ? k : len), cols = c0 + (j.left ? len : k);
    if (rows <= ldm && ozaki_tensor_map(&B.maps[0], m, ldm, rows, cols, j.left, k)) j.map = 0;
  }
  launch_ozaki_prep(c->stream, P, slices);
  launch_ozaki_update(c->stream, B, slices);
  QZ_CK(cudaGetLastError());
  int herr = 0;
  QZ_CK(cudaMemcpyAsync(&herr, c->ozerr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  QZ_CK(cudaStreamSynchronize(c->stream));
  if (c->err != cudaSuccess) return 10001;
  return herr ? 10004 : 0;
}

// ---------------------------------------------------------------------------
// Batched pencils
// ---------------------------------------------------------------------------
namespace {

// order: pencils by decreasing size (longest first on the work queue)
int batch_prepare(b200qz_ctx* c, int count, const int* n, const long long* moff, const long long* eoff, int** d_order,
                  int** d_n, int** d_counter, int64_t** d_moff, int64_t** d_eoff) {
  size_t need = (size_t)count * (2 * sizeof(int) + 2 * sizeof(int64_t)) + 64;
  if (c->bdesc_bytes < need) {
    if (c->bdesc) cudaFree(c->bdesc);
    c->bdesc = nullptr;
    c->bdesc_bytes = 0;
    if (cudaMalloc(&c->bdesc, need) != cudaSuccess) return 10001;
    c->bdesc_bytes = need;
  }
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[a] > n[b]; });
  char* base = (char*)c->bdesc;
  *d_moff = (int64_t*)base;
  *d_eoff = (int64_t*)(base + (size_t)count * sizeof(int64_t));
  *d_order = (int*)(base + 2 * (size_t)count * sizeof(int64_t));
  *d_n = *d_order + count;
  *d_counter = *d_n + count;
  QZ_CK(cudaMemcpyAsync(*d_moff, (const int64_t*)moff, count * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
  QZ_CK(cudaMemcpyAsync(*d_eoff, (const int64_t*)eoff, count * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
  QZ_CK(cudaMemcpyAsync(*d_order, order.data(), count * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  QZ_CK(cudaMemcpyAsync(*d_n, n, count * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  QZ_CK(cudaStreamSynchronize(c->stream));
  return c->err == cudaSuccess ? 0 : 10001;
}

int batch_grid(const b200qz_ctx* c) { return std::max(1, c->sm_count * c->batch_ctas_per_sm); }

}  // namespace

extern "C" int b200qz_solve_batched_dev(b200qz_ctx* c, int count, const int* n, const long long* moff,
                                        const long long* eoff, double* h, double* t, double* q, double* z,
                                        double* alphar, double* alphai, double* beta, int* info) {
  if (!c) return 10001;
  if (count < 0) return -2;
  for (int i = 0; i < count; ++i)
    if (n[i] < 1 || n[i] > 46340) return -(3 * 1000 + 1);
  if (count == 0) return 0;
  c->err = cudaSuccess;
  QZ_CK(cudaSetDevice(c->device));
  int *d_order, *d_n, *d_counter;
  int64_t *d_moff, *d_eoff;
  if (batch_prepare(c, count, n, moff, eoff, &d_order, &d_n, &d_counter, &d_moff, &d_eoff) != 0) return 10001;
  // one persistent launch, captured in a CUDA graph and replayed while
  // every operand pointer, the count and the configuration stay the same
  BatchKey key;
  const void* ops[13] = {d_order, d_n, d_counter, d_moff, d_eoff, h, t, q, z, alphar, alphai, beta, info};
  for (int i = 0; i < 13; ++i) key.ptr[i] = ops[i];
  key.count = count;
  key.threads = c->batch_threads;
  key.smem_max = c->batch_smem_max;
  key.ctas_per_sm = c->batch_ctas_per_sm;
  if (!c->bexec || !(key == c->bkey)) {
    if (c->bexec) { cudaGraphExecDestroy(c->bexec); c->bexec = nullptr; }
    if (c->bgraph) { cudaGraphDestroy(c->bgraph); c->bgraph = nullptr; }
    QZ_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    launch_batch(c->stream, batch_grid(c), c->batch_threads, c->batch_smem_max, count, d_order, d_n, d_moff, d_eoff,
                 h, t, q, z, alphar, alphai, beta, info, d_counter);
    QZ_CK(cudaStreamEndCapture(c->stream, &c->bgraph));
    if (c->err == cudaSuccess) QZ_CK(cudaGraphInstantiate(&c->bexec, c->bgraph, 0));
    if (c->err != cudaSuccess) return 10001;
    c->bkey = key;
  }
  QZ_CK(cudaEventRecord(c->ev0, c->stream));
  QZ_CK(cudaGraphLaunch(c->bexec, c->stream));
  QZ_CK(cudaEventRecord(c->ev1, c->stream));
  QZ_CK(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  QZ_CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->batch_seconds = ms * 1e-3;
  return c->err == cudaSuccess ? 0 : 10001;
}

extern "C" double b200qz_batched_seconds(const b200qz_ctx* c) { return c ? c->batch_seconds : 0.0; }

// Autotuner: time every configuration (threads per CTA, largest pencil kept
// in shared memory, CTAs per SM) on a copy of a sample of the batch and keep
// the fastest.  The caller's arrays are not modified.
extern "C" int b200qz_batched_autotune(b200qz_ctx* c, int count, const int* n, const long long* moff,
                                       const double* h, const double* t, int sample, double* best_seconds) {
  if (!c || count <= 0) return -1;
  c->err = cudaSuccess;
  QZ_CK(cudaSetDevice(c->device));
  // deterministic sample spread over the size range
  int k = std::min(count, std::max(1, sample));
  std::vector<int> idx(count);
  for (int i = 0; i < count; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return n[a] > n[b]; });
  std::vector<int> pick, sn;
  std::vector<long long> so, se;
  int64_t off = 0, eo = 0;
  for (int j = 0; j < k; ++j) {
    int p = idx[(int64_t)j * count / k];
    pick.push_back(p);
    sn.push_back(n[p]);
    so.push_back(off);
    se.push_back(eo);
    off += (int64_t)n[p] * n[p];
    eo += n[p];
  }
  double *bh = nullptr, *bt = nullptr, *bq = nullptr, *bz = nullptr, *bs = nullptr, *be = nullptr;
  int* bi = nullptr;
  QZ_CK(cudaMalloc(&bh, off * sizeof(double)));
  QZ_CK(cudaMalloc(&bt, off * sizeof(double)));
  QZ_CK(cudaMalloc(&bq, off * sizeof(double)));
  QZ_CK(cudaMalloc(&bz, off * sizeof(double)));
  QZ_CK(cudaMalloc(&bs, off * 2 * sizeof(double)));
  QZ_CK(cudaMalloc(&be, eo * 3 * sizeof(double)));
  QZ_CK(cudaMalloc(&bi, k * sizeof(int)));
  if (c->err != cudaSuccess) return 10001;
  for (int j = 0; j < k; ++j) {
    size_t bytes = (size_t)sn[j] * sn[j] * sizeof(double);
    QZ_CK(cudaMemcpyAsync(bs + so[j], h + moff[pick[j]], bytes, cudaMemcpyDeviceToDevice, c->stream));
    QZ_CK(cudaMemcpyAsync(bs + off + so[j], t + moff[pick[j]], bytes, cudaMemcpyDeviceToDevice, c->stream));
  }
  const int threads[2] = {128, 256};
  const int smems[4] = {0, 48, 64, kBatchSmemMax};
  double best = 1e300;
  int bt_ = c->batch_threads, bs_ = c->batch_smem_max, bc_ = c->batch_ctas_per_sm;
  for (int th : threads)
    for (int sm : smems)
      for (int cps = 1; cps <= 4; cps *= 2) {
        size_t smem = batch_smem_bytes(sm);
        if (smem * cps > 220 * 1024) continue;
        c->batch_threads = th;
        c->batch_smem_max = sm;
        c->batch_ctas_per_sm = cps;
        QZ_CK(cudaMemcpyAsync(bh, bs, off * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        QZ_CK(cudaMemcpyAsync(bt, bs + off, off * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        int rc = b200qz_solve_batched_dev(c, k, sn.data(), so.data(), se.data(), bh, bt, bq, bz, be, be + eo,
                                          be + 2 * eo, bi);
        if (rc != 0) continue;
        if (c->batch_seconds < best) {
          best = c->batch_seconds;
          bt_ = th; bs_ = sm; bc_ = cps;
        }
      }
  c->batch_threads = bt_;
  c->batch_smem_max = bs_;
  c->batch_ctas_per_sm = bc_;
  if (c->bexec) { cudaGraphExecDestroy(c->bexec); c->bexec = nullptr; }
  if (c->bgraph) { cudaGraphDestroy(c->bgraph); c->bgraph = nullptr; }
  cudaFree(bh); cudaFree(bt); cudaFree(bq); cudaFree(bz); cudaFree(bs); cudaFree(be); cudaFree(bi);
  if (best_seconds) *best_seconds = best;
  return c->err == cudaSuccess ? 0 : 10001;
}

extern "C" int b200qz_batched_config(const b200qz_ctx* c, int* threads, int* smem_max, int* ctas_per_sm) {
  if (!c) return -1;
  if (threads) *threads = c->batch_threads;
  if (smem_max) *smem_max = c->batch_smem_max;
  if (ctas_per_sm) *ctas_per_sm = c->batch_ctas_per_sm;
  return 0;
}

// ---------------------------------------------------------------------------
// Learned (nw, ns) policy
// ---------------------------------------------------------------------------
extern "C" int b200qz_policy_nparams(void) { return kPolicyParams; }

extern "C" int b200qz_set_policy(b200qz_ctx* c, const float* params, int nparams) {
  if (!c) return 10001;
  if (nparams == 0 || params == nullptr) {
    c->pol_on = false;
    return 0;
  }
  if (nparams != kPolicyParams) return -3;
  for (int i = 0; i < nparams; ++i)
    if (!std::isfinite(params[i])) return -2;
  c->err = cudaSuccess;
  QZ_CK(cudaSetDevice(c->device));
  QZ_CK(cudaMemcpy(c->pol, params, kPolicyParams * sizeof(float), cudaMemcpyHostToDevice));
  if (c->err != cudaSuccess) return 10001;
  c->pol_on = true;
  return 0;
}

extern "C" int b200qz_policy_features(b200qz_ctx* c, const double* h, int ld, int ktop, int kbot, double lastfrac,
                                      float* out) {
  if (!c || !out) return 10001;
  if (ktop < 0 || kbot <= ktop || ld < kbot + 1) return -1;
  c->err = cudaSuccess;
  QZ_CK(cudaSetDevice(c->device));
  float* X = c->pol + kPolicyParams;
  launch_policy_features(c->stream, h, ld, ktop, kbot, (float)lastfrac, X);
  QZ_CK(cudaMemcpyAsync(out, X, kPolicyIn * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  QZ_CK(cudaStreamSynchronize(c->stream));
  return c->err == cudaSuccess ? 0 : 10001;
}

extern "C" int b200qz_mlp_forward(const float* params, const float* x, int batch, float* a1, float* a2, float* y,
                                  void* stream) {
  if (batch < 0) return -1;
  launch_mlp_forward((cudaStream_t)stream, params, x, batch, a1, a2, y);
  return cudaGetLastError() == cudaSuccess ? 0 : 10001;
}

extern "C" int b200qz_mlp_backward(const float* params, const float* x, const float* target, int batch,
                                   const float* a1, const float* a2, const float* y, float* dy, float* d2,
                                   float* d1, float* grad, void* stream) {
  if (batch < 0) return -1;
  launch_mlp_backward((cudaStream_t)stream, params, x, target, batch, a1, a2, y, dy, d2, d1, grad);
  return cudaGetLastError() == cudaSuccess ? 0 : 10001;
}

extern "C" int b200qz_mlp_train(float* params, const float* x, const float* target, int batch, int epochs, float lr,
                                float* loss) {
  if (batch < 1 || epochs < 0) return -1;
  cudaStream_t st = nullptr;
  size_t nf = (size_t)batch * (2 * kPolicyHidden + kPolicyHidden * 2 + 2 * kPolicyOut) + 3 * kPolicyParams + 1;
  float* w = nullptr;
  if (cudaMalloc(&w, nf * sizeof(float)) != cudaSuccess) return 10001;
  float* A1 = w;
  float* A2 = A1 + (size_t)batch * kPolicyHidden;
  float* D1 = A2 + (size_t)batch * kPolicyHidden;
  float* D2 = D1 + (size_t)batch * kPolicyHidden;
  float* Y = D2 + (size_t)batch * kPolicyHidden;
  float* DY = Y + (size_t)batch * kPolicyOut;
  float* G = DY + (size_t)batch * kPolicyOut;
  float* M = G + kPolicyParams;
  float* V = M + kPolicyParams;
  float* L = V + kPolicyParams;
  cudaMemsetAsync(M, 0, 2 * kPolicyParams * sizeof(float), st);
  for (int e = 1; e <= epochs; ++e) {
    launch_mlp_forward(st, params, x, batch, A1, A2, Y);
    launch_mlp_backward(st, params, x, target, batch, A1, A2, Y, DY, D2, D1, G);
    launch_adam(st, params, G, M, V, lr, e);
  }
  launch_mlp_forward(st, params, x, batch, A1, A2, Y);
  launch_mse(st, Y, target, batch * kPolicyOut, L);
  float hl = 0.f;
  cudaError_t err = cudaMemcpy(&hl, L, sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(w);
  if (loss) *loss = hl;
  return err == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 10001;
}

// ---------------------------------------------------------------------------
// Fortran drop-in
// ---------------------------------------------------------------------------
static std::mutex g_mu;
static b200qz_ctx* g_ctx = nullptr;

void kkqzconf_(const double* eps) { (void)eps; }

void pdhgeqz_(const char* job, const char* compq, const char* compz, const int* n, const int* ilo, const int* ihi,
              double* h, const int* desch, double* t, const int* desct, double* alphar, double* alphai,
              double* beta, double* q, const int* descq, double* z, const int* descz, double* dwork,
              const int* ldwork, int* iwork, const int* liwork, int* info, size_t len_job, size_t len_compq,
              size_t len_compz) {
  (void)len_job; (void)len_compq; (void)len_compz;
  const int N = *n, ILO = *ilo, IHI = *ihi;
  // quick return (PDHGEQZ.f:320-323)
  if (N <= 0 || IHI < ILO) { *info = 0; return; }
  // descriptor fields (1-based in Fortran): MB_=5, NB_=6, LLD_=9
  int a = check_args(*job, *compq, *compz, N, ILO, IHI);
  if (a == 0 && desch[5] < 5) a = -7;
  if (a == 0 && desch[5] != desch[4]) a = -8;
  if (a != 0) { *info = a; return; }
  int nb = desch[5];
  // workspace (same order as PDHGEQZ1.f:369-372)
  int ldwmin = std::max(1, N * nb), liwmin = std::max(1, 2 * N);
  if (*ldwork == -1 || *liwork == -1) {
    dwork[0] = (double)ldwmin;
    iwork[0] = liwmin;
    *info = 0;
    return;
  }
  if (*ldwork < ldwmin) { *info = -9; return; }
  if (*liwork < liwmin) { *info = -10; return; }
  int ldh = desch[8], ldt = desct[8], ldq = descq[8], ldz = descz[8];
  // ALPHAR/ALPHAI/BETA(ILO:IHI) = -1 on entry (PDHGEQZ.f:469-471)
  for (int i = ILO - 1; i < IHI; ++i) { alphar[i] = -1.0; alphai[i] = -1.0; beta[i] = -1.0; }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ctx) {
    int dev = 0;
    const char* e = std::getenv("B200QZ_DEVICE");
    if (e) dev = std::atoi(e);
    if (b200qz_create(&g_ctx, dev) != 0) { g_ctx = nullptr; *info = 10001; return; }
  }
  *info = b200qz_solve_host(g_ctx, *job, *compq, *compz, N, ILO, IHI, h, ldh, t, ldt, q, ldq, z, ldz, alphar,
                            alphai, beta);
}

// ---------------------------------------------------------------------------
// Balancing (DGGBAL / DGGBAK semantics) on device or host arrays.
// ---------------------------------------------------------------------------
static int ggbal_args(char job, int n, int lda, int ldb) {
  if (!is(job, 'N') && !is(job, 'P') && !is(job, 'S') && !is(job, 'B')) return -1;
  if (n < 0) return -2;
  if (lda < std::max(1, n)) return -4;
  if (ldb < std::max(1, n)) return -6;
  return 0;
}

int b200qz_ggbal_dev(b200qz_ctx* c, char job, int n, double* a, int lda, double* b, int ldb, int* ilo, int* ihi,
                     double* lscale, double* rscale) {
  if (!c) return 10001;
  const int bad = ggbal_args(job, n, lda, ldb);
  if (bad) return bad;
  if (cudaSetDevice(c->device) != cudaSuccess) return 10001;
  return qz::ggbal_device(c->stream, job, n, a, lda, b, ldb, ilo, ihi, lscale, rscale) == cudaSuccess ? 0 : 10001;
}

int b200qz_ggbal_host(b200qz_ctx* c, char job, int n, double* a, int lda, double* b, int ldb, int* ilo, int* ihi,
                      double* lscale, double* rscale) {
  if (!c) return 10001;
  const int bad = ggbal_args(job, n, lda, ldb);
  if (bad) return bad;
  if (n == 0) { *ilo = 1; *ihi = 0; return 0; }
  if (cudaSetDevice(c->device) != cudaSuccess) return 10001;
  double* d = nullptr;
  const size_t nn = (size_t)n * n;
  if (cudaMalloc(&d, 2 * nn * sizeof(double)) != cudaSuccess) return 10001;
  cudaError_t e = cudaMemcpy2DAsync(d, n * sizeof(double), a, (size_t)lda * sizeof(double), n * sizeof(double), n,
                                    cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(d + nn, n * sizeof(double), b, (size_t)ldb * sizeof(double), n * sizeof(double), n,
                          cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = qz::ggbal_device(c->stream, job, n, d, n, d + nn, n, ilo, ihi, lscale, rscale);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(a, (size_t)lda * sizeof(double), d, n * sizeof(double), n * sizeof(double), n,
                          cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(b, (size_t)ldb * sizeof(double), d + nn, n * sizeof(double), n * sizeof(double), n,
                          cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  return e == cudaSuccess ? 0 : 10001;
}

static int ggbak_args(char job, char side, int n, int ilo, int ihi, int m, int ldv) {
  if (!is(job, 'N') && !is(job, 'P') && !is(job, 'S') && !is(job, 'B')) return -1;
  if (!is(side, 'L') && !is(side, 'R')) return -2;
  if (n < 0) return -3;
  if (n > 0 ? (ilo < 1 || ilo > n) : ilo != 1) return -4;
  if (n > 0 ? (ihi < ilo || ihi > n) : ihi != 0) return -5;
  if (m < 0) return -8;
  if (ldv < std::max(1, n)) return -10;
  return 0;
}

int b200qz_ggbak_dev(b200qz_ctx* c, char job, char side, int n, int ilo, int ihi, const double* lscale,
                     const double* rscale, int m, double* v, int ldv) {
  if (!c) return 10001;
  const int bad = ggbak_args(job, side, n, ilo, ihi, m, ldv);
  if (bad) return bad;
  if (cudaSetDevice(c->device) != cudaSuccess) return 10001;
  return qz::ggbak_device(c->stream, job, side, n, ilo, ihi, lscale, rscale, m, v, ldv) == cudaSuccess ? 0 : 10001;
}

int b200qz_ggbak_host(b200qz_ctx* c, char job, char side, int n, int ilo, int ihi, const double* lscale,
                      const double* rscale, int m, double* v, int ldv) {
  if (!c) return 10001;
  const int bad = ggbak_args(job, side, n, ilo, ihi, m, ldv);
  if (bad) return bad;
  if (n == 0 || m == 0) return 0;
  if (cudaSetDevice(c->device) != cudaSuccess) return 10001;
  double* d = nullptr;
  if (cudaMalloc(&d, (size_t)n * m * sizeof(double)) != cudaSuccess) return 10001;
  cudaError_t e = cudaMemcpy2DAsync(d, n * sizeof(double), v, (size_t)ldv * sizeof(double), n * sizeof(double), m,
                                    cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = qz::ggbak_device(c->stream, job, side, n, ilo, ihi, lscale, rscale, m, d, n);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(v, (size_t)ldv * sizeof(double), d, n * sizeof(double), n * sizeof(double), m,
                          cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  return e == cudaSuccess ? 0 : 10001;
}

// ---------------------------------------------------------------------------
// Reordering of a generalized Schur form (DTGSEN semantics, IJOB 0 and 1).
// ---------------------------------------------------------------------------
static int tgsen_args(int ijob, int wantq, int wantz, int n, int lds, int ldt, int ldq, int ldz) {
  if (ijob != 0 && ijob != 1 && ijob != 3 && ijob != 5) return -1;
  if (n < 0) return -5;
  if (lds < std::max(1, n)) return -7;
  if (ldt < std::max(1, n)) return -9;
  if (ldq < 1 || (wantq && ldq < n)) return -14;
  if (ldz < 1 || (wantz && ldz < n)) return -16;
  return 0;
}

int b200qz_tgsen_dev(b200qz_ctx* c, int ijob, int wantq, int wantz, const int* select, int n, double* s, int lds,
                     double* t, int ldt, double* q, int ldq, double* z, int ldz, double* alphar, double* alphai,
                     double* beta, int* m, double* pl, double* pr, double* dif, int* info, int* counts) {
  if (!c) return 10001;
  const int bad = tgsen_args(ijob, wantq, wantz, n, lds, ldt, ldq, ldz);
  if (bad) return bad;
  if (cudaSetDevice(c->device) != cudaSuccess) return 10001;
  qz::ReorderOut o;
  const cudaError_t e = qz::tgsen_device(c->stream, ijob, wantq != 0, wantz != 0, select, n, s, lds, t, ldt, q, ldq,
                                         z, ldz, alphar, alphai, beta, &o);
  if (e != cudaSuccess) return 10001;
  *m = o.m;
  *pl = o.pl;
  *pr = o.pr;
  if (dif && (ijob == 3 || ijob == 5)) { dif[0] = o.dif[0]; dif[1] = o.dif[1]; }
  *info = o.info;
  if (counts) { counts[0] = o.swaps; counts[1] = o.windows; }
  return 0;
}

int b200qz_tgsen_host(b200qz_ctx* c, int ijob, int wantq, int wantz, const int* select, int n, double* s, int lds,
                      double* t, int ldt, double* q, int ldq, double* z, int ldz, double* alphar, double* alphai,
                      double* beta, int* m, double* pl, double* pr, double* dif, int* info) {
  if (!c) return 10001;
  const int bad = tgsen_args(ijob, wantq, wantz, n, lds, ldt, ldq, ldz);
  if (bad) return bad;
  if (n == 0) {
    *m = 0; *pl = *pr = 1.0; *info = 0;
    if (dif && (ijob == 3 || ijob == 5)) dif[0] = dif[1] = 0.0;
    return 0;
  }
  if (cudaSetDevice(c->device) != cudaSuccess) return 10001;
  const size_t nn = (size_t)n * n;
  double* d = nullptr;
  if (cudaMalloc(&d, (4 * nn + 3 * (size_t)n) * sizeof(double)) != cudaSuccess) return 10001;
  double *ds = d, *dt = d + nn, *dq = d + 2 * nn, *dz = d + 3 * nn, *de = d + 4 * nn;
  const size_t w = n * sizeof(double);
  cudaError_t e = cudaMemcpy2DAsync(ds, w, s, (size_t)lds * sizeof(double), w, n, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(dt, w, t, (size_t)ldt * sizeof(double), w, n, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && wantq)
    e = cudaMemcpy2DAsync(dq, w, q, (size_t)ldq * sizeof(double), w, n, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && wantz)
    e = cudaMemcpy2DAsync(dz, w, z, (size_t)ldz * sizeof(double), w, n, cudaMemcpyHostToDevice, c->stream);
  qz::ReorderOut o;
  if (e == cudaSuccess)
    e = qz::tgsen_device(c->stream, ijob, wantq != 0, wantz != 0, select, n, ds, n, dt, n, dq, n, dz, n, de, de + n,
                         de + 2 * n, &o);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(s, (size_t)lds * sizeof(double), ds, w, w, n, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(t, (size_t)ldt * sizeof(double), dt, w, w, n, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && wantq)
    e = cudaMemcpy2DAsync(q, (size_t)ldq * sizeof(double), dq, w, w, n, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && wantz)
    e = cudaMemcpy2DAsync(z, (size_t)ldz * sizeof(double), dz, w, w, n, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(alphar, de, w, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(alphai, de + n, w, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(beta, de + 2 * n, w, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  if (e != cudaSuccess) return 10001;
  *m = o.m;
  *pl = o.pl;
  *pr = o.pr;
  if (dif && (ijob == 3 || ijob == 5)) { dif[0] = o.dif[0]; dif[1] = o.dif[1]; }
  *info = o.info;
  return 0;
}

// ---------------------------------------------------------------------------
// Hessenberg-triangular reduction (DGGHRD semantics; the reference's
// PDGGHRD, src/ab2ht/PDGGHRD.f:13).
// ---------------------------------------------------------------------------
static int comp_code(char c) { return is(c, 'N') ? 0 : is(c, 'V') ? 1 : is(c, 'I') ? 2 : -1; }

// Argument numbering of DGGHRD: COMPQ 1, COMPZ 2, N 3, ILO 4, IHI 5, LDA 7,
// LDB 9, LDQ 11, LDZ 13.
static int gghrd_args(char compq, char compz, int n, int ilo, int ihi, int lda, int ldb, int ldq, int ldz) {
  const int cq = comp_code(compq), cz = comp_code(compz);
  if (cq < 0) return -1;
  if (cz < 0) return -2;
  if (n < 0) return -3;
  if (ilo < 1) return -4;
  if (ihi > n || ihi < ilo - 1) return -5;
  if (lda < std::max(1, n)) return -7;
  if (ldb < std::max(1, n)) return -9;
  if ((cq > 0 && ldq < n) || ldq < 1) return -11;
  if ((cz > 0 && ldz < n) || ldz < 1) return -13;
  return 0;
}

static int gghrd_run(b200qz_ctx* c, int cq, int cz, bool qrows, int n, int ilo, int ihi, double* a, int lda, double* b,
                     int ldb, double* q, int ldq, double* z, int ldz) {
  qz::GghrdOut o;
  const cudaError_t e =
      qz::gghrd_device(c->stream, cq, cz, qrows, n, ilo - 1, ihi - 1, a, lda, b, ldb, q, ldq, z, ldz, c->hr_win, &o);
  return e == cudaSuccess ? 0 : 10001;
}

int b200qz_gghrd_dev(b200qz_ctx* c, char compq, char compz, int n, int ilo, int ihi, double* a, int lda, double* b,
                     int ldb, double* q, int ldq, double* z, int ldz) {
  if (!c) return 10001;
  const int bad = gghrd_args(compq, compz, n, ilo, ihi, lda, ldb, ldq, ldz);
  if (bad) return bad;
  if (n == 0) return 0;
  if (cudaSetDevice(c->device) != cudaSuccess) return 10001;
  return gghrd_run(c, comp_code(compq), comp_code(compz), false, n, ilo, ihi, a, lda, b, ldb, q, ldq, z, ldz);
}

// Host arrays: copied in, reduced, copied out (Q, Z only when referenced;
// an input Q, Z only for COMPQ, COMPZ = 'V').
static int gghrd_host_impl(b200qz_ctx* c, int cq, int cz, bool qrows, int n, int ilo, int ihi, double* a, int lda,
                           double* b, int ldb, double* q, int ldq, double* z, int ldz) {
  if (cudaSetDevice(c->device) != cudaSuccess) return 10001;
  const size_t nn = (size_t)n * n, w = (size_t)n * sizeof(double);
  double* d = nullptr;
  if (cudaMalloc(&d, 4 * nn * sizeof(double)) != cudaSuccess) return 10001;
  double *da = d, *db = d + nn, *dq = d + 2 * nn, *dz = d + 3 * nn;
  auto h2d = [&](double* dst, const double* src, int ld) {
    return cudaMemcpy2DAsync(dst, w, src, (size_t)ld * sizeof(double), w, n, cudaMemcpyHostToDevice, c->stream);
  };
  auto d2h = [&](double* dst, int ld, const double* src) {
    return cudaMemcpy2DAsync(dst, (size_t)ld * sizeof(double), src, w, w, n, cudaMemcpyDeviceToHost, c->stream);
  };
  cudaError_t e = h2d(da, a, lda);
  if (e == cudaSuccess) e = h2d(db, b, ldb);
  if (e == cudaSuccess && cq == 1) e = h2d(dq, q, ldq);
  if (e == cudaSuccess && cz == 1) e = h2d(dz, z, ldz);
  int r = 10001;
  if (e == cudaSuccess) r = gghrd_run(c, cq, cz, qrows, n, ilo, ihi, da, n, db, n, dq, n, dz, n);
  if (r == 0) {
    e = d2h(a, lda, da);
    if (e == cudaSuccess) e = d2h(b, ldb, db);
    if (e == cudaSuccess && cq > 0) e = d2h(q, ldq, dq);
    if (e == cudaSuccess && cz > 0) e = d2h(z, ldz, dz);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) r = 10001;
  }
  cudaFree(d);
  return r;
}

int b200qz_gghrd_host(b200qz_ctx* c, char compq, char compz, int n, int ilo, int ihi, double* a, int lda, double* b,
                      int ldb, double* q, int ldq, double* z, int ldz) {
  if (!c) return 10001;
  const int bad = gghrd_args(compq, compz, n, ilo, ihi, lda, ldb, ldq, ldz);
  if (bad) return bad;
  if (n == 0) return 0;
  return gghrd_host_impl(c, comp_code(compq), comp_code(compz), false, n, ilo, ihi, a, lda, b, ldb, q, ldq, z, ldz);
}

// PDGGHRD on a 1x1 grid (src/ab2ht/PDGGHRD.f:13-31): the same argument
// list with descriptors, a workspace query that returns MB_ in WORK(1)
// (PDGGHRD.f:243-250), Q returned transposed (row rotations accumulated
// from the left, as the reference's callers expect: examples/EXRAND2.f:
// 352-356 transposes it back) and INFO numbering of PDGGHRD.f:278-296.
void pdgghrd_(const char* compq, const char* compz, const int* n, const int* ilo, const int* ihi, double* a,
              const int* desca, double* b, const int* descb, double* q, const int* descq, double* z, const int* descz,
              double* work, const int* lwork, int* info, size_t len_compq, size_t len_compz) {
  (void)len_compq; (void)len_compz;
  const int N = *n, ILO = *ilo, IHI = *ihi;
  *info = 0;
  if (N <= 1) return;  // quick return before any check (PDGGHRD.f:198)
  const int mb = desca[4], nb = desca[5];
  if (*lwork == -1) { work[0] = (double)mb; return; }
  const int cq = comp_code(*compq), cz = comp_code(*compz);
  if (cq < 0) *info = -1;
  else if (cz < 0) *info = -2;
  else if (N < 0) *info = -3;
  else if (ILO < 1) *info = -4;
  else if (IHI > N || IHI < ILO - 1) *info = -5;
  else if (nb != mb) *info = -6;
  else if (*lwork < mb) *info = -7;
  if (*info != 0) return;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ctx) {
    int dev = 0;
    const char* e = std::getenv("B200QZ_DEVICE");
    if (e) dev = std::atoi(e);
    if (b200qz_create(&g_ctx, dev) != 0) { g_ctx = nullptr; *info = 10001; return; }
  }
  const int r = gghrd_host_impl(g_ctx, cq, cz, true, N, ILO, IHI, a, desca[8], b, descb[8], q, descq[8], z, descz[8]);
  if (r != 0) *info = r;
}

}  // extern "C"
