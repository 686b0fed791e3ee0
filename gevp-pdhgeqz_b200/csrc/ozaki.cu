// Split-precision off-diagonal updates: FP64 products recovered from INT8
// tensor-core slices (Ozaki scheme) on the 5th-generation tensor cores.
//
// Role in the reference: the PDGEMM / DGEMM updates of PDHGEQZ6
// (PDHGEQZ6.f:276-380, 1x1 grid) and after AED (PDHGEQZ0.f:776-864,
// PDHGEQZ3.f:1630-1726):
//   left :  M(r0:r0+k, c0:c0+L) <- W^T * M(r0:r0+k, c0:c0+L)
//   right:  M(r0:r0+L, c0:c0+k) <- M(r0:r0+L, c0:c0+k) * W
// Both are computed as one product D = A * W with A an L x k tile of the
// slab (A = X^T for the left update, A = X for the right update).
//
// Scheme.  Each row i of A is scaled by 2^-e_i (e_i: exponent of its
// largest entry) and each column j of W by 2^-f_j, so every entry x lies in
// (-1, 1), and split into S (7 or 8) signed 7-bit digits
//   x = sum_{s=1..S} q_s 2^(-6-7(s-1)) + r,   |q_s| <= 64,  |r| <= 2^(-7S).
// With int8 digit matrices QA_s, QB_t the product is
//   D(i,j) = 2^(e_i+f_j-12) * sum_{d=2..S+1} 2^(-7(d-2)) * acc_d(i,j),
//   acc_d = sum_{s+t=d} QA_s * QB_t   (S(S+1)/2 slice products, exact in
// int32: 28 for S = 7, 36 for S = 8); the products with s+t > S+1 are
// dropped, at the same order as r.  S = 7 leaves errors near 2^-48 of the
// row and column scales, S = 8 near 2^-55.  acc_d is formed on the tensor cores (tcgen05.mma kind::i8, A and
// B from shared memory, accumulators in TMEM), read back with tcgen05.ld and
// combined in FP64 by Horner's rule from d = 8 down.
//
// Kernels
//   k_ozaki_prep    one CTA per factor W: column scales and the seven digit
//                   matrices of W in the tensor cores' K-major layout
//   k_ozaki_update  one CTA per 128-row tile of a slab: stages the FP64
//                   tile in two halves and slices it, runs S(S+1)/2 x (k/32)
//                   MMAs per 32-column output chunk into S TMEM
//                   accumulators, combines them, and writes the chunk back
//                   in place
//
// Shared-memory operand layout (K-major, no swizzle): 8-row x 16-byte core
// matrices; rows of a core matrix 16 B apart, row groups SBO = 128 B apart,
// 16-wide K chunks LBO apart (2048 B for A's 128 rows, kp/8 * 128 B for B).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "ozaki.h"

namespace qz {

namespace {

constexpr int kOzThreads = 256;     // k_ozaki_update: 8 warps (two per TMEM lane quarter)
constexpr int kOzPrepThreads = 128;
constexpr int kOzRows = 128;  // MMA M
constexpr int kOzChunkN = 64; // output columns per MMA pass (one TMEM accumulator each)
constexpr int kOzOutN = 32;   // output columns per staged write-back
constexpr int kOzTmemCols = 512;  // (slices) accumulators x 64 columns
constexpr uint32_t kOzSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major, no-swizzle shared-memory matrix descriptor (Blackwell version 1)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor: S8 x S8 -> S32, both K-major, M = 128
__device__ __forceinline__ uint32_t idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kOzRows >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int32_t* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// S signed 7-bit digits of 16 values y = x * 2^(6+7(S-1)) (|x| < 1, the
// scale already applied), packed per digit into 16 bytes.  y is rounded to
// an integer V (exact for |V| < 2^53, already integral above), and V is
// written in balanced base 128 from the least significant digit up:
//   d = ((V + 64) mod 128) - 64,  V <- (V - d) / 128,
// the top digit taking what is left (|q_1| <= 64).
template <int S>
__device__ __forceinline__ void digits16(const double (&y)[16], uint4 (&out)[S]) {
  uint32_t w[S][4];
#pragma unroll
  for (int s = 0; s < S; ++s)
#pragma unroll
    for (int q = 0; q < 4; ++q) w[s][q] = 0u;
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    long long v = __double2ll_rn(y[e]);
#pragma unroll
    for (int s = S - 1; s >= 1; --s) {
      const long long d = ((v + 64) & 127) - 64;
      v = (v - d) >> 7;
      w[s][e >> 2] |= ((uint32_t)(d & 0xFF)) << (8 * (e & 3));
    }
    w[0][e >> 2] |= ((uint32_t)(v & 0xFF)) << (8 * (e & 3));
  }
#pragma unroll
  for (int s = 0; s < S; ++s) out[s] = make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
}

// a * 2^(sh) for the digit grid: one multiplication when 2^sh is a normal
// number, ldexp otherwise (rows whose scale is near the exponent range ends)
struct DigitScale {
  double m;
  int sh;
  bool fast;
  __device__ DigitScale(int S, int e) {
    sh = 6 + 7 * (S - 1) - e;
    fast = sh > -1000 && sh < 1000;
    m = fast ? ldexp(1.0, sh) : 0.0;
  }
  __device__ double operator()(double a) const { return fast ? a * m : ldexp(a, sh); }
};

// v * 2^e: one multiplication by the power of two built from its exponent
// bits while 2^e is a normal number, ldexp otherwise
__device__ __forceinline__ double scale_pow2(double v, int e) {
  if (e >= -1022 && e <= 1023) return v * __longlong_as_double((long long)(e + 1023) << 52);
  return ldexp(v, e);
}

// ---------------------------------------------------------------------------
template <int S>
__global__ void __launch_bounds__(kOzPrepThreads) k_ozaki_prep(OzPrep P) {
  const int f = blockIdx.x;
  const double* W = P.W[f];
  const int ldw = P.ldw[f];
  const int k = P.k[f];
  const int kp = (k + 15) & ~15;
  const int Kp = (k + 31) & ~31;
  const int kc_n = Kp / 16;
  uint8_t* out = P.out + (size_t)f * kOzFacBytes;
  int* scale = (int*)(out + (size_t)S * kp * Kp);
  for (int j = threadIdx.x; j < kp; j += blockDim.x) {
    double mx = 0.0;
    if (j < k)
      for (int kk = 0; kk < k; ++kk) mx = fmax(mx, fabs(W[kk + (int64_t)j * ldw]));
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);
    scale[j] = e;
    const DigitScale sc(S, e);
    for (int kc = 0; kc < kc_n; ++kc) {
      double x[16];
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        const int kk = kc * 16 + t;
        x[t] = (j < k && kk < k) ? sc(W[kk + (int64_t)j * ldw]) : 0.0;
      }
      uint4 d[S];
      digits16<S>(x, d);
      const size_t off = (size_t)(kc * (kp / 8) + j / 8) * 128 + (j % 8) * 16;
#pragma unroll
      for (int s = 0; s < S; ++s) *(uint4*)(out + (size_t)s * kp * Kp + off) = d[s];
    }
  }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ int oz_find_job(const OzBatch& B, int& tile) {
  int t = blockIdx.x;
  for (int j = 0; j < B.njobs; ++j) {
    if (t < B.job[j].tiles) { tile = t; return j; }
    t -= B.job[j].tiles;
  }
  tile = -1;
  return -1;
}

// shared memory: A digits (S x 128 x Kp) | B digits + scales | FP64 staging
// (half a slab tile: a TMA box of 66 x k or kbox x 64, or 64 x (k+1) for
// plain loads; or one 128 x 33 output chunk)
constexpr int kOzStageDoubles = kOzBoxRows * kOzMaxK;
static_assert(kOzStageDoubles >= kOzRows * (kOzOutN + 1), "staging too small");
static_assert(kOzStageDoubles >= 64 * (kOzMaxK + 1), "staging too small");
static_assert(kOzStageDoubles >= 64 * oz_left_box(kOzMaxK), "staging too small");

__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* m, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
// bounded wait on an mbarrier phase; false if it did not complete
__device__ __forceinline__ bool mbar_wait(uint64_t* m, uint32_t parity) {
  uint32_t done = 0, spins = 0;
  while (!done && spins < kOzSpinLimit) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(m)), "r"(parity)
        : "memory");
    ++spins;
  }
  return done != 0;
}
// one-dimensional bulk copy global -> shared (16-byte aligned, size a
// multiple of 16), completion counted on the mbarrier
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* m) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(m))
               : "memory");
}
// two-dimensional TMA tile load (no multicast): box of the tensor map at
// element coordinates (x, y), x the contiguous dimension
__device__ __forceinline__ void tma_g2s_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* m) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(m))
      : "memory");
}

template <int S>
__global__ void __launch_bounds__(kOzThreads, 1) k_ozaki_update(const __grid_constant__ OzBatch B) {
  extern __shared__ __align__(1024) uint8_t oz_smem[];
  __shared__ uint64_t mbar;
  __shared__ uint64_t lbar;  // loads (bulk copy of the B digits, TMA halves of the slab tile)
  __shared__ uint32_t tmem_base_s;
  __shared__ int escale[kOzRows];
  int tile;
  const int jb = oz_find_job(B, tile);
  if (jb < 0) return;
  const OzJob J = B.job[jb];
  const int k = J.k;
  const int kp = (k + 15) & ~15;
  const int Kp = (k + 31) & ~31;
  const int kc_n = Kp / 16;
  const int ldx = k + 1;
  const int row0 = tile * kOzRows;
  const int nrow = min(kOzRows, J.len - row0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  uint8_t* As = oz_smem;                                  // S x 128 x Kp
  uint8_t* Bs = As + (size_t)S * kOzRows * kOzMaxKp;      // S x kp x Kp, then kp ints
  double* Xs = (double*)(Bs + kOzFacBytes);               // staging
  const uint8_t* Bg = B.bslices + (size_t)J.fac * kOzFacBytes;
  const int* fscale = (const int*)(Bs + (size_t)S * kp * Kp);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(kOzTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&mbar, 1);
    mbar_init(&lbar, 1);
  }
  __syncthreads();
  // Loads.  The B digits and column scales (prepared once per factor) come
  // in one bulk copy; the FP64 slab tile comes in two halves of 64 rows of A
  // by TMA when the job has a tensor map (right update: box 66 x k at the
  // tile's first row rounded down to even; left update: box kbox x 64 at
  // row r0 rounded down to even), else by plain loads.  Each half is sliced
  // into the INT8 digit planes of A; thread t takes row (t & 63) of the half
  // and every other K chunk.
  const bool tma = J.map >= 0;
  const CUtensorMap* map = tma ? &B.maps[J.map] : nullptr;
  const int kbox = oz_left_box(k);
  const uint32_t box_bytes = (uint32_t)(J.left ? kbox * 64 : kOzBoxRows * k) * 8u;
  bool lok = true;
  uint32_t lphase = 0;
  if (tid == 0) {
    mbar_expect_tx(&lbar, (uint32_t)kOzFacBytes + (tma ? box_bytes : 0u));
    bulk_g2s(Bs, Bg, (uint32_t)kOzFacBytes, &lbar);
  }
  for (int h = 0; h < 2; ++h) {
    const int rb = 64 * h;
    int off = 0;  // rows the box starts above the first wanted one
    if (tma) {
      const int xr = J.left ? J.r0 : J.r0 + row0 + rb;
      off = xr & 1;
      if (tid == 0) {
        if (h == 1) {
          fence_async_smem();  // the first half's reads of the staging buffer come first
          mbar_expect_tx(&lbar, box_bytes);
        }
        if (J.left) tma_g2s_2d(Xs, map, xr - off, J.c0 + row0 + rb, &lbar);
        else tma_g2s_2d(Xs, map, xr - off, J.c0, &lbar);
      }
      lok = __syncthreads_and(mbar_wait(&lbar, lphase) ? 1 : 0) != 0;
      lphase ^= 1u;
      if (!lok) break;
    } else {
      if (h == 0) {
        lok = __syncthreads_and(mbar_wait(&lbar, lphase) ? 1 : 0) != 0;  // B digits
        lphase ^= 1u;
        if (!lok) break;
      }
      if (J.left) {
        // A(i, kk) = M(r0 + kk, c0 + row0 + i): contiguous in kk
        for (int idx = tid; idx < 64 * k; idx += kOzThreads) {
          const int kk = idx % k, i = idx / k;
          Xs[i * ldx + kk] = (rb + i < nrow) ? J.M[(J.r0 + kk) + (int64_t)(J.c0 + row0 + rb + i) * J.ld] : 0.0;
        }
      } else {
        // A(i, kk) = M(r0 + row0 + i, c0 + kk): contiguous in i
        for (int idx = tid; idx < 64 * k; idx += kOzThreads) {
          const int i = idx % 64, kk = idx / 64;
          Xs[i * ldx + kk] = (rb + i < nrow) ? J.M[(J.r0 + row0 + rb + i) + (int64_t)(J.c0 + kk) * J.ld] : 0.0;
        }
      }
      __syncthreads();
    }
    {
      const int il = tid & 63, par = tid >> 6;  // par: 0 .. kOzThreads/64 - 1
      const int i = rb + il;
      // element (il, kk) of the half in the staging layout
      auto xv = [&](int kk) -> double {
        if (!tma) return Xs[il * ldx + kk];
        if (J.left) return Xs[il * kbox + kk + off];
        return Xs[kk * kOzBoxRows + il + off];
      };
      double mx = 0.0;
      if (rb + il < nrow)
        for (int kk = 0; kk < k; ++kk) mx = fmax(mx, fabs(xv(kk)));
      int e = 0;
      if (mx > 0.0) frexp(mx, &e);
      if (par == 0) escale[i] = e;
      const DigitScale sc(S, e);
      for (int kc = par; kc < kc_n; kc += kOzThreads / 64) {
        double x[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) {
          const int kk = kc * 16 + t;
          x[t] = (kk < k && rb + il < nrow) ? sc(xv(kk)) : 0.0;
        }
        uint4 d[S];
        digits16<S>(x, d);
        const size_t o = (size_t)(kc * (kOzRows / 8) + i / 8) * 128 + (i % 8) * 16;
#pragma unroll
        for (int s = 0; s < S; ++s) *(uint4*)(As + (size_t)s * kOzRows * Kp + o) = d[s];
      }
    }
    __syncthreads();  // the staging buffer is reused by the next half
  }
  if (!lok) {
    // a load did not complete in time: nothing was computed; report it, and
    // give the copy in flight one more bounded wait before the CTA (and its
    // shared memory) goes away
    if (tid == 0) atomicExch(B.err, 1);
    (void)mbar_wait(&lbar, lphase ^ 1u);
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base_s),
                                "r"(kOzTmemCols));
    return;
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;
  const uint32_t a_base = smem_u32(As), b_base = smem_u32(Bs);
  const uint32_t lbo_a = (kOzRows / 8) * 128, lbo_b = (uint32_t)(kp / 8) * 128;
  const int nchunk = (kp + kOzChunkN - 1) / kOzChunkN;
  const int ldo = kOzOutN + 1;
  bool ok = true;
  for (int nc = 0; nc < nchunk; ++nc) {
    const int n0 = nc * kOzChunkN;
    const int nn = min(kOzChunkN, kp - n0);  // 16, 32, 48 or 64
    if (tid == 0) {
      tc_fence_after();
      const uint32_t idesc = idesc_i8(nn);
      for (int d = 2; d <= S + 1; ++d) {
        uint32_t acc = 0;
        const uint32_t dcol = tmem + (uint32_t)(d - 2) * kOzChunkN;
        for (int s = (d - S > 1 ? d - S : 1); s <= (d - 1 < S ? d - 1 : S); ++s) {
          const int t = d - s;
          for (int ks = 0; ks < Kp / 32; ++ks) {
            const uint64_t a = umma_desc(a_base + (uint32_t)((s - 1) * kOzRows * Kp) + (uint32_t)(2 * ks) * lbo_a,
                                         lbo_a, 128);
            const uint64_t b = umma_desc(b_base + (uint32_t)((t - 1) * kp * Kp) + (uint32_t)(2 * ks) * lbo_b +
                                             (uint32_t)(n0 / 8) * 128,
                                         lbo_b, 128);
            mma_i8(dcol, a, b, idesc, acc);
            acc = 1;
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mbar))
                   : "memory");
    }
    // wait for the chunk's MMAs (bounded); the outcome is made uniform
    // across the CTA, and after a timeout no further MMA is issued: one more
    // bounded wait lets the chunk in flight drain before the TMEM is freed
    {
      const uint32_t parity = (uint32_t)(nc & 1);
      auto wait = [&]() {
        uint32_t done = 0, spins = 0;
        while (!done && spins < kOzSpinLimit) {
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
              "selp.b32 %0, 1, 0, p;\n\t}\n"
              : "=r"(done)
              : "r"(smem_u32(&mbar)), "r"(parity)
              : "memory");
          ++spins;
        }
        return done != 0;
      };
      ok = __syncthreads_and(wait() ? 1 : 0) != 0;
      if (!ok) {
        (void)wait();
        break;
      }
    }
    tc_fence_after();
    // epilogue in 32-column pieces: thread = row i (TMEM lane); per 8
    // columns all S accumulators are loaded, then combined by Horner's
    // rule from the smallest weight up; the piece is staged and written
    // back in place, coalesced
    for (int p0 = 0; p0 < nn; p0 += kOzOutN) {
      const int pn = min(kOzOutN, nn - p0);
      if (ok) {
        // a warp reads the TMEM lanes of its quarter (warp % 4); the two
        // warps of a quarter take alternate 8-column groups
        const int wq = warp & 3, half = warp >> 2;
        const int i = wq * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(wq * 32) << 16);
        for (int g = half; g < pn / 8; g += kOzThreads / 128) {
          int32_t v[S][8];
#pragma unroll
          for (int d = 0; d < S; ++d) tmem_ld8(lane_addr + (uint32_t)(d * kOzChunkN + p0 + 8 * g), v[d]);
          tmem_wait_ld();
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            double val = (double)v[S - 1][e];
#pragma unroll
            for (int d = S - 2; d >= 0; --d) val = fma(val, 0.0078125, (double)v[d][e]);
            const int j = n0 + p0 + 8 * g + e;
            Xs[i * ldo + 8 * g + e] = (j < k) ? scale_pow2(val, escale[i] + fscale[j] - 12) : 0.0;
          }
        }
      }
      __syncthreads();
      if (ok) {
        const int cb = n0 + p0;
        const int ncol = min(pn, k - cb);
        if (J.left) {
          // D(i, cb + j) -> M(r0 + cb + j, c0 + row0 + i)
          for (int idx = tid; idx < kOzRows * ncol; idx += kOzThreads) {
            const int j = idx % ncol, i = idx / ncol;
            if (i < nrow) J.M[(J.r0 + cb + j) + (int64_t)(J.c0 + row0 + i) * J.ld] = Xs[i * ldo + j];
          }
        } else {
          // D(i, cb + j) -> M(r0 + row0 + i, c0 + cb + j)
          for (int idx = tid; idx < kOzRows * ncol; idx += kOzThreads) {
            const int i = idx % kOzRows, j = idx / kOzRows;
            if (i < nrow) J.M[(J.r0 + row0 + i) + (int64_t)(J.c0 + cb + j) * J.ld] = Xs[i * ldo + j];
          }
        }
      }
      __syncthreads();
    }
    tc_fence_before();
    __syncthreads();
  }
  if (!ok && tid == 0) atomicExch(B.err, 1);
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kOzTmemCols));
}

}  // namespace

bool ozaki_tensor_map(CUtensorMap* map, const double* M, int64_t ld, int rows, int cols, int left, int k) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Encode encode = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = (Encode)fn;
  }
  if (!encode || !M || rows < 1 || cols < 1 || k < 1 || k > kOzMaxK) return false;
  // TMA: base 16-byte aligned, column stride a multiple of 16 bytes
  if (((uintptr_t)M & 15u) != 0 || (ld * 8) % 16 != 0 || ld < rows) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 8u};
  const cuuint32_t box[2] = {left ? (cuuint32_t)oz_left_box(k) : (cuuint32_t)kOzBoxRows,
                             left ? 64u : (cuuint32_t)k};
  const cuuint32_t estr[2] = {1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void*)M, dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t ozaki_smem_bytes(int slices) {
  return (size_t)slices * kOzRows * kOzMaxKp + kOzFacBytes + (size_t)kOzStageDoubles * sizeof(double);
}

cudaError_t ozaki_init() {
  cudaError_t e = cudaFuncSetAttribute(k_ozaki_update<7>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)ozaki_smem_bytes(7));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_ozaki_update<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)ozaki_smem_bytes(8));
}

void launch_ozaki_prep(cudaStream_t st, const OzPrep& P, int slices) {
  if (P.nfac <= 0) return;
  if (slices == 8) k_ozaki_prep<8><<<P.nfac, kOzPrepThreads, 0, st>>>(P);
  else k_ozaki_prep<7><<<P.nfac, kOzPrepThreads, 0, st>>>(P);
}

void launch_ozaki_update(cudaStream_t st, const OzBatch& B, int slices) {
  int tiles = 0;
  for (int j = 0; j < B.njobs; ++j) tiles += B.job[j].tiles;
  if (tiles <= 0) return;
  if (slices == 8) k_ozaki_update<8><<<tiles, kOzThreads, ozaki_smem_bytes(8), st>>>(B);
  else k_ozaki_update<7><<<tiles, kOzThreads, ozaki_smem_bytes(7), st>>>(B);
}

}  // namespace qz
