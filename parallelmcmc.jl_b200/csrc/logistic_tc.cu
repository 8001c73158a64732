// logistic_tc.cu -- one logistic-regression pass on the 5th-generation tensor
// cores (tcgen05 + TMEM + TMA), fused GEMM -> epilogue -> GEMM.
//
// For a tile of BT trajectory columns (value columns v_t = x_bar_t or y_t, and
// the matching tangent columns z_t or w_t) and all N data rows:
//   GEMM1  L[n, t] = sum_d X[n, d] B[d, t]                     (M = 128 rows of X)
//   epilogue (per row n, per column t): p = sigmoid(L), r = y_n - p,
//          s = p (1 - p) L_tangent, loglik = y_n L - softplus(L)  (bayes_logreg.jl:118-154)
//   GEMM2  G[d, t] += sum_n X[n, d] R[n, t],  R = [r | s]       (M = 128 values of d)
// The N x 2T intermediate never leaves the SM: L lives in TMEM, R in shared
// memory.  G starts afresh in TMEM at every 128-row block and the epilogue
// threads add the blocks' partial sums in registers (round-to-nearest FP32):
// one TMEM accumulation chain over all N rows left the N = 10000 gradient about
// 10x less accurate than an FP32 SGEMM, enough to move the chain by 1.5e-5.
// The same shared-memory X tile is GEMM1's K-major A operand and GEMM2's
// MN-major A operand.
//
// Precision: X, the value columns and r are carried as FP16 hi + lo pairs
// (about 22 significant bits); each value-column product is
// hi*hi + hi*lo + lo*hi with FP32 accumulation.  Tangent columns (only used
// for the Jacobian estimate) and s use a single FP16 term.
//
// The MMAs are bound by shared-memory reads of the X operand at these widths,
// so each k step issues two: Xh [Bh | Bt | Bl] (N = 96, the hi*lo product in
// accumulator columns of its own, added in the epilogue) and Xl Bh (N = 32,
// accumulated onto the hi*hi columns).  GEMM2 is arranged the same way with
// [Rh | S | Rl].
//
// Roles: warps 0-15 run the epilogue (warps w, w+4, w+8, w+12 share TMEM lane
// quarter w % 4 and take 8 columns each); lane 0 of warp 16 issues TMA loads
// and MMAs and warp 16 owns the TMEM allocation.
// Every mbarrier wait is bounded; on timeout the kernel records an error,
// drains its own MMAs and frees TMEM before returning.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "deer_device.cuh"
#include "deer_launch.h"
#include "logistic.h"

namespace pmcmc {
namespace tc {

constexpr int BN = 128;  // data rows per block (GEMM1 M)
constexpr int BT = 32;   // value columns per CTA (plus BT tangent columns)
constexpr int kThreadsTC = 544;  // 16 epilogue warps + 1 producer warp
constexpr int kEpi = 16;
constexpr int kProd = 16;  // producer / TMEM-owner warp
constexpr int kParts = kEpi / 4;  // epilogue warps per TMEM lane quarter
constexpr uint32_t kTmemCols = 512;  // L at 0, G half h at 128 (h + 1); 96 columns each
constexpr long long kWaitCycles = 2000000000ll;  // ~1 s at B200 clocks
constexpr uint32_t kBoxX = BN * 128;       // one 64-wide d box of X: 128 rows x 128 B
constexpr uint32_t kBoxB = 3 * BT * 128;  // value hi rows | tangent rows | value lo rows
// R (GEMM2's B operand, N = 96 columns [r hi | s | r lo] by K = BN rows) is
// MN-major with the 128-byte swizzle, like X^T: two 64-column atoms of BN rows
// x 128 B; chunk c (8 columns) of row k sits at chunk c ^ (k & 7).
constexpr uint32_t kRAtom = BN * 128;

struct Layout {
  uint32_t xh, xl, b, r, bars, total;
};

__host__ __device__ inline Layout layout(int nkb) {
  Layout L;
  uint32_t off = 0;
  L.xh = off;
  off += nkb * kBoxX;
  L.xl = off;
  off += nkb * kBoxX;
  L.b = off;
  off += nkb * kBoxB;
  L.r = off;
  off += 2 * kRAtom;
  L.bars = off;
  off += 128;
  L.total = off + 1024;  // slack for 1024-B alignment of the dynamic window
  return L;
}

__device__ __forceinline__ uint32_t su32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(su32(b))
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
          su32(b)),
      "r"(bytes)
      : "memory");
}
// Bounded wait for the completion of the phase with the given parity: gives up
// after about a second of SM clock (or at once when another CTA of the launch
// has already reported an error).
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity,
                                          const volatile int* err) {
  const uint32_t a = su32(b);
  const long long start = clock64();
  for (long long i = 0;; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 255) == 255 && (*err || clock64() - start > kWaitCycles)) return false;
  }
}

__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* tm, int x, int y,
                                       uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3}], [%4];" ::"r"(su32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(su32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void mma_f16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 32 consecutive FP32 TMEM columns of this warp's 32 lanes (one per thread).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Three 8-column TMEM loads of this warp's 32 lanes, then one wait.  The wait
// is in the same asm statement as the loads, so no use of the registers can
// move above it.
__device__ __forceinline__ void tmem_ld8x3(uint32_t ta, uint32_t tb, uint32_t tc, float (&a)[8],
                                           float (&b)[8], float (&c)[8]) {
  uint32_t r[24];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%24];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8, %9, %10, %11, %12, %13, %14, %15}, [%25];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%16, %17, %18, %19, %20, %21, %22, %23}, [%26];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23])
      : "r"(ta), "r"(tb), "r"(tc)
      : "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    a[i] = __uint_as_float(r[i]);
    b[i] = __uint_as_float(r[8 + i]);
    c[i] = __uint_as_float(r[16 + i]);
  }
}

// Shared-memory matrix descriptor (tcgen05): start, leading / stride byte
// offsets, version 1, layout (0 = no swizzle, 2 = 128-byte swizzle).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo,
                                          uint32_t layout) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  d |= static_cast<uint64_t>(layout & 7u) << 61;
  return d;
}

// Instruction descriptor, kind::f16 with FP16 A/B and FP32 accumulation.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

// log(1 + e) for e in [0, 1]: e q(e), q the degree-9 Chebyshev least-squares
// fit of log1p(e) / e on [0, 1] written in powers of e with FP32 coefficients.
// Absolute error below 1.3e-7 on [0, 1] (a correctly rounded FP32 log1p has
// 6e-8; the FP32 rounding of the log-likelihood term it enters is larger than
// either).  FMAs only: no division, no special-function unit.
__device__ __forceinline__ float log1p_unit(float e) {
  float q = -0.0032140363473445177f;
  q = fmaf(q, e, 0.019649166613817215f);
  q = fmaf(q, e, -0.056435029953718185f);
  q = fmaf(q, e, 0.10533228516578674f);
  q = fmaf(q, e, -0.1525145173072815f);
  q = fmaf(q, e, 0.19651491940021515f);
  q = fmaf(q, e, -0.24947808682918549f);
  q = fmaf(q, e, 0.3332909941673279f);
  q = fmaf(q, e, -0.4999985098838806f);
  q = fmaf(q, e, 1.0f);
  return e * q;
}

// Two FP32 values as one FP16x2 word (a in the low half), one conversion.
__device__ __forceinline__ uint32_t half2_bits(float a, float b) {
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// hi = x with its low 13 mantissa bits cleared: exact in FP16 for
// 2^-14 <= |x| < 65504, and x - hi is exact in FP32 (|x - hi| < 2^-10 |x|).
__device__ __forceinline__ float split_hi(float x) {
  return __uint_as_float(__float_as_uint(x) & 0xffffe000u);
}

// G (Dp x 2T column-major: value block then tangent block, FP32) and lp (T,
// FP64) for the column tile blockIdx.x.  has_tangent = 0: value columns only,
// no G (the logp pass over a returned trajectory).
__global__ void __launch_bounds__(kThreadsTC, 1)
    logistic_pass_tc_kernel(const __grid_constant__ CUtensorMap tmXh,
                            const __grid_constant__ CUtensorMap tmXl,
                            const __grid_constant__ CUtensorMap tmBh,
                            const __grid_constant__ CUtensorMap tmBl,
                            const __grid_constant__ CUtensorMap tmBt,
                            const float* __restrict__ ylab, int64_t N, int nkb, int64_t T,
                            int64_t Dp, float* __restrict__ G, double* __restrict__ lp,
                            int has_tangent, int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  const Layout Ly = layout(nkb);
  unsigned char* sXh = base + Ly.xh;
  unsigned char* sXl = base + Ly.xl;
  unsigned char* sB = base + Ly.b;
  unsigned char* sR = base + Ly.r;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + Ly.bars);
  // X moves box by box (64 values of d, hi and lo): GEMM2's d-half h reads
  // exactly boxes 2h and 2h + 1, so the next block's boxes of half h load
  // while GEMM2's later half runs, and GEMM1 starts on box 0 as soon as it lands.
  uint64_t* bar_b = bars + 0;  // B tile loaded
  uint64_t* bar_x = bars + 1;  // [4] X box kb loaded
  uint64_t* bar_l = bars + 5;  // GEMM1 done (L ready)
  uint64_t* bar_r = bars + 6;  // epilogue wrote R (32 kEpi arrivals)
  uint64_t* bar_g = bars + 7;  // [2] GEMM2 half h done (X boxes of half h free; R free after the last)
  uint64_t* bar_z = bars + 9;  // teardown drain
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  __shared__ double s_red[kEpi][BT / kParts];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * BT;
  const int nblocks = static_cast<int>((N + BN - 1) / BN);
  const int nh = nkb / 2;
  const bool has_g = has_tangent != 0;

  if (threadIdx.x == 0) {
    mbar_init(bar_b, 1);
    for (int kb = 0; kb < 4; ++kb) mbar_init(bar_x + kb, 1);
    mbar_init(bar_l, 1);
    mbar_init(bar_r, 32 * kEpi);
    mbar_init(bar_g, 1);
    mbar_init(bar_g + 1, 1);
    mbar_init(bar_z, 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kProd) tmem_alloc(&s_tmem, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  // L: columns [0, 96) = value (hi*hi + lo*hi) | tangent | value hi*lo.
  // G half h: columns [128 (h + 1), 128 (h + 1) + 96), the same three parts.
  const uint32_t tL = tmem;
  const uint32_t tG = tmem + 128;

  if (warp == kProd) {
    if (lane == 0) {
      bool ok = true;
      const uint32_t i1_all = idesc_f16(128, 3 * BT, false, false);
      const uint32_t i1_v = idesc_f16(128, BT, false, false);
      const uint32_t i2_all = idesc_f16(128, 3 * BT, true, true);
      const uint32_t i2_v = idesc_f16(128, BT, true, true);
      mbar_expect_tx(bar_b, nkb * kBoxB);
      for (int kb = 0; kb < nkb; ++kb) {
        unsigned char* b = sB + kb * kBoxB;
        tma_2d(b, &tmBh, kb * 64, static_cast<int>(t0), bar_b);
        // without tangent columns the middle rows repeat Bh: the MMA reads
        // them and nothing uses their products
        tma_2d(b + BT * 128, has_tangent ? &tmBt : &tmBh, kb * 64, static_cast<int>(t0), bar_b);
        tma_2d(b + 2 * BT * 128, &tmBl, kb * 64, static_cast<int>(t0), bar_b);
      }
      ok = mbar_wait(bar_b, 0, err);
      auto load_x = [&](int nb, int kb) {
        mbar_expect_tx(bar_x + kb, 2 * kBoxX);
        tma_2d(sXh + kb * kBoxX, &tmXh, kb * 64, nb * BN, bar_x + kb);
        tma_2d(sXl + kb * kBoxX, &tmXl, kb * 64, nb * BN, bar_x + kb);
      };
      if (ok)
        for (int kb = 0; kb < nkb; ++kb) load_x(0, kb);
      for (int nb = 0; nb < nblocks && ok; ++nb) {
        // GEMM1: L = Xh [Bh | Bt | Bl] + Xl Bh, box by box as X arrives
        for (int kb = 0; kb < nkb; ++kb) {
          if (!(ok = mbar_wait(bar_x + kb, nb & 1, err))) break;
          tc_fence_after();
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            const uint64_t ah = sdesc(su32(sXh + kb * kBoxX) + ks * 32, 16, 1024, 2);
            const uint64_t al = sdesc(su32(sXl + kb * kBoxX) + ks * 32, 16, 1024, 2);
            const uint64_t bb = sdesc(su32(sB + kb * kBoxB) + ks * 32, 16, 1024, 2);
            mma_f16(tL, ah, bb, i1_all, (kb | ks) != 0);
            mma_f16(tL, al, bb, i1_v, 1);
          }
        }
        if (!ok) break;
        mma_commit(bar_l);
        if (!(ok = mbar_wait(bar_r, nb & 1, err))) break;
        tc_fence_after();
        // GEMM2: G_h += Xh^T [Rh | S | Rl] + Xl^T Rh  (A MN-major, B MN-major)
        for (int h = 0; h < nh; ++h) {
          if (has_g) {
#pragma unroll
            for (int kn = 0; kn < BN / 16; ++kn) {
              const uint64_t ah = sdesc(su32(sXh + 2 * h * kBoxX) + kn * 2048, kBoxX, 1024, 2);
              const uint64_t al = sdesc(su32(sXl + 2 * h * kBoxX) + kn * 2048, kBoxX, 1024, 2);
              const uint64_t br = sdesc(su32(sR) + kn * 2048, kRAtom, 1024, 2);
              // every row block starts G afresh: the epilogue has added the
              // previous block's G into its registers before it wrote R
              const uint32_t acc = kn > 0 ? 1u : 0u;
              mma_f16(tG + 128 * h, ah, br, i2_all, acc);
              mma_f16(tG + 128 * h, al, br, i2_v, 1);
            }
          }
          mma_commit(bar_g + h);
        }
        // the next block's X, half h as soon as GEMM2's half h has read it
        if (nb + 1 < nblocks)
          for (int h = 0; h < nh; ++h) {
            if (!(ok = mbar_wait(bar_g + h, nb & 1, err))) break;
            load_x(nb + 1, 2 * h);
            load_x(nb + 1, 2 * h + 1);
          }
      }
      if (!ok) {
        s_abort = 1;
        atomicExch(err, 1);
      }
      // drain every MMA this thread issued before TMEM is released
      mma_commit(bar_z);
      if (!mbar_wait(bar_z, 0, err)) atomicExch(err, 1);
    }
    __syncwarp();
  } else {
    // ---- epilogue: thread = TMEM lane = data row; warp part = column block ----
    const int quarter = warp & 3, part = warp >> 2;  // columns [8 part, 8 part + 8)
    const int row = quarter * 32 + lane;
    const uint32_t lane_off = static_cast<uint32_t>(quarter * 32) << 16;
    constexpr int BH = BT / kParts;
    static_assert(BH == 8, "one 8-column block of R a thread");
    // log-likelihood sums, compensated (Kahan) in FP32: ls the sum, lc the
    // running error; the column total is ls - lc, formed in FP64 at the end
    float ls[BH], lc[BH];
#pragma unroll
    for (int t = 0; t < BH; ++t) ls[t] = lc[t] = 0.f;
    bool ok = true;
    float y_next = row < N ? __ldg(ylab + row) : 0.f;  // label of this row, one block ahead
    // G accumulates one row block at a time in TMEM; the blocks' partial sums
    // are added here, in FP32 with round-to-nearest.  Part 2 h + b owns d-half
    // h of G, the value block (b = 0, hi*lo columns added) or the tangent block.
    const bool g_owner = has_g && part < 2 * nh;
    const int gh = part >> 1, gb = part & 1;
    float gacc[BT];
#pragma unroll
    for (int t = 0; t < BT; ++t) gacc[t] = 0.f;
    auto add_g = [&]() {
      const uint32_t ga = tG + 128 * gh + lane_off + BT * gb;
#pragma unroll
      for (int c = 0; c < BT; c += 8) {
        float a[8], b8[8], unused[8];
        if (gb == 0) {
          tmem_ld8x3(ga + c, tG + 128 * gh + lane_off + 2 * BT + c, ga + c, a, b8, unused);
#pragma unroll
          for (int i = 0; i < 8; ++i) gacc[c + i] += a[i] + b8[i];
        } else {
          tmem_ld8x3(ga + c, ga + c, ga + c, a, b8, unused);
#pragma unroll
          for (int i = 0; i < 8; ++i) gacc[c + i] += a[i];
        }
      }
    };
    for (int nb = 0; nb < nblocks; ++nb) {
      const int64_t n = static_cast<int64_t>(nb) * BN + row;
      const bool valid = n < N;
      const float yn = y_next;
      if (n + BN < N) y_next = __ldg(ylab + n + BN);
      if (g_owner && nb > 0) {
        // the previous block's G partials are final once its GEMM2 has committed,
        // and the next GEMM2 restarts G only after this block's R (bar_r): they
        // are added while this block's X arrives and its GEMM1 runs
        if (!(ok = mbar_wait(bar_g + (nh - 1), (nb - 1) & 1, err))) break;
        tc_fence_after();
        add_g();
      }
      if (!(ok = mbar_wait(bar_l, nb & 1, err))) break;
      tc_fence_after();
      float v[BH], vl[BH], w[BH];
      tmem_ld8x3(tL + lane_off + BH * part, tL + lane_off + 2 * BT + BH * part,
                 tL + lane_off + BT + BH * part, v, vl, w);
      float r[BH], s[BH];
#pragma unroll
      for (int t = 0; t < BH; ++t) {
        const float l = v[t] + vl[t];
        const float e = __expf(-fabsf(l));
        const float inv = __fdividef(1.f, 1.f + e);
        const float p = l >= 0.f ? inv : e * inv;
        r[t] = valid ? yn - p : 0.f;
        s[t] = (valid && has_tangent) ? p * (1.f - p) * w[t] : 0.f;
        if (valid) {
          const float y = (yn * l - (fmaxf(l, 0.f) + log1p_unit(e))) - lc[t];
          const float sum = ls[t] + y;
          lc[t] = (sum - ls[t]) - y;
          ls[t] = sum;
        }
      }
      if (has_g) {
        // R columns as FP16: r split hi + lo, s one term; two values a conversion
        uint32_t wh[BH / 2], wl[BH / 2], ws[BH / 2];
#pragma unroll
        for (int q = 0; q < BH / 2; ++q) {
          const float h0 = split_hi(r[2 * q]), h1 = split_hi(r[2 * q + 1]);
          wh[q] = half2_bits(h0, h1);
          wl[q] = half2_bits(r[2 * q] - h0, r[2 * q + 1] - h1);
          ws[q] = half2_bits(s[2 * q], s[2 * q + 1]);
        }
        // value hi: atom 0 chunk part; s: atom 0 chunk 4 + part; value lo: atom 1 chunk part
        unsigned char* rrow = sR + row * 128;
        const int sw = row & 7;
        *reinterpret_cast<uint4*>(rrow + ((part ^ sw) << 4)) = make_uint4(wh[0], wh[1], wh[2], wh[3]);
        *reinterpret_cast<uint4*>(rrow + (((4 + part) ^ sw) << 4)) = make_uint4(ws[0], ws[1], ws[2], ws[3]);
        *reinterpret_cast<uint4*>(rrow + kRAtom + ((part ^ sw) << 4)) = make_uint4(wl[0], wl[1], wl[2], wl[3]);
        fence_async_smem();
      }
      tc_fence_before();
      mbar_arrive(bar_r);
    }
    if (ok && has_g && mbar_wait(bar_g + (nh - 1), (nblocks - 1) & 1, err)) {
      tc_fence_after();
      if (g_owner) {
        add_g();  // the last row block
        const int64_t d = 128 * gh + row;
        if (d < Dp) {
          const int64_t cbase = gb ? T : 0;
#pragma unroll
          for (int t = 0; t < BT; ++t)
            if (t0 + t < T) G[(cbase + t0 + t) * Dp + d] = gacc[t];
        }
      }
    } else if (!ok) {
      atomicExch(err, 1);
    }
#pragma unroll
    for (int t = 0; t < BH; ++t) {
      const double sum = warp_sum(static_cast<double>(ls[t]) - static_cast<double>(lc[t]));
      if (lane == 0) s_red[warp][t] = sum;
    }
    asm volatile("bar.sync 1, %0;" ::"n"(32 * kEpi) : "memory");
    if (threadIdx.x < BT && t0 + threadIdx.x < T) {
      const int t = threadIdx.x, hh = t / BH, tt = t % BH;
      double a = 0.0;
      for (int q = 0; q < 4; ++q) a += s_red[4 * hh + q][tt];
      lp[t0 + t] = a;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kProd) tmem_dealloc(tmem, kTmemCols);
}

// Builds the FP16 split operands of one pass: Bh/Bl (value columns hi / lo)
// and Bt (tangent columns), each T x Dk (t-major rows, d contiguous).
//   mode 0: value x_bar_t, tangent z_t (probe `probe`); mode 1: value y_t, tangent w_t;
//   mode 2: value S_t, no tangent.
template <typename Real>
__global__ void tc_prep_kernel(const DevParams* __restrict__ Pg, const DevState* __restrict__ st,
                               int mode, int probe, int64_t Dk, __half* __restrict__ Bh,
                               __half* __restrict__ Bl, __half* __restrict__ Bt) {
  const DevParams& P = *Pg;
  const int iter = st->iter;
  const bool from_x0 = iter == 0;
  const Real* S = static_cast<const Real*>(P.S[st->cur]);
  const Real* x0 = static_cast<const Real*>(P.x0);
  const TapeKey key(P.seed, P.block);
  const int64_t n = P.T * Dk;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = i / Dk, d = i % Dk;
    float v = 0.f, tv = 0.f;
    if (d < P.D) {
      if (mode == 0) {
        v = static_cast<float>((from_x0 || t == 0) ? x0[d] : S[(t - 1) * P.Dp + d]);
        const U4 pb = probe_bits(key, static_cast<uint32_t>(d >> 7),
                                 static_cast<uint32_t>(t + P.t_off),
                                 probe, iter);
        tv = ((u4_word(pb, static_cast<int>((d >> 5) & 3)) >> (d & 31)) & 1u) ? 1.f : -1.f;
      } else if (mode == 1) {
        v = static_cast<float>(static_cast<const Real*>(P.lg[1])[t * P.Dp + d]);
        tv = static_cast<float>(static_cast<const Real*>(P.lg[2])[t * P.Dp + d]);
      } else {
        v = static_cast<float>(S[t * P.Dp + d]);
      }
    }
    const __half h = __float2half_rn(v);
    Bh[i] = h;
    Bl[i] = __float2half_rn(v - __half2float(h));
    if (mode != 2) Bt[i] = __float2half_rn(tv);
  }
}

// ---------------------------------------------------------------------------
// Wide variant, 256 < D <= 512 (Dk = 512): 16 value columns a CTA (plus 16
// tangent columns) so that B (48 KB) and R fit beside a ring of four X boxes
// (128 KB).  The eight 64-wide d boxes of a row block pass through the ring:
// GEMM1 runs over boxes 0-3, then 4-7 as each slot frees; GEMM2 takes the d
// quarters 2 and 3 from the resident boxes 4-7, then the quarters 0 and 1
// from boxes 0-3 loaded again.  Per 128-row block this is the FLOPs of the
// D <= 256 kernel (half the columns, twice the depth) with 12 box loads
// instead of 8.  Each slot sees three loads and three releases a block, so
// its two mbarriers stay one phase per use.
// ---------------------------------------------------------------------------
constexpr int BTW = 16;          // value columns per CTA (plus BTW tangent columns)
constexpr int kSlots = 4;        // X boxes resident at a time
constexpr int kNkbW = 8;         // 64-wide d boxes of Dk = 512
constexpr uint32_t kBoxBW = 3 * BTW * 128;  // value hi | tangent | value lo rows of a d box

struct LayoutW {
  uint32_t xh, xl, b, r, bars, total;
};

__host__ __device__ inline LayoutW layout_wide() {
  LayoutW L;
  uint32_t off = 0;
  L.xh = off;
  off += kSlots * kBoxX;
  L.xl = off;
  off += kSlots * kBoxX;
  L.b = off;
  off += kNkbW * kBoxBW;
  L.r = off;
  off += kRAtom;  // one 64-column atom: [r hi 16 | s 16 | r lo 16 | unused 16]
  L.bars = off;
  off += 256;
  L.total = off + 1024;
  return L;
}

// 4 consecutive FP32 TMEM columns of this warp's 32 lanes, three times, then
// one wait in the same asm statement.
__device__ __forceinline__ void tmem_ld4x3(uint32_t ta, uint32_t tb, uint32_t tc, float (&a)[4],
                                           float (&b)[4], float (&c)[4]) {
  uint32_t r[12];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%12];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%4, %5, %6, %7}, [%13];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%8, %9, %10, %11}, [%14];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11])
      : "r"(ta), "r"(tb), "r"(tc)
      : "memory");
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    a[i] = __uint_as_float(r[i]);
    b[i] = __uint_as_float(r[4 + i]);
    c[i] = __uint_as_float(r[8 + i]);
  }
}

// 16 consecutive FP32 TMEM columns of this warp's 32 lanes, twice, one wait.
__device__ __forceinline__ void tmem_ld16x2(uint32_t ta, uint32_t tb, float (&a)[16],
                                            float (&b)[16]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%32];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, "
      "%26, %27, %28, %29, %30, %31}, [%33];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(ta), "r"(tb)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    a[i] = __uint_as_float(r[i]);
    b[i] = __uint_as_float(r[16 + i]);
  }
}

__global__ void __launch_bounds__(kThreadsTC, 1)
    logistic_pass_tc_wide_kernel(const __grid_constant__ CUtensorMap tmXh,
                                 const __grid_constant__ CUtensorMap tmXl,
                                 const __grid_constant__ CUtensorMap tmBh,
                                 const __grid_constant__ CUtensorMap tmBl,
                                 const __grid_constant__ CUtensorMap tmBt,
                                 const float* __restrict__ ylab, int64_t N, int64_t T,
                                 int64_t Dp, float* __restrict__ G, double* __restrict__ lp,
                                 int has_tangent, int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  const LayoutW Ly = layout_wide();
  unsigned char* sXh = base + Ly.xh;
  unsigned char* sXl = base + Ly.xl;
  unsigned char* sB = base + Ly.b;
  unsigned char* sR = base + Ly.r;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + Ly.bars);
  uint64_t* bar_b = bars + 0;   // B loaded
  uint64_t* bar_x = bars + 1;   // [4] slot loaded
  uint64_t* bar_f = bars + 5;   // [4] the MMAs reading the slot are done
  uint64_t* bar_l = bars + 9;   // GEMM1 done (L ready; also GEMM2 of the block before: R free)
  uint64_t* bar_r = bars + 10;  // epilogue wrote R (32 kEpi arrivals)
  uint64_t* bar_g = bars + 11;  // GEMM2 of the block done (G final after the last block)
  uint64_t* bar_z = bars + 12;  // teardown drain
  __shared__ uint32_t s_tmem;
  constexpr int BH = BTW / kParts;  // 4 value columns a thread
  __shared__ double s_red[kEpi][BH];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * BTW;
  const int nblocks = static_cast<int>((N + BN - 1) / BN);
  const bool has_g = has_tangent != 0;

  if (threadIdx.x == 0) {
    for (int i = 0; i < 13; ++i) mbar_init(bars + i, i == 10 ? 32 * kEpi : 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kProd) tmem_alloc(&s_tmem, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  // L: columns [0, 48) = value (hi*hi + lo*hi) | tangent | value hi*lo;
  // G quarter q: columns [64 (q + 1), 64 (q + 1) + 48), the same three parts.
  const uint32_t tL = tmem;
  auto tG = [&](int q) { return tmem + 64u * static_cast<uint32_t>(q + 1); };

  if (warp == kProd) {
    if (lane == 0) {
      bool ok = true;
      uint32_t xph = 0, fph = 0;  // phase bit of each slot's two barriers
      const uint32_t i1_all = idesc_f16(128, 3 * BTW, false, false);
      const uint32_t i1_v = idesc_f16(128, BTW, false, false);
      const uint32_t i2_all = idesc_f16(128, 3 * BTW, true, true);
      const uint32_t i2_v = idesc_f16(128, BTW, true, true);
      auto wait_x = [&](int s) {
        const bool r = mbar_wait(bar_x + s, (xph >> s) & 1u, err);
        xph ^= 1u << s;
        return r;
      };
      auto wait_f = [&](int s) {
        const bool r = mbar_wait(bar_f + s, (fph >> s) & 1u, err);
        fph ^= 1u << s;
        return r;
      };
      auto load_box = [&](int s, int box, int nb) {
        mbar_expect_tx(bar_x + s, 2 * kBoxX);
        tma_2d(sXh + s * kBoxX, &tmXh, box * 64, nb * BN, bar_x + s);
        tma_2d(sXl + s * kBoxX, &tmXl, box * 64, nb * BN, bar_x + s);
      };
      // GEMM1 over the box in slot s: L += Xh [Bh | Bt | Bl] + Xl Bh
      auto gemm1 = [&](int s, int box) {
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
          const uint64_t ah = sdesc(su32(sXh + s * kBoxX) + ks * 32, 16, 1024, 2);
          const uint64_t al = sdesc(su32(sXl + s * kBoxX) + ks * 32, 16, 1024, 2);
          const uint64_t bb = sdesc(su32(sB + box * kBoxBW) + ks * 32, 16, 1024, 2);
          mma_f16(tL, ah, bb, i1_all, (box | ks) != 0);
          mma_f16(tL, al, bb, i1_v, 1);
        }
      };
      // GEMM2 for d quarter q from the boxes in slots 2p, 2p + 1
      auto gemm2 = [&](int q, int p, int nb) {
        if (!has_g) return;
#pragma unroll
        for (int kn = 0; kn < BN / 16; ++kn) {
          const uint64_t ah = sdesc(su32(sXh + 2 * p * kBoxX) + kn * 2048, kBoxX, 1024, 2);
          const uint64_t al = sdesc(su32(sXl + 2 * p * kBoxX) + kn * 2048, kBoxX, 1024, 2);
          const uint64_t br = sdesc(su32(sR) + kn * 2048, kRAtom, 1024, 2);
          // every row block starts G afresh (the epilogue adds the blocks up)
          const uint32_t acc = kn > 0 ? 1u : 0u;
          mma_f16(tG(q), ah, br, i2_all, acc);
          mma_f16(tG(q), al, br, i2_v, 1);
        }
      };
      mbar_expect_tx(bar_b, kNkbW * kBoxBW);
      for (int kb = 0; kb < kNkbW; ++kb) {
        unsigned char* b = sB + kb * kBoxBW;
        tma_2d(b, &tmBh, kb * 64, static_cast<int>(t0), bar_b);
        tma_2d(b + BTW * 128, has_tangent ? &tmBt : &tmBh, kb * 64, static_cast<int>(t0), bar_b);
        tma_2d(b + 2 * BTW * 128, &tmBl, kb * 64, static_cast<int>(t0), bar_b);
      }
      ok = mbar_wait(bar_b, 0, err);
      if (ok)
        for (int s = 0; s < kSlots; ++s) load_box(s, s, 0);
      for (int nb = 0; nb < nblocks && ok; ++nb) {
        // GEMM1, boxes 0-3
        for (int s = 0; s < kSlots && ok; ++s) {
          if (!(ok = wait_x(s))) break;
          tc_fence_after();
          gemm1(s, s);
          mma_commit(bar_f + s);
        }
        // boxes 4-7 into the slots as they free, then their GEMM1
        for (int s = 0; s < kSlots && ok; ++s) {
          if (!(ok = wait_f(s))) break;
          load_box(s, kSlots + s, nb);
        }
        for (int s = 0; s < kSlots && ok; ++s) {
          if (!(ok = wait_x(s))) break;
          tc_fence_after();
          gemm1(s, kSlots + s);
        }
        if (!ok) break;
        mma_commit(bar_l);
        if (!(ok = mbar_wait(bar_r, nb & 1, err))) break;
        tc_fence_after();
        // GEMM2, quarters 2 and 3 from the resident boxes 4-7
        for (int p = 0; p < 2; ++p) {
          gemm2(2 + p, p, nb);
          mma_commit(bar_f + 2 * p);
          mma_commit(bar_f + 2 * p + 1);
        }
        // boxes 0-3 again, then quarters 0 and 1
        for (int s = 0; s < kSlots && ok; ++s) {
          if (!(ok = wait_f(s))) break;
          load_box(s, s, nb);
        }
        for (int p = 0; p < 2 && ok; ++p) {
          if (!(ok = wait_x(2 * p)) || !(ok = wait_x(2 * p + 1))) break;
          tc_fence_after();
          gemm2(p, p, nb);
          mma_commit(bar_f + 2 * p);
          mma_commit(bar_f + 2 * p + 1);
        }
        if (!ok) break;
        mma_commit(bar_g);
        // the next block's boxes 0-3
        if (nb + 1 < nblocks)
          for (int s = 0; s < kSlots && ok; ++s) {
            if (!(ok = wait_f(s))) break;
            load_box(s, s, nb + 1);
          }
      }
      if (!ok) atomicExch(err, 1);
      // drain every MMA this thread issued before TMEM is released
      mma_commit(bar_z);
      if (!mbar_wait(bar_z, 0, err)) atomicExch(err, 1);
    }
    __syncwarp();
  } else {
    // ---- epilogue: thread = TMEM lane = data row; warp part = 4 value columns ----
    const int quarter = warp & 3, part = warp >> 2;  // columns [4 part, 4 part + 4)
    const int row = quarter * 32 + lane;
    const uint32_t lane_off = static_cast<uint32_t>(quarter * 32) << 16;
    float ls[BH], lc[BH];
#pragma unroll
    for (int t = 0; t < BH; ++t) ls[t] = lc[t] = 0.f;
    bool ok = true;
    float y_next = row < N ? __ldg(ylab + row) : 0.f;
    // part q owns d quarter q of G: the row blocks' partial sums of its value
    // (hi*lo added) and tangent columns, added in FP32 with round-to-nearest
    float gv[BTW], gt[BTW];
#pragma unroll
    for (int t = 0; t < BTW; ++t) gv[t] = gt[t] = 0.f;
    auto add_g = [&]() {
      float a[16], b[16], c[16], unused[16];
      tmem_ld16x2(tG(part) + lane_off, tG(part) + lane_off + 2 * BTW, a, b);
      tmem_ld16x2(tG(part) + lane_off + BTW, tG(part) + lane_off + BTW, c, unused);
#pragma unroll
      for (int t = 0; t < BTW; ++t) {
        gv[t] += a[t] + b[t];
        gt[t] += c[t];
      }
    };
    for (int nb = 0; nb < nblocks; ++nb) {
      const int64_t n = static_cast<int64_t>(nb) * BN + row;
      const bool valid = n < N;
      const float yn = y_next;
      if (n + BN < N) y_next = __ldg(ylab + n + BN);
      if (has_g && nb > 0) {
        // the previous block's G partials, final at its GEMM2's commit and kept
        // until this block's R arrives: added while this block's GEMM1 runs
        if (!(ok = mbar_wait(bar_g, (nb - 1) & 1, err))) break;
        tc_fence_after();
        add_g();
      }
      if (!(ok = mbar_wait(bar_l, nb & 1, err))) break;
      tc_fence_after();
      float v[BH], vl[BH], w[BH];
      tmem_ld4x3(tL + lane_off + BH * part, tL + lane_off + 2 * BTW + BH * part,
                 tL + lane_off + BTW + BH * part, v, vl, w);
      float r[BH], sv[BH];
#pragma unroll
      for (int t = 0; t < BH; ++t) {
        const float l = v[t] + vl[t];
        const float e = __expf(-fabsf(l));
        const float inv = __fdividef(1.f, 1.f + e);
        const float p = l >= 0.f ? inv : e * inv;
        r[t] = valid ? yn - p : 0.f;
        sv[t] = (valid && has_tangent) ? p * (1.f - p) * w[t] : 0.f;
        if (valid) {
          const float y = (yn * l - (fmaxf(l, 0.f) + log1p_unit(e))) - lc[t];
          const float sum = ls[t] + y;
          lc[t] = (sum - ls[t]) - y;
          ls[t] = sum;
        }
      }
      if (has_g) {
        uint32_t wh[2], wl[2], ws[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const float h0 = split_hi(r[2 * q]), h1 = split_hi(r[2 * q + 1]);
          wh[q] = half2_bits(h0, h1);
          wl[q] = half2_bits(r[2 * q] - h0, r[2 * q + 1] - h1);
          ws[q] = half2_bits(sv[2 * q], sv[2 * q + 1]);
        }
        // 8-column chunks: r hi 0-1, s 2-3, r lo 4-5; this part's half chunk
        unsigned char* rrow = sR + row * 128 + (part & 1) * 8;
        const int sw = row & 7, c = part >> 1;
        *reinterpret_cast<uint2*>(rrow + ((c ^ sw) << 4)) = make_uint2(wh[0], wh[1]);
        *reinterpret_cast<uint2*>(rrow + (((2 + c) ^ sw) << 4)) = make_uint2(ws[0], ws[1]);
        *reinterpret_cast<uint2*>(rrow + (((4 + c) ^ sw) << 4)) = make_uint2(wl[0], wl[1]);
        fence_async_smem();
      }
      tc_fence_before();
      mbar_arrive(bar_r);
    }
    if (ok && has_g && mbar_wait(bar_g, (nblocks - 1) & 1, err)) {
      tc_fence_after();
      add_g();  // the last row block
      const int64_t d = 128 * part + row;
      if (d < Dp) {
#pragma unroll
        for (int t = 0; t < BTW; ++t)
          if (t0 + t < T) {
            G[(t0 + t) * Dp + d] = gv[t];
            G[(T + t0 + t) * Dp + d] = gt[t];
          }
      }
    } else if (!ok) {
      atomicExch(err, 1);
    }
#pragma unroll
    for (int t = 0; t < BH; ++t) {
      const double sum = warp_sum(static_cast<double>(ls[t]) - static_cast<double>(lc[t]));
      if (lane == 0) s_red[warp][t] = sum;
    }
    asm volatile("bar.sync 1, %0;" ::"n"(32 * kEpi) : "memory");
    if (threadIdx.x < BTW && t0 + threadIdx.x < T) {
      const int t = threadIdx.x, hh = t / BH, tt = t % BH;
      double a = 0.0;
      for (int q = 0; q < 4; ++q) a += s_red[4 * hh + q][tt];
      lp[t0 + t] = a;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kProd) tmem_dealloc(tmem, 512);
}

// Bound check of the mbarrier wait used by the tensor-core pass: one thread
// initialises a barrier that expects one arrival, nobody arrives, and the
// bounded wait on phase 0 gives up after kWaitCycles; err[0] = 1 then.
__global__ void mbar_bound_kernel(int* err) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_err;
  if (threadIdx.x == 0) {
    s_err = 0;
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) err[0] = mbar_wait(&bar, 0, &s_err) ? 0 : 1;
}

}  // namespace tc


// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 2-D FP16 tensor (rows x cols, row-major) with a 64 x box_rows box, 128-B swizzle.
static bool make_map(CUtensorMap* m, const void* ptr, uint64_t rows, uint64_t cols,
                     uint32_t box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {cols * 2};
  const cuuint32_t box[2] = {64, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(ptr), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

bool lg_tc_supported(const LogisticDev& X) { return X.Xh != nullptr && encode_fn() != nullptr; }

size_t lg_tc_ws_bytes(const LogisticDev& X, int64_t T) {
  return 3 * static_cast<size_t>(T) * X.Dk * 2 + 1024;
}

int* lg_tc_err_word(void* ws, const LogisticDev& X, int64_t T) {
  return reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(ws) + 3 * T * X.Dk * 2);
}

int lg_tc_pass(cudaStream_t s, const LogisticDev& X, const DevParams* dP, const DevState* dS,
               double* lp, int mode, int64_t T, void* ws, float* G_out, int probe) {
  const int64_t Dk = X.Dk;
  __half* Bh = static_cast<__half*>(ws);
  __half* Bl = Bh + T * Dk;
  __half* Bt = Bl + T * Dk;
  float* G = G_out;
  int* err = lg_tc_err_word(ws, X, T);
  const int g = static_cast<int>((T * Dk + 255) / 256 < 148 * 16 ? (T * Dk + 255) / 256 : 148 * 16);
  tc::tc_prep_kernel<float><<<g, 256, 0, s>>>(dP, dS, mode, probe, Dk, Bh, Bl, Bt);
  if (cudaGetLastError() != cudaSuccess) return 3;
  CUtensorMap mXh, mXl, mBh, mBl, mBt;
  if (!make_map(&mXh, X.Xh, X.Np, Dk, tc::BN) || !make_map(&mXl, X.Xl, X.Np, Dk, tc::BN) ||
      !make_map(&mBh, Bh, T, Dk, tc::BT) || !make_map(&mBl, Bl, T, Dk, tc::BT) ||
      !make_map(&mBt, Bt, T, Dk, tc::BT))
    return 3;
  if (Dk == 512) {  // 256 < D <= 512: the wide variant, 16 value columns a CTA
    CUtensorMap wBh, wBl, wBt;
    if (!make_map(&wBh, Bh, T, Dk, tc::BTW) || !make_map(&wBl, Bl, T, Dk, tc::BTW) ||
        !make_map(&wBt, Bt, T, Dk, tc::BTW))
      return 3;
    const uint32_t smem = tc::layout_wide().total;
    if (raise_smem_limit(reinterpret_cast<const void*>(tc::logistic_pass_tc_wide_kernel), smem) !=
        cudaSuccess)
      return 3;
    const int grid = static_cast<int>((T + tc::BTW - 1) / tc::BTW);
    tc::logistic_pass_tc_wide_kernel<<<grid, tc::kThreadsTC, smem, s>>>(
        mXh, mXl, wBh, wBl, wBt, X.y32, X.N, T, X.Dp, G, lp, mode != 2 ? 1 : 0, err);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
  }
  const int nkb = static_cast<int>(Dk / 64);
  const tc::Layout Ly = tc::layout(nkb);
  raise_smem_limit(reinterpret_cast<const void*>(tc::logistic_pass_tc_kernel), tc::layout(4).total);
  const int grid = static_cast<int>((T + tc::BT - 1) / tc::BT);
  tc::logistic_pass_tc_kernel<<<grid, tc::kThreadsTC, Ly.total, s>>>(
      mXh, mXl, mBh, mBl, mBt, X.y32, X.N, nkb, T, X.Dp, G, lp, mode != 2 ? 1 : 0, err);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

cudaError_t lg_tc_mbar_bound(cudaStream_t s, int* err) {
  tc::mbar_bound_kernel<<<1, 32, 0, s>>>(err);
  return cudaGetLastError();
}

}  // namespace pmcmc
