// deer_device.cuh -- device-resident solve parameters/state and the shared
// building blocks of the DEER sweep: warp reductions, tile-local affine scan
// and the decoupled look-back across tiles.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "pmcmc_rng.cuh"

namespace pmcmc {

constexpr int kThreads = 256;  // threads per CTA of the sweep / scan kernels
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kFlagAgg = 1u, kFlagIncl = 2u;
constexpr long long kMaxSpins = 1ll << 22;  // bounded look-back wait (~0.3 s), then error

enum TargetKind : int32_t { kDiagGauss = 0, kDenseGauss = 1, kLogistic = 2 };
enum JacKind : int32_t { kJacStoch = 0, kJacDiag = 1, kJacFull = 2 };
enum DevStatus : int32_t { kStOk = 0, kStNonfinite = 4, kStTimeout = 5 };

// Everything a solve needs, resident in device memory so that one captured
// CUDA graph serves every call (kernels copy it to shared memory on entry).
struct DevState;

struct DevParams {
  int64_t D, Dp, T, W;  // Dp = D rounded up to 4; W = window width (T if none)
  int64_t ncols_out;    // columns copied to S_out by the finalize pass
  double eps, sqrt2eps, inv4eps, inv2eps, damping, tol_abs, tol_rel;
  uint64_t seed, block;
  int32_t jac, probes, maxiter, tile_cols;
  int32_t ntiles, tkind, out_device;
  int32_t t_off;  // tape column of local column 0 (a slice of the block; 0 otherwise)
  // target (device copies, both precisions)
  const double* mean_d;
  const double* prec_d;
  const float* mean_f;
  const float* prec_f;
  // trajectory ping-pong buffers and start state (Real)
  void* S[2];
  const void* x0;
  // look-back scratch
  uint32_t* flags;  // [ntiles]
  void* agg_a;      // [ntiles * Dp]
  void* agg_b;
  void* incl;
  float* colmax;  // [T] per-column max |dS| (window mode)
  // outputs
  void* S_out;
  void* logp_out;
  uint8_t* accept_out;
  void* x_next;  // [D] last kept column (next block's x0)
  // logistic target: per-column quantities produced by the two GEMM passes
  // (T x Dp, Real): g_x, y, w = z + eps H(x) z, g_y, H(y) w; likelihood sums
  // lpx/lpy (T, FP64); the sweep records accept flags and log-alpha per column.
  void* lg[5];
  double* lpx;
  double* lpy;
  uint8_t* acc_col;
  double* la_col;
  // log alpha of every column with near-tie columns recomputed in FP64
  // (logistic_tie.cu); nullptr: the sweep forms log alpha itself
  const double* la_ref;
  // probes > 1: sum of z_k .* J z_k over the probes 0 .. probes-2 of the sweep (T x Dp, Real)
  void* lg_acc;
  // error word of the tensor-core pass (a bounded wait gave up), or nullptr
  const int* tc_err;
  double tau;  // prior precision
  // tape of the block, written once by the init kernel: xi (T x Dp, FP32,
  // padded rows zero) and log(u_t) in FP64
  float* xi;
  double* logu;
  // persistent solve (deer_persist.cu)
  double* part;         // [2 * ntiles * 4] per-CTA partial reductions
  const void* x0_src;   // start state as given (D entries, unpadded), or nullptr: use x0
  DevState* st_host;    // pinned host copy of the final state (nullptr: none)
  // blocks solved back to back in one persistent launch (0 or 1: one).  Block b
  // is tape block `block + b`, starts from block b - 1's x_next, writes its
  // rows at S_out + b T D (logp, accept: + b T) and its state to st_host[b];
  // ncols_out is then the last block's kept columns (the others keep T).
  int64_t nblk;
};

struct DevState {
  int32_t iter, cur, converged, status;
  int64_t t_lo, t_lo_prev;
  uint32_t epoch, tile_counter, done_counter, fin_counter;
  unsigned long long dmax_bits, smax_bits;  // non-negative doubles as ordered bits
  double metric;
  unsigned long long n_accept;
  unsigned long long min_margin_bits, max_defect_bits;
};

__host__ __device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int64_t imax64(int64_t a, int64_t b) { return a > b ? a : b; }

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Sum / max over aligned groups of W lanes (W a power of two <= 32); every
// lane of the warp takes part.
template <int W, typename T>
__device__ __forceinline__ T seg_sum(T v) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <int W, typename T>
__device__ __forceinline__ T seg_max(T v) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ unsigned long long dbits(double v) {
  return static_cast<unsigned long long>(__double_as_longlong(v));
}
__device__ __forceinline__ double bitsd(unsigned long long b) {
  return __longlong_as_double(static_cast<long long>(b));
}

// Inclusive scan of the affine maps x -> A[c][d] x + B[c][d] along c (columns
// 0..ncols-1 of a tile), independently for every coordinate d, in place.
// After the call (A[c][d], B[c][d]) is the composition of columns 0..c.
// Threads own (d, chunk) pairs: a serial scan inside each chunk, then each
// chunk is offset by the composition of the chunks before it.
template <typename Real>
__device__ void tile_scan_inplace(Real* As, Real* Bs, int ncols, int D, int Dp) {
  const int tid = threadIdx.x, nt = blockDim.x;
  if (ncols <= 0) return;
  int C = D >= nt ? 1 : min(nt / D, ncols);
  const int L = (ncols + C - 1) / C;
  C = (ncols + L - 1) / L;
  for (int base = 0; base < D * C; base += nt) {
    const int k = base + tid;
    if (k < D * C) {
      const int d = k % D, ch = k / D;
      const int c0 = ch * L, c1 = min(ncols, c0 + L);
      Real a = As[c0 * Dp + d], b = Bs[c0 * Dp + d];
      for (int c = c0 + 1; c < c1; ++c) {
        const Real ac = As[c * Dp + d], bc = Bs[c * Dp + d];
        b = ac * b + bc;
        a = ac * a;
        As[c * Dp + d] = a;
        Bs[c * Dp + d] = b;
      }
    }
  }
  if (C == 1) return;
  __syncthreads();
  // Exclusive prefix of each chunk from the chunk aggregates (read first, then apply).
  Real ea[4], eb[4];  // up to 4 (d, chunk) items per thread when D*C > nt
  int nitems = 0;
  for (int base = 0; base < D * C; base += nt, ++nitems) {
    const int k = base + tid;
    Real a = 1, b = 0;
    if (k < D * C) {
      const int d = k % D, ch = k / D;
      for (int j = 0; j < ch; ++j) {
        const int e = min(ncols, (j + 1) * L) - 1;
        const Real aj = As[e * Dp + d], bj = Bs[e * Dp + d];
        b = aj * b + bj;
        a = aj * a;
      }
    }
    if (nitems < 4) {
      ea[nitems] = a;
      eb[nitems] = b;
    }
  }
  __syncthreads();
  nitems = 0;
  for (int base = 0; base < D * C; base += nt, ++nitems) {
    const int k = base + tid;
    if (k < D * C && nitems < 4) {
      const int d = k % D, ch = k / D;
      if (ch == 0) continue;
      const int c0 = ch * L, c1 = min(ncols, c0 + L);
      for (int c = c0; c < c1; ++c) {
        const Real ac = As[c * Dp + d];
        Bs[c * Dp + d] = ac * eb[nitems] + Bs[c * Dp + d];
        As[c * Dp + d] = ac * ea[nitems];
      }
    }
  }
}

// Decoupled look-back (Merrill & Garland) with a fixed association: `tile`
// composes the aggregates of the tiles (jd, tile) onto the inclusive state of
// jd, the last tile of the previous group of 32 (tile 0 for the first group).  The composition, and so
// the FP rounding, is the same in every run, whichever tile finished first.
// Lane l of warp 0 waits for tile jd + l (its inclusive state for l = 0, its
// aggregate otherwise).  Waits are bounded: on timeout *err = 1 and -1 is
// returned (the caller records the error and carries on, never hangs).
constexpr int kLookGroup = 32;
__device__ __forceinline__ int lookback_fixed(int tile, uint32_t epoch, const uint32_t* flags,
                                              int* err) {
  const int lane = threadIdx.x & 31;
  const uint32_t ep = epoch & 0x3fffffffu;
  const int jd = tile < kLookGroup ? 0 : (tile / kLookGroup) * kLookGroup - 1;
  const int j = jd + lane;
  bool timeout = false;
  if (j < tile) {
    const uint32_t need = lane == 0 ? kFlagIncl : kFlagAgg;
    long long spins = 0;
    while (true) {
      const uint32_t f = ld_acquire(flags + j);
      if ((f >> 2) == ep && (f & 3u) >= need) break;
      if (++spins > kMaxSpins) {
        timeout = true;
        break;
      }
      if (spins > 16) __nanosleep(32);
    }
  }
  if (__any_sync(0xffffffffu, timeout)) {
    *err = 1;
    return -1;
  }
  return jd;
}

// State entering `tile` for coordinate d: the aggregates of tiles (jstar, tile)
// composed onto the inclusive state of jstar.  The loads are independent of
// the composition chain, so they are issued ahead of it.
template <typename Real>
__device__ __forceinline__ Real lookback_compose(int tile, int jstar, int d, int Dp,
                                                 const Real* agg_a, const Real* agg_b,
                                                 const Real* incl) {
  Real a = 1, b = 0;
#pragma unroll 4
  for (int j = tile - 1; j > jstar; --j) {
    const Real aj = __ldcg(agg_a + static_cast<size_t>(j) * Dp + d);
    const Real bj = __ldcg(agg_b + static_cast<size_t>(j) * Dp + d);
    b = a * bj + b;
    a = a * aj;
  }
  return a * __ldcg(incl + static_cast<size_t>(jstar) * Dp + d) + b;
}

// Cooperative sweep, phase B: for coordinate d, the state entering every tile
// (exclusive scan of the tile aggregates in tile order, applied to s_lo) by
// one CTA: each thread composes a run of consecutive tiles, a Kogge-Stone scan
// over the 256 run aggregates in shared memory, then each run is replayed.
template <typename Real>
__device__ void carry_scan_tiles_long(int ntiles, int d, int Dp, const Real* __restrict__ agg_a,
                                 const Real* __restrict__ agg_b, Real s_lo,
                                 Real* __restrict__ carry, Real* sa, Real* sb) {
  const int tid = threadIdx.x;
  const int K = (ntiles + kThreads - 1) / kThreads;
  const int j0 = min(ntiles, tid * K), j1 = min(ntiles, j0 + K);
  Real a = 1, b = 0;
  for (int j = j0; j < j1; ++j) {
    const Real aj = __ldcg(agg_a + static_cast<size_t>(j) * Dp + d);
    const Real bj = __ldcg(agg_b + static_cast<size_t>(j) * Dp + d);
    b = aj * b + bj;
    a = aj * a;
  }
  sa[tid] = a;
  sb[tid] = b;
  __syncthreads();
  for (int off = 1; off < kThreads; off <<= 1) {
    Real pa = 1, pb = 0;
    if (tid >= off) {
      pa = sa[tid - off];
      pb = sb[tid - off];
    }
    __syncthreads();
    if (tid >= off) {
      const Real ma = sa[tid], mb = sb[tid];
      sa[tid] = ma * pa;
      sb[tid] = ma * pb + mb;
    }
    __syncthreads();
  }
  Real st = s_lo;
  if (tid > 0) st = sa[tid - 1] * s_lo + sb[tid - 1];
  for (int j = j0; j < j1; ++j) {
    carry[static_cast<size_t>(j) * Dp + d] = st;
    const Real aj = __ldcg(agg_a + static_cast<size_t>(j) * Dp + d);
    const Real bj = __ldcg(agg_b + static_cast<size_t>(j) * Dp + d);
    st = aj * st + bj;
  }
  __syncthreads();
}

// The same for up to 4 tiles a thread (every persistent and cooperative grid
// here): each thread keeps its run's aggregates in registers for the replay,
// and the runs are scanned with warp shuffles, then over the 8 warp totals,
// with two CTA barriers instead of two a Kogge-Stone step.
template <typename Real>
__device__ void carry_scan_tiles(int ntiles, int d, int Dp, const Real* __restrict__ agg_a,
                                 const Real* __restrict__ agg_b, Real s_lo,
                                 Real* __restrict__ carry, Real* sa, Real* sb) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr unsigned kAll = 0xffffffffu;
  constexpr int kRun = 4;  // runs of up to 4 tiles stay in registers for the replay
  const int K = (ntiles + kThreads - 1) / kThreads;
  if (K > kRun) {  // more tiles than kRun a thread: the general form
    carry_scan_tiles_long<Real>(ntiles, d, Dp, agg_a, agg_b, s_lo, carry, sa, sb);
    return;
  }
  const int j0 = min(ntiles, tid * K), j1 = min(ntiles, j0 + K);
  Real ra[kRun], rb[kRun];
#pragma unroll
  for (int k = 0; k < kRun; ++k) {
    const int j = j0 + k;
    const bool in = j < j1;
    ra[k] = in ? __ldcg(agg_a + static_cast<size_t>(j) * Dp + d) : Real(1);
    rb[k] = in ? __ldcg(agg_b + static_cast<size_t>(j) * Dp + d) : Real(0);
  }
  Real a = 1, b = 0;  // this thread's run, composed (identity entries change nothing)
#pragma unroll
  for (int k = 0; k < kRun; ++k) {
    b = ra[k] * b + rb[k];
    a = ra[k] * a;
  }
  // inclusive scan of the runs within the warp (later composed after earlier)
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const Real pa = __shfl_up_sync(kAll, a, off), pb = __shfl_up_sync(kAll, b, off);
    if (lane >= off) {
      b = a * pb + b;
      a = a * pa;
    }
  }
  if (lane == 31) {
    sa[warp] = a;
    sb[warp] = b;
  }
  __syncthreads();
  if (warp == 0) {  // inclusive scan of the warp totals
    Real wa = lane < kWarps ? sa[lane] : Real(1), wb = lane < kWarps ? sb[lane] : Real(0);
#pragma unroll
    for (int off = 1; off < kWarps; off <<= 1) {
      const Real pa = __shfl_up_sync(kAll, wa, off), pb = __shfl_up_sync(kAll, wb, off);
      if (lane >= off) {
        wb = wa * pb + wb;
        wa = wa * pa;
      }
    }
    if (lane < kWarps) {
      sa[kWarps + lane] = wa;
      sb[kWarps + lane] = wb;
    }
  }
  __syncthreads();
  // state entering this thread's run: the earlier warps, then the earlier lanes
  Real st = s_lo;
  if (warp > 0) st = sa[kWarps + warp - 1] * st + sb[kWarps + warp - 1];
  const Real la = __shfl_up_sync(kAll, a, 1), lb = __shfl_up_sync(kAll, b, 1);
  if (lane > 0) st = la * st + lb;
#pragma unroll
  for (int k = 0; k < kRun; ++k) {
    const int j = j0 + k;
    if (j < j1) {
      carry[static_cast<size_t>(j) * Dp + d] = st;
      st = ra[k] * st + rb[k];
    }
  }
  __syncthreads();  // sa / sb are read again by the caller's next use
}

}  // namespace pmcmc
