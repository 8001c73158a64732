// tape_scan.cu -- tape materialisation and the standalone diagonal affine scan.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <unordered_map>

#include "deer_device.cuh"
#include "deer_launch.h"

namespace pmcmc {

// Tape block of (seed, block): Xi (D x T, column-major) and u (T)
// (counterpart of _make_mala_tape_block, interface.jl:334-358).
__global__ void tape_kernel(int64_t D, int64_t T, uint64_t seed, uint64_t block, float* Xi,
                            float* u) {
  const int64_t nq = (D + 3) / 4;
  const int64_t n = nq * T;
  const TapeKey key(seed, block);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = i / nq, j = i % nq;
    float v[4];
    tape_xi4(key, static_cast<uint32_t>(j), static_cast<uint32_t>(t), v);
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (4 * j + e < D) Xi[t * D + 4 * j + e] = v[e];
    if (j == 0 && u) u[t] = tape_u(key, static_cast<uint32_t>(t));
  }
}

cudaError_t launch_tape(cudaStream_t s, int64_t D, int64_t T, uint64_t seed, uint64_t block,
                        float* Xi, float* u) {
  const int64_t n = ((D + 3) / 4) * T;
  if (n == 0) return cudaSuccess;
  const int grid = static_cast<int>(imin64((n + 255) / 256, 148 * 16));
  tape_kernel<<<grid, 256, 0, s>>>(D, T, seed, block, Xi, u);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// S[:,t] = A[:,t] .* S[:,t-1] + B[:,t] (solve_affine_scan_diag!, DEERScan.jl:102-173)
// as one pass: each CTA stages a tile of TT columns, scans it in shared memory,
// and obtains the state entering the tile by decoupled look-back.  HBM traffic
// is one read of A and B and one write of S.
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void __launch_bounds__(kThreads)
    affine_scan_kernel(int64_t D, int64_t T, int TT, const Real* __restrict__ A,
                       const Real* __restrict__ B, const Real* __restrict__ s0,
                       Real* __restrict__ S, ScanScratch scr, uint32_t epoch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_tile, s_err, s_jstar;
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_tile = static_cast<int>(atomicAdd(scr.counter, 1u));
    s_err = 0;
  }
  __syncthreads();
  const int tile = s_tile;
  const int Di = static_cast<int>(D);
  const int64_t t0 = static_cast<int64_t>(tile) * TT;
  const int ncols = static_cast<int>(imin64(TT, T - t0));
  Real* As = reinterpret_cast<Real*>(smem_raw);
  Real* Bs = As + static_cast<size_t>(TT) * Di;
  Real* carry = Bs + static_cast<size_t>(TT) * Di;
  const int64_t base = t0 * D, n = static_cast<int64_t>(ncols) * D;
  for (int64_t i = tid; i < n; i += kThreads) {
    As[i] = A[base + i];
    Bs[i] = B[base + i];
  }
  __syncthreads();
  tile_scan_inplace<Real>(As, Bs, ncols, Di, Di);
  __syncthreads();
  Real* agg_a = static_cast<Real*>(scr.agg_a);
  Real* agg_b = static_cast<Real*>(scr.agg_b);
  Real* incl = static_cast<Real*>(scr.incl);
  const size_t last = static_cast<size_t>(ncols - 1) * Di;
  if (tile == 0) {
    for (int d = tid; d < Di; d += kThreads) {
      carry[d] = s0[d];
      incl[d] = As[last + d] * s0[d] + Bs[last + d];
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) st_release(scr.flags, (epoch << 2) | kFlagIncl);
  } else {
    for (int d = tid; d < Di; d += kThreads) {
      agg_a[static_cast<size_t>(tile) * Di + d] = As[last + d];
      agg_b[static_cast<size_t>(tile) * Di + d] = Bs[last + d];
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) st_release(scr.flags + tile, (epoch << 2) | kFlagAgg);
    if ((tid >> 5) == 0) {
      int err = 0;
      const int js = lookback_fixed(tile, epoch, scr.flags, &err);
      if (tid == 0) {
        s_jstar = js;
        if (err) s_err = 1;
      }
    }
    __syncthreads();
    const int js = s_jstar;
    for (int d = tid; d < Di; d += kThreads) {
      const Real c = js >= 0 ? lookback_compose<Real>(tile, js, d, Di, agg_a, agg_b, incl)
                             : Real(0);
      carry[d] = c;
      incl[static_cast<size_t>(tile) * Di + d] = As[last + d] * c + Bs[last + d];
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) st_release(scr.flags + tile, (epoch << 2) | kFlagIncl);
  }
  __syncthreads();
  for (int64_t i = tid; i < n; i += kThreads) {
    const int d = static_cast<int>(i % D);
    S[base + i] = As[i] * carry[d] + Bs[i];
  }
  if (tid == 0 && s_err) atomicExch(scr.counter + 1, 1u);  // timeout flag
}

cudaError_t raise_smem_limit(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::unordered_map<const void*, size_t> limit;
  // (also below 48 KB: static plus dynamic shared memory above 48 KB needs the
  // opt-in even when the dynamic part alone is under it)
  if (bytes == 0) return cudaSuccess;
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = limit[fn];
  if (bytes <= cur) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(bytes));
  if (e == cudaSuccess) cur = bytes;
  return e;
}

int scan_tile_cols(int64_t D, int64_t T) {
  // Largest power of two <= 64 whose tile (A, B, carry) fits 96 KB, reduced
  // while that leaves fewer than ~2 tiles per SM.
  int TT = 64;
  while (TT > 1 && static_cast<int64_t>(2 * TT + 1) * D * 8 > 96 * 1024) TT >>= 1;
  while (TT > 8 && (T + TT - 1) / TT < 296) TT >>= 1;
  return TT;
}

size_t scan_scratch_bytes(bool f64, int64_t D, int64_t T) {
  const int TT = scan_tile_cols(D, T);
  const int64_t nt = (T + TT - 1) / TT;
  const size_t es = f64 ? 8 : 4;
  return 256 + 4 * static_cast<size_t>(nt) + 3 * es * static_cast<size_t>(nt * D) + 64;
}

cudaError_t launch_affine_scan(cudaStream_t s, bool f64, int64_t D, int64_t T, const void* A,
                               const void* B, const void* s0, void* S, const ScanScratch& scr,
                               uint32_t epoch) {
  if (T == 0 || D == 0) return cudaSuccess;
  const int TT = scan_tile_cols(D, T);
  const int ntiles = static_cast<int>((T + TT - 1) / TT);
  const size_t es = f64 ? 8 : 4;
  const size_t smem = es * (2 * static_cast<size_t>(TT) + 1) * D;
  cudaError_t e = cudaMemsetAsync(scr.counter, 0, 2 * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  if (f64) {
    if (smem > 0)
      raise_smem_limit(reinterpret_cast<const void*>(affine_scan_kernel<double>), smem);
    affine_scan_kernel<double><<<ntiles, kThreads, smem, s>>>(
        D, T, TT, static_cast<const double*>(A), static_cast<const double*>(B),
        static_cast<const double*>(s0), static_cast<double*>(S), scr, epoch);
  } else {
    if (smem > 0)
      raise_smem_limit(reinterpret_cast<const void*>(affine_scan_kernel<float>), smem);
    affine_scan_kernel<float><<<ntiles, kThreads, smem, s>>>(
        D, T, TT, static_cast<const float*>(A), static_cast<const float*>(B),
        static_cast<const float*>(s0), static_cast<float*>(S), scr, epoch);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Plain path: Hillis-Steele doubling scan, one launch per level
// (DEERScan.jl:135-171), then damping and the metric reductions.
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void doubling_level_kernel(int64_t Dp, int64_t T, int64_t off,
                                      const Real* __restrict__ al, const Real* __restrict__ be,
                                      Real* __restrict__ aln, Real* __restrict__ ben) {
  const int64_t n = T * Dp;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = i / Dp;
    if (t >= off) {
      const Real a2 = al[i];
      aln[i] = a2 * al[i - off * Dp];
      ben[i] = a2 * be[i - off * Dp] + be[i];
    } else {
      aln[i] = al[i];
      ben[i] = be[i];
    }
  }
}

template <typename Real>
__global__ void doubling_apply_kernel(int64_t Dp, int64_t T, const Real* __restrict__ al,
                                      const Real* __restrict__ be, const Real* __restrict__ s0,
                                      Real* __restrict__ S) {
  const int64_t n = T * Dp;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    S[i] = al[i] * s0[i % Dp] + be[i];
}

template <typename Real>
__global__ void damp_metric_kernel(int64_t D, int64_t Dp, int64_t T, const Real* __restrict__ So,
                                   Real* __restrict__ Sn, double damping,
                                   unsigned long long* red) {
  const int64_t n = T * Dp;
  double dm = 0, sm = 0;
  bool bad = false;
  const Real dmp = static_cast<Real>(damping), omd = static_cast<Real>(1.0 - damping);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (i % Dp >= D) continue;
    Real v = Sn[i];
    if (damping != 1.0) {
      v = omd * So[i] + dmp * v;
      Sn[i] = v;
    }
    dm = max(dm, static_cast<double>(fabs(v - So[i])));
    sm = max(sm, static_cast<double>(fabs(v)));
    bad |= !isfinite(v);
  }
  dm = warp_max(dm);
  sm = warp_max(sm);
  if ((threadIdx.x & 31) == 0) {
    if (dm > 0) atomicMax(red, dbits(dm));
    if (sm > 0) atomicMax(red + 1, dbits(sm));
    if (bad) atomicExch(red + 2, 1ull);
  }
}

cudaError_t launch_doubling_scan(cudaStream_t s, bool f64, int64_t Dp, int64_t T, const void* A,
                                 const void* B, const void* s0, void* S, void* al0, void* be0,
                                 void* al1, void* be1) {
  const int64_t n = T * Dp;
  const int grid = static_cast<int>(imin64((n + 255) / 256, 148 * 8));
  const void* al = A;
  const void* be = B;
  void* bufs[2][2] = {{al0, be0}, {al1, be1}};
  int which = 0;
  for (int64_t off = 1; off < T; off <<= 1, which ^= 1) {
    if (f64)
      doubling_level_kernel<double><<<grid, 256, 0, s>>>(
          Dp, T, off, static_cast<const double*>(al), static_cast<const double*>(be),
          static_cast<double*>(bufs[which][0]), static_cast<double*>(bufs[which][1]));
    else
      doubling_level_kernel<float><<<grid, 256, 0, s>>>(
          Dp, T, off, static_cast<const float*>(al), static_cast<const float*>(be),
          static_cast<float*>(bufs[which][0]), static_cast<float*>(bufs[which][1]));
    al = bufs[which][0];
    be = bufs[which][1];
  }
  if (f64)
    doubling_apply_kernel<double><<<grid, 256, 0, s>>>(Dp, T, static_cast<const double*>(al),
                                                       static_cast<const double*>(be),
                                                       static_cast<const double*>(s0),
                                                       static_cast<double*>(S));
  else
    doubling_apply_kernel<float><<<grid, 256, 0, s>>>(Dp, T, static_cast<const float*>(al),
                                                      static_cast<const float*>(be),
                                                      static_cast<const float*>(s0),
                                                      static_cast<float*>(S));
  return cudaGetLastError();
}

cudaError_t launch_damp_metric(cudaStream_t s, bool f64, int64_t D, int64_t Dp, int64_t T,
                               const void* S_old, void* S_new, double damping,
                               unsigned long long* red) {
  const int64_t n = T * Dp;
  const int grid = static_cast<int>(imin64((n + 255) / 256, 148 * 8));
  cudaError_t e = cudaMemsetAsync(red, 0, 3 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  if (f64)
    damp_metric_kernel<double><<<grid, 256, 0, s>>>(D, Dp, T, static_cast<const double*>(S_old),
                                                    static_cast<double*>(S_new), damping, red);
  else
    damp_metric_kernel<float><<<grid, 256, 0, s>>>(D, Dp, T, static_cast<const float*>(S_old),
                                                   static_cast<float*>(S_new), damping, red);
  return cudaGetLastError();
}

template <typename Real>
__global__ void broadcast_kernel(int64_t Dp, int64_t T, const Real* __restrict__ x0,
                                 Real* __restrict__ S) {
  const int64_t n = T * Dp;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    S[i] = x0[i % Dp];
}

cudaError_t launch_broadcast(cudaStream_t s, bool f64, int64_t Dp, int64_t T, const void* x0,
                             void* S) {
  const int64_t n = T * Dp;
  const int grid = static_cast<int>(imin64((n + 255) / 256, 148 * 8));
  if (f64)
    broadcast_kernel<double><<<grid, 256, 0, s>>>(Dp, T, static_cast<const double*>(x0),
                                                  static_cast<double*>(S));
  else
    broadcast_kernel<float><<<grid, 256, 0, s>>>(Dp, T, static_cast<const float*>(x0),
                                                 static_cast<float*>(S));
  return cudaGetLastError();
}

// Bound check of the look-back wait: one warp looks back from tile 1 over a
// flag array that nothing publishes (all zeros: no epoch, no state), so lane 0
// spins on tile 0 until kMaxSpins and the warp reports the give-up in err[0].  The same
// routine guards every scan and sweep launch.
__global__ void lookback_bound_kernel(const uint32_t* flags, int* err) {
  int e = 0;
  lookback_fixed(1, 1u, flags, &e);
  if (threadIdx.x == 0) err[0] = e;
}

cudaError_t launch_lookback_bound(cudaStream_t s, const uint32_t* flags, int* err) {
  lookback_bound_kernel<<<1, 32, 0, s>>>(flags, err);
  return cudaGetLastError();
}

}  // namespace pmcmc
