// mala_chains.cu -- many independent sequential MALA chains on the device, one
// warp a chain (Gaussian device targets).
//
// Chain c runs the taped MALA step of MALA.jl:377-411 (proposal MALA.jl:207-229,
// FP64 log-acceptance, strict log u < log alpha) for T steps from x0_c, with
// the tape of (seed_c, block): the same tape a DEER solve with that seed and
// block reads, so chain c reproduces the trajectory DEER converges to.  This
// is the sequential sampler of the reference run side by side on the GPU: the
// baseline a single DEER chain is compared with, and a source of warm-up
// states.  The chain's state stays in a warp-private shared vector; the tape
// is drawn in registers at every step.
//
// Adaptive mode (AdaptiveMALASampler, src/interface.jl:899-933, 1024-1065): every
// chain carries its own (epsilon, epsilon_bar, H_bar, m).  Step m (0-based)
// uses epsilon while m < n_warmup and epsilon_bar after; during warmup the
// dual-averaging update (_dual_average_update, src/interface.jl:962-984) follows
// each step, fed that step's log alpha.  The step sizes live in the warp's own
// copy of the parameters, which the column code reads; the update runs in FP64
// on every lane alike (log alpha is warp-uniform), so no broadcast is needed.
#include <cuda_runtime.h>

#include <cstdint>

#include "deer_column.cuh"
#include "deer_device.cuh"
#include "deer_launch.h"

namespace pmcmc {

template <typename Real, int TK, int QPL>
__global__ void __launch_bounds__(kThreads)
    mala_chains_kernel(const DevParams Pv, const ChainAdapt ad, int64_t nchains,
                       const Real* __restrict__ x0, const uint64_t* __restrict__ seeds,
                       Real* __restrict__ S, Real* __restrict__ logp,
                       uint8_t* __restrict__ acc_out, double* __restrict__ eps_out,
                       double* __restrict__ state_out) {
  __shared__ DevParams P;
  __shared__ DevParams Pw_all[kWarps];  // per-warp step sizes (adaptive mode)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (threadIdx.x == 0) P = Pv;
  if (threadIdx.x < kWarps) Pw_all[threadIdx.x] = Pv;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  const int64_t T = P.T;
  Smem<Real> sm = carve<Real>(smem_raw, P, 0, TK == kDenseGauss);  // dense: per-warp vectors
  Real* xs = reinterpret_cast<Real*>(smem_raw + plan_sweep_smem<Real>(Dp, 0, TK == kDenseGauss).total) +
             warp * Dp;
  __syncthreads();
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + warp;
  if (c >= nchains) return;  // warp-uniform; no CTA barrier follows
  DevParams& Pw = Pw_all[warp];
  for (int d = lane; d < Dp; d += 32) xs[d] = d < D ? x0[c * D + d] : Real(0);
  __syncwarp();
  const TapeKey key(seeds[c], P.block);
  // dual-averaging state (identical on every lane)
  double eps = P.eps, eps_bar = P.eps, h_bar = 0.0;
  const double mu = log(10.0 * P.eps);
  for (int64_t t = 0; t < T; ++t) {
    const bool warm = ad.active && t < ad.n_warmup;
    const double eps_t = !ad.active ? P.eps : warm ? eps : eps_bar;
    if (ad.active) {
      __syncwarp();  // the previous step's reads of the step sizes are done
      if (lane == 0) {
        Pw.eps = eps_t;
        Pw.sqrt2eps = sqrt(2.0 * eps_t);
        Pw.inv4eps = 1.0 / (4.0 * eps_t);
        Pw.inv2eps = 1.0 / (2.0 * eps_t);
      }
      __syncwarp();
    }
    float xi[QPL][4];
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + 32 * q;
      if (4 * j < D) {
        tape_xi4(key, static_cast<uint32_t>(j), static_cast<uint32_t>(t), xi[q]);
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (4 * j + e >= D) xi[q][e] = 0.f;
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) xi[q][e] = 0.f;
      }
    }
    const double logu = log(static_cast<double>(tape_u(key, static_cast<uint32_t>(t))));
    Col<Real, QPL> col;
    column_forward<Real, TK, QPL>(Pw, sm, key, xs, static_cast<int>(t), col, xi);
    const bool acc = logu < col.la;
    if (warm) {  // _dual_average_update with m = t + 1
      const double m = static_cast<double>(t + 1);
      const double alpha = col.la < 0.0 ? exp(col.la) : 1.0;
      const double w = 1.0 / (m + ad.t0);
      h_bar = (1.0 - w) * h_bar + w * (ad.target_accept - alpha);
      const double log_eps = mu - sqrt(m) / ad.gamma * h_bar;
      const double mk = pow(m, -ad.kappa);
      const double log_eps_bar = mk * log_eps + (1.0 - mk) * log(eps_bar);
      eps = exp(log_eps);
      eps_bar = exp(log_eps_bar);
    }
    if (eps_out && lane == 0) eps_out[c * T + t] = eps_t;
    __syncwarp();
    double lp = 0.0;
    Real* row = S + (c * T + t) * D;
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + 32 * q;
      if (4 * j < D) {
        Real n4[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) n4[e] = (4 * j + e < D) ? (acc ? col.y[q][e] : col.x[q][e]) : Real(0);
        store4(xs + 4 * j, n4);
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (4 * j + e < D) {
            row[4 * j + e] = n4[e];
            if constexpr (TK == kDiagGauss) {
              const double sd = static_cast<double>(n4[e]) - P.mean_d[4 * j + e];
              lp += -0.5 * P.prec_d[4 * j + e] * sd * sd;
            }
          }
      }
    }
    __syncwarp();
    if constexpr (TK == kDenseGauss) {
      if (logp) {  // logp of the new state through the warp's FP64 vector
        double* vd = sm.Vd + warp * Dp;
        for (int d = lane; d < D; d += 32) vd[d] = static_cast<double>(xs[d]) - P.mean_d[d];
        __syncwarp();
#pragma unroll
        for (int q = 0; q < QPL; ++q) {
          const int j = lane + 32 * q;
          if (4 * j < D) {
            double o[4];
            matvec4<double, double, double>(sm.Pd, vd, D, Dp, j, o);
#pragma unroll
            for (int e = 0; e < 4; ++e)
              if (4 * j + e < D) lp += -0.5 * vd[4 * j + e] * o[e];
          }
        }
        __syncwarp();
      }
    }
    if (logp) lp = warp_sum(lp);
    if (lane == 0) {
      if (logp) logp[c * T + t] = static_cast<Real>(lp);
      if (acc_out) acc_out[c * T + t] = acc ? 1 : 0;
    }
  }
  if (state_out && lane == 0) {
    state_out[3 * c] = eps;
    state_out[3 * c + 1] = eps_bar;
    state_out[3 * c + 2] = h_bar;
  }
}

namespace {

template <typename Real, int TK>
const void* pick_chains(int qpl) {
  switch (qpl) {
    case 1: return reinterpret_cast<const void*>(&mala_chains_kernel<Real, TK, 1>);
    case 2: return reinterpret_cast<const void*>(&mala_chains_kernel<Real, TK, 2>);
    default: return reinterpret_cast<const void*>(&mala_chains_kernel<Real, TK, 4>);
  }
}

}  // namespace

size_t mala_chains_smem(bool f64, int64_t Dp, bool dense) {
  const size_t base = f64 ? plan_sweep_smem<double>(Dp, 0, dense).total
                          : plan_sweep_smem<float>(Dp, 0, dense).total;
  return base + (f64 ? 8 : 4) * static_cast<size_t>(kWarps) * Dp;
}

cudaError_t launch_mala_chains(cudaStream_t s, bool f64, int tk, const DevParams& P,
                               const ChainAdapt& ad, int64_t nchains, const void* x0,
                               const uint64_t* seeds, void* S, void* logp, uint8_t* acc,
                               double* eps_out, double* state_out) {
  if (nchains <= 0 || P.T <= 0) return cudaSuccess;
  const int qpl = P.D <= 128 ? 1 : (P.D <= 256 ? 2 : 4);
  const bool dense = tk == kDenseGauss;
  const void* fn = f64 ? (dense ? pick_chains<double, kDenseGauss>(qpl)
                                : pick_chains<double, kDiagGauss>(qpl))
                       : (dense ? pick_chains<float, kDenseGauss>(qpl)
                                : pick_chains<float, kDiagGauss>(qpl));
  const size_t smem = mala_chains_smem(f64, P.Dp, dense);
  cudaError_t e = raise_smem_limit(fn, smem);
  if (e != cudaSuccess) return e;
  DevParams Pv = P;
  ChainAdapt adv = ad;
  int64_t n = nchains;
  void* args[] = {&Pv, &adv, &n, const_cast<void**>(&x0), const_cast<uint64_t**>(&seeds), &S,
                  &logp, &acc, &eps_out, &state_out};
  const int grid = static_cast<int>((nchains + kWarps - 1) / kWarps);
  return cudaLaunchKernel(fn, dim3(grid), dim3(kThreads), args, smem, s);
}

}  // namespace pmcmc
