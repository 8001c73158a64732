// deer_sweep.cu -- fused Newton sweep for the Gaussian device targets.
//
// One launch = one DEER iteration over the whole block (DEER.jl:553-581):
//   x_bar_t = S_{t-1} (x0 for t = 0)                       DEER.jl:402-405
//   MALA proposal, FP64 log-acceptance, forward step        MALA.jl:577-597
//   Jacobian diagonal: Hutchinson probes (MALA.jl:599-625, DEER.jl:407-418)
//     or the exact diagonal (jac_diag_via_jvps, DEER.jl:327-342) in closed form
//   B = F - A .* x_bar                                      DEER.jl:419
//   S_t = A_t .* S_{t-1} + B_t                              DEERScan.jl:102-173
//   damping, max|dS| and max|S| in FP64                     DEER.jl:471-473, 567-571
// Each CTA owns a tile of consecutive columns: it stages S_old (plus one halo
// column) in shared memory, evaluates the tile, scans it locally and joins its
// predecessors through a decoupled look-back, then writes S_new once.  The
// tape (xi, u) and the probes are regenerated in registers, so a sweep reads
// and writes the trajectory once.  The last CTA to finish evaluates the
// convergence test and drives the CUDA-graph while-node.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "deer_device.cuh"
#include "deer_launch.h"
#include "deer_column.cuh"

namespace cg = cooperative_groups;

namespace pmcmc {

// Logistic target: the gradient / HVP contractions over the N data rows come
// from the two GEMM passes of this sweep (g_x, y, w, g_y, H(y) w in HBM,
// likelihood sums in FP64); this evaluates the rest of the batched
// fwd + JVP (MALA.jl:592-625) for one column, probe `probe`, and returns
// A = scale * (z .* J z + acc_in) and B = F - A .* x_bar: with several
// probes, acc_in holds the earlier probes' z .* J z and scale is 1 / probes
// (the probe average of DEER.jl:412-418).
template <typename Real, int QPL>
__device__ __forceinline__ void column_logistic(const DevParams& P, const TapeKey& key,
                                                const Real* xcol, int t, int iter, int probe,
                                                const Real* acc_in, Real scale,
                                                Real (&A)[QPL][4], Real (&Bv)[QPL][4]) {
  const int lane = threadIdx.x & 31;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  const Real eps = static_cast<Real>(P.eps), inv2eps = static_cast<Real>(P.inv2eps);
  const size_t off = static_cast<size_t>(t) * Dp;
  const Real* gxp = static_cast<const Real*>(P.lg[0]) + off;
  const Real* yp = static_cast<const Real*>(P.lg[1]) + off;
  const Real* wp = static_cast<const Real*>(P.lg[2]) + off;
  const Real* gyp = static_cast<const Real*>(P.lg[3]) + off;
  const Real* hvp = static_cast<const Real*>(P.lg[4]) + off;
  Real x[QPL][4], gx[QPL][4], y[QPL][4], gy[QPL][4], w[QPL][4], hvy[QPL][4], z[QPL][4];
  double la = 0.0;
#pragma unroll
  for (int q = 0; q < QPL; ++q) {
    const int j = lane + 32 * q;
    if (4 * j < D) {
      load4(xcol + 4 * j, x[q]);
      load4(gxp + 4 * j, gx[q]);
      load4(yp + 4 * j, y[q]);
      load4(gyp + 4 * j, gy[q]);
      load4(wp + 4 * j, w[q]);
      load4(hvp + 4 * j, hvy[q]);
      float xi[4];
      load4(P.xi + off + 4 * j, xi);
      const U4 pb = probe_bits(key, static_cast<uint32_t>(j >> 5),
                               static_cast<uint32_t>(t + P.t_off),
                               probe, iter);
      const uint32_t wv = u4_word(pb, (j >> 3) & 3);
      const int sh = (j & 7) * 4;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        z[q][e] = ((wv >> (sh + e)) & 1u) ? Real(1) : Real(-1);
        if (4 * j + e < D) {
          const double xd = static_cast<double>(x[q][e]), yd = static_cast<double>(y[q][e]);
          const double r1 = P.sqrt2eps * static_cast<double>(xi[e]);
          const double r2 = (xd - yd) - P.eps * static_cast<double>(gy[q][e]);
          la += -0.5 * P.tau * (yd * yd - xd * xd) + (r1 * r1 - r2 * r2) * P.inv4eps;
        } else {
          z[q][e] = Real(0);
        }
      }
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        x[q][e] = gx[q][e] = y[q][e] = gy[q][e] = w[q][e] = hvy[q][e] = z[q][e] = Real(0);
    }
  }
  la = warp_sum(la) + (P.lpy[t] - P.lpx[t]);
  // near-tie columns: the FP64 value of the same log alpha (logistic_tie.cu)
  if (P.la_ref) la = P.la_ref[t];
  const double logu = P.logu[t];
  const bool acc = logu < la;
  const Real gp = sigmoid_slope<Real>(la - logu);
  Real dla = 0;
#pragma unroll
  for (int q = 0; q < QPL; ++q)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const Real r = x[q][e] - y[q][e] - eps * gy[q][e];
      const Real dr = z[q][e] - w[q][e] - eps * hvy[q][e];
      dla += gy[q][e] * w[q][e] - gx[q][e] * z[q][e] - inv2eps * r * dr;
    }
  dla = warp_sum(dla);
  const Real dg = gp * dla;
#pragma unroll
  for (int q = 0; q < QPL; ++q) {
    Real prev[4] = {Real(0), Real(0), Real(0), Real(0)};
    const int j = lane + 32 * q;
    if (acc_in && 4 * j < D) load4(acc_in + off + 4 * j, prev);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const Real jz = (acc ? w[q][e] : z[q][e]) + (y[q][e] - x[q][e]) * dg;
      A[q][e] = scale * (z[q][e] * jz + prev[e]);
      const Real f = acc ? y[q][e] : x[q][e];
      Bv[q][e] = f - A[q][e] * x[q][e];
    }
  }
  if (lane == 0) {
    P.acc_col[t] = acc ? 1 : 0;
    P.la_col[t] = la - logu;
  }
}

// Logistic target, exact diagonal (:diag): J_ii = a (1 + eps H_x,ii) + (1 - a)
// + (y - x_bar)_i g' dla_i, with diag H_x in lg[2] and dla in lg[4] from the
// four passes of the sweep (logistic.cu, stages 3-6); A and B for one column.
template <typename Real, int QPL>
__device__ __forceinline__ void column_logistic_diag(const DevParams& P, const Real* xcol, int t,
                                                     Real (&A)[QPL][4], Real (&Bv)[QPL][4]) {
  const int lane = threadIdx.x & 31;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  const Real eps = static_cast<Real>(P.eps);
  const size_t off = static_cast<size_t>(t) * Dp;
  const Real* yp = static_cast<const Real*>(P.lg[1]) + off;
  const Real* hdp = static_cast<const Real*>(P.lg[2]) + off;
  const Real* gyp = static_cast<const Real*>(P.lg[3]) + off;
  const Real* dlp = static_cast<const Real*>(P.lg[4]) + off;
  Real x[QPL][4], y[QPL][4], hd[QPL][4], dl[QPL][4];
  double la = 0.0;
#pragma unroll
  for (int q = 0; q < QPL; ++q) {
    const int j = lane + 32 * q;
    if (4 * j < D) {
      Real gy[4];
      float xi[4];
      load4(xcol + 4 * j, x[q]);
      load4(yp + 4 * j, y[q]);
      load4(hdp + 4 * j, hd[q]);
      load4(dlp + 4 * j, dl[q]);
      load4(gyp + 4 * j, gy);
      load4(P.xi + off + 4 * j, xi);
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (4 * j + e < D) {
          const double xd = static_cast<double>(x[q][e]), yd = static_cast<double>(y[q][e]);
          const double r1 = P.sqrt2eps * static_cast<double>(xi[e]);
          const double r2 = (xd - yd) - P.eps * static_cast<double>(gy[e]);
          la += -0.5 * P.tau * (yd * yd - xd * xd) + (r1 * r1 - r2 * r2) * P.inv4eps;
        }
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) x[q][e] = y[q][e] = hd[q][e] = dl[q][e] = Real(0);
    }
  }
  la = warp_sum(la) + (P.lpy[t] - P.lpx[t]);
  if (P.la_ref) la = P.la_ref[t];
  const double logu = P.logu[t];
  const bool acc = logu < la;
  const Real gp = sigmoid_slope<Real>(la - logu);
#pragma unroll
  for (int q = 0; q < QPL; ++q)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      A[q][e] = (acc ? Real(1) + eps * hd[q][e] : Real(1)) + (y[q][e] - x[q][e]) * gp * dl[q][e];
      const Real f = acc ? y[q][e] : x[q][e];
      Bv[q][e] = f - A[q][e] * x[q][e];
    }
  if (lane == 0) {
    P.acc_col[t] = acc ? 1 : 0;
    P.la_col[t] = la - logu;
  }
}

// ---------------------------------------------------------------------------
// The sweep kernel
// ---------------------------------------------------------------------------
// COOP = true: launched cooperatively with every tile resident; the cross-tile
// scan is two grid-wide barriers around a per-coordinate scan of the tile
// aggregates (no look-back chains).  COOP = false: decoupled look-back.
template <typename Real, int TK, int JAC, int QPL, bool COOP>
__global__ void __launch_bounds__(kThreads)
    deer_sweep_kernel(const DevParams* __restrict__ Pg, DevState* __restrict__ st,
                      cudaGraphConditionalHandle cond, int use_cond) {
  __shared__ DevParams P;
  __shared__ int s_tile, s_last, s_err, s_nonfinite, s_jstar;
  __shared__ Real s_sa[kThreads], s_sb[kThreads];
  __shared__ double s_red[2][kWarps];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  load_params(Pg, P);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int32_t iter = *reinterpret_cast<volatile int32_t*>(&st->iter);
  if (!use_cond) {
    // eager mode: extra launches after convergence are no-ops
    if (*reinterpret_cast<volatile int32_t*>(&st->converged) || iter >= P.maxiter ||
        *reinterpret_cast<volatile int32_t*>(&st->status) != 0)
      return;
  }
  const int cur = *reinterpret_cast<volatile int32_t*>(&st->cur);
  const int64_t t_lo = *reinterpret_cast<volatile int64_t*>(&st->t_lo);
  const int64_t t_lo_prev = *reinterpret_cast<volatile int64_t*>(&st->t_lo_prev);
  const uint32_t epoch = *reinterpret_cast<volatile uint32_t*>(&st->epoch);
  if (tid == 0) {
    s_tile = COOP ? static_cast<int>(blockIdx.x)
                  : static_cast<int>(atomicAdd(&st->tile_counter, 1u));
    s_err = 0;
    s_nonfinite = 0;
  }
  __syncthreads();
  const int tile = s_tile;
  const int TT = P.tile_cols;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  const int64_t T = P.T;
  const bool windowed = P.W < T;
  const int64_t t_hi = min(T, t_lo + P.W);
  const int64_t t0 = t_lo + static_cast<int64_t>(tile) * TT;
  const int64_t rem = t_hi - t0;
  const int ncols = rem <= 0 ? 0 : static_cast<int>(rem < TT ? rem : TT);
  const Real* Sold = static_cast<const Real*>(P.S[cur]);
  Real* Snew = static_cast<Real*>(P.S[cur ^ 1]);
  const Real* x0 = static_cast<const Real*>(P.x0);
  const bool from_x0 = (!windowed) && iter == 0;  // first sweep: S_old = s0 broadcast

  // Window mode: columns finalised by the previous sweep are copied into the
  // buffer this sweep writes, so both buffers agree on every final column.
  if (windowed && t_lo > t_lo_prev) {
    const int64_t n = (t_lo - t_lo_prev) * Dp;
    for (int64_t i = static_cast<int64_t>(tile) * kThreads + tid; i < n;
         i += static_cast<int64_t>(gridDim.x) * kThreads)
      Snew[t_lo_prev * Dp + i] = Sold[t_lo_prev * Dp + i];
  }

  Smem<Real> sm = carve<Real>(smem_raw, P, TT, TK == kDenseGauss);
  double my_dmax = 0.0, my_smax = 0.0;

  if (ncols > 0) {
    // ---- stage S_old columns t0-1 .. t0+ncols-1 ----
    // quads, several loads in flight per thread
    const int nq = Dp / 4;
    const int nstage = (ncols + 1) * nq;
#pragma unroll 4
    for (int i = tid; i < nstage; i += kThreads) {
      const int c = i / nq, k = 4 * (i - c * nq);
      const int64_t t = t0 - 1 + c;
      const Real* src = (from_x0 || t < 0) ? x0 + k
                        : t < t_lo        ? Sold + (t_lo - 1) * Dp + k  // s_{t_lo - 1}
                                          : Sold + t * Dp + k;
      Real v[4];
      load4(src, v);
      store4(sm.Xs + c * Dp + k, v);
    }
    __syncthreads();

    // ---- phase 1: evaluate columns (one warp per column) ----
    // The tape of the warp's next column is loaded while this one is computed.
    const TapeKey key(P.seed, P.block);
    float xin[QPL][4];
    double lun = 0.0;
    if constexpr (TK != kLogistic) {
      if (warp < ncols) {
        load_xi<Real, QPL>(P, t0 + warp, xin);
        lun = P.logu[t0 + warp];
      }
    }
    for (int c = warp; c < ncols; c += kWarps) {
      const int t = static_cast<int>(t0 + c);
      Real A[QPL][4], Bq[QPL][4];
      if constexpr (TK == kLogistic && JAC == kJacDiag) {
        column_logistic_diag<Real, QPL>(P, sm.Xs + c * Dp, t, A, Bq);
      } else if constexpr (TK == kLogistic) {
        // the last probe of the sweep; the earlier ones are in lg_acc
        const bool multi = P.probes > 1;
        column_logistic<Real, QPL>(P, key, sm.Xs + c * Dp, t, iter, P.probes - 1,
                                   multi ? static_cast<const Real*>(P.lg_acc) : nullptr,
                                   multi ? Real(1) / static_cast<Real>(P.probes) : Real(1), A,
                                   Bq);
      } else {
        float xic[QPL][4];
#pragma unroll
        for (int q = 0; q < QPL; ++q)
#pragma unroll
          for (int e = 0; e < 4; ++e) xic[q][e] = xin[q][e];
        const double logu = lun;
        if (c + kWarps < ncols) {
          load_xi<Real, QPL>(P, t + kWarps, xin);
          lun = P.logu[t + kWarps];
        }
        Col<Real, QPL> col;
        column_forward<Real, TK, QPL>(P, sm, key, sm.Xs + c * Dp, t, col, xic);
        const bool acc = logu < col.la;
        const Real gp = sigmoid_slope<Real>(col.la - logu);
        column_jacobian<Real, TK, JAC, QPL>(P, sm, key, t, iter, acc, gp, col, A);
#pragma unroll
        for (int q = 0; q < QPL; ++q)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const Real f = acc ? col.y[q][e] : col.x[q][e];
            Bq[q][e] = f - A[q][e] * col.x[q][e];
          }
      }
#pragma unroll
      for (int q = 0; q < QPL; ++q) {
        const int j = lane + 32 * q;
        if (4 * j < D) {
          Real a4[4], b4[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            a4[e] = (4 * j + e < D) ? A[q][e] : Real(0);
            b4[e] = (4 * j + e < D) ? Bq[q][e] : Real(0);
          }
          store4(sm.As + c * Dp + 4 * j, a4);
          store4(sm.Bs + c * Dp + 4 * j, b4);
        }
      }
    }
    __syncthreads();

    // ---- phase 2: tile-local inclusive scan ----
    tile_scan_inplace<Real>(sm.As, sm.Bs, ncols, D, Dp);
    __syncthreads();

    // ---- phase 3: state entering the tile ----
    Real* agg_a = static_cast<Real*>(P.agg_a);
    Real* agg_b = static_cast<Real*>(P.agg_b);
    Real* incl = static_cast<Real*>(P.incl);
    const size_t last = static_cast<size_t>(ncols - 1) * Dp;
    if constexpr (COOP) {
      for (int d = tid; d < D; d += kThreads) {
        agg_a[static_cast<size_t>(tile) * Dp + d] = sm.As[last + d];
        agg_b[static_cast<size_t>(tile) * Dp + d] = sm.Bs[last + d];
      }
    } else {
      if (tile == 0) {
        for (int d = tid; d < D; d += kThreads) {
          const Real s_lo = sm.Xs[d];
          sm.carry[d] = s_lo;
          incl[d] = sm.As[last + d] * s_lo + sm.Bs[last + d];
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release(P.flags, (epoch << 2) | kFlagIncl);
      } else {
        for (int d = tid; d < D; d += kThreads) {
          agg_a[static_cast<size_t>(tile) * Dp + d] = sm.As[last + d];
          agg_b[static_cast<size_t>(tile) * Dp + d] = sm.Bs[last + d];
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release(P.flags + tile, (epoch << 2) | kFlagAgg);
        if (warp == 0) {
          int err = 0;
          const int js = lookback_fixed(tile, epoch, P.flags, &err);
          if (lane == 0) {
            s_jstar = js;
            if (err) s_err = 1;
          }
        }
        __syncthreads();
        const int js = s_jstar;
        for (int d = tid; d < D; d += kThreads) {
          const Real cin = js >= 0 ? lookback_compose<Real>(tile, js, d, Dp, agg_a, agg_b, incl)
                                   : Real(0);
          sm.carry[d] = cin;
          incl[static_cast<size_t>(tile) * Dp + d] = sm.As[last + d] * cin + sm.Bs[last + d];
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release(P.flags + tile, (epoch << 2) | kFlagIncl);
      }
      __syncthreads();
    }
  }

  if constexpr (COOP) {
    // ---- phase B: per-coordinate scan of the tile aggregates (all CTAs) ----
    cg::grid_group grid = cg::this_grid();
    grid.sync();
    const int nact = static_cast<int>((t_hi - t_lo + TT - 1) / TT);
    const Real* agg_a = static_cast<const Real*>(P.agg_a);
    const Real* agg_b = static_cast<const Real*>(P.agg_b);
    Real* incl = static_cast<Real*>(P.incl);
    for (int d = blockIdx.x; d < D; d += gridDim.x) {
      const Real s_lo = (from_x0 || t_lo == 0) ? x0[d] : Sold[(t_lo - 1) * Dp + d];
      carry_scan_tiles<Real>(nact, d, Dp, agg_a, agg_b, s_lo, incl, s_sa, s_sb);
    }
    grid.sync();
    if (ncols > 0) {
      for (int d = tid; d < D; d += kThreads)
        sm.carry[d] = __ldcg(incl + static_cast<size_t>(tile) * Dp + d);
    }
    __syncthreads();
  }

  if (ncols > 0) {
    // ---- phase 4: apply carry, damping, metric, write S_new ----
    const Real dmp = static_cast<Real>(P.damping), omd = static_cast<Real>(1.0 - P.damping);
    const bool undamped = P.damping == 1.0;
    Real cr[QPL][4];
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + 32 * q;
      if (4 * j < D) load4(sm.carry + 4 * j, cr[q]);
    }
    bool bad = false;
    for (int c = warp; c < ncols; c += kWarps) {
      const int64_t t = t0 + c;
      Real cmax = 0;
#pragma unroll
      for (int q = 0; q < QPL; ++q) {
        const int j = lane + 32 * q;
        if (4 * j < D) {
          Real a4[4], b4[4], o4[4], n4[4];
          load4(sm.As + c * Dp + 4 * j, a4);
          load4(sm.Bs + c * Dp + 4 * j, b4);
          load4(sm.Xs + (c + 1) * Dp + 4 * j, o4);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const Real s = a4[e] * cr[q][e] + b4[e];
            n4[e] = undamped ? s : omd * o4[e] + dmp * s;
            if (4 * j + e < D) {
              const Real dv = fabs(n4[e] - o4[e]);
              cmax = max(cmax, dv);
              my_dmax = max(my_dmax, static_cast<double>(dv));
              my_smax = max(my_smax, static_cast<double>(fabs(n4[e])));
              bad |= !isfinite(n4[e]);
            } else {
              n4[e] = Real(0);
            }
          }
          store4(Snew + t * Dp + 4 * j, n4);
        }
      }
      if (windowed) {
        cmax = warp_max(cmax);
        if (lane == 0) P.colmax[t] = static_cast<float>(cmax);
      }
    }
    if (bad) s_nonfinite = 1;
  }

  // ---- block reduction of the metric, one atomic per CTA ----
  my_dmax = warp_max(my_dmax);
  my_smax = warp_max(my_smax);
  if (lane == 0) {
    s_red[0][warp] = my_dmax;
    s_red[1][warp] = my_smax;
  }
  __syncthreads();
  if (tid == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < kWarps; ++w) a = max(a, s_red[0][w]), b = max(b, s_red[1][w]);
    if (a > 0) atomicMax(&st->dmax_bits, dbits(a));
    if (b > 0) atomicMax(&st->smax_bits, dbits(b));
    if (s_err) atomicExch(&st->status, static_cast<int>(kStTimeout));
    if (s_nonfinite) atomicCAS(&st->status, 0, static_cast<int>(kStNonfinite));
    __threadfence();
    // the last CTA to arrive runs the convergence test (no third grid barrier)
    const unsigned prev = atomicAdd(&st->done_counter, 1u);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;

  // ---- last CTA: convergence test (DEER.jl:567-578) and loop control ----
  __threadfence();
  const double dmax = bitsd(atomicAdd(&st->dmax_bits, 0ull));
  const double smax = bitsd(atomicAdd(&st->smax_bits, 0ull));
  const double scale = P.tol_abs + P.tol_rel * smax;
  const double metric = dmax / scale;
  int64_t new_t_lo = t_lo;
  if (windowed) {
    // t_lo advances to the first column whose change exceeds the scale.
    __shared__ long long s_first;
    if (tid == 0) s_first = t_hi;
    __syncthreads();
    long long mine = t_hi;
    for (int64_t t = t_lo + tid; t < t_hi; t += kThreads)
      if (static_cast<double>(__ldcg(P.colmax + t)) > scale) {
        mine = t;
        break;
      }
    atomicMin(&s_first, mine);
    __syncthreads();
    new_t_lo = s_first;
  }
  if (tid == 0) {
    // a tensor-core pass of this sweep gave up a wait: its results are not to be used
    if (P.tc_err && *reinterpret_cast<const volatile int*>(P.tc_err))
      atomicCAS(&st->status, 0, static_cast<int>(kStTimeout));
    const int status = atomicAdd(&st->status, 0);
    const int converged = windowed ? (new_t_lo >= T) : (metric <= 1.0);
    st->metric = metric;
    st->iter = iter + 1;
    st->cur = cur ^ 1;
    st->t_lo_prev = t_lo;
    st->t_lo = new_t_lo;
    st->converged = converged;
    st->epoch = epoch + 1;
    st->tile_counter = 0;
    st->done_counter = 0;
    st->dmax_bits = 0;
    st->smax_bits = 0;
    __threadfence();
    const bool more = !converged && (iter + 1 < P.maxiter) && status == 0;
    if (use_cond) cudaGraphSetConditional(cond, more ? 1u : 0u);
  }
}

// ---------------------------------------------------------------------------
// Reset of the per-solve device state (and, in window mode, both buffers).
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void deer_init_kernel(const DevParams* __restrict__ Pg, DevState* __restrict__ st) {
  const DevParams& P = *Pg;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->iter = 0;
    st->cur = 0;
    st->converged = 0;
    st->status = 0;
    st->t_lo = 0;
    st->t_lo_prev = 0;
    st->epoch = st->epoch + 1;
    st->tile_counter = 0;
    st->done_counter = 0;
    st->fin_counter = 0;
    st->dmax_bits = 0;
    st->smax_bits = 0;
    st->metric = __longlong_as_double(0x7ff0000000000000ll);
    st->n_accept = 0;
    st->min_margin_bits = 0x7ff0000000000000ull;  // +inf
    st->max_defect_bits = 0;
  }
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t i0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  // The block's tape (xi_t, log u_t), generated once and read by every sweep.
  const TapeKey key(P.seed, P.block);
  const int64_t nq = P.Dp / 4;
  for (int64_t i = i0; i < nq * P.T; i += stride) {
    const int64_t t = i / nq, j = i % nq;
    float n[4];
    const uint32_t tg = static_cast<uint32_t>(t + P.t_off);
    tape_xi4(key, static_cast<uint32_t>(j), tg, n);
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (4 * j + e >= P.D) n[e] = 0.f;
    *reinterpret_cast<float4*>(P.xi + t * P.Dp + 4 * j) = make_float4(n[0], n[1], n[2], n[3]);
    if (j == 0) P.logu[t] = log(static_cast<double>(tape_u(key, tg)));
  }
  if (P.W < P.T) {
    const Real* x0 = static_cast<const Real*>(P.x0);
    const int64_t n = P.T * P.Dp;
    for (int64_t i = i0; i < n; i += stride) {
      const Real v = x0[i % P.Dp];
      static_cast<Real*>(P.S[0])[i] = v;
      static_cast<Real*>(P.S[1])[i] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Finalize: verify the returned trajectory column by column (exact MALA step
// from S_{t-1} in FP64 log-acceptance), emit accept flags, margins, the
// recursion defect and logp(S_t) (_trajectory_logps, interface.jl:517-524),
// and copy the kept columns out.
// ---------------------------------------------------------------------------
template <typename Real, int TK, int QPL>
__global__ void __launch_bounds__(kThreads)
    deer_finalize_kernel(const DevParams* __restrict__ Pg, DevState* __restrict__ st) {
  __shared__ DevParams P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  load_params(Pg, P);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  Smem<Real> sm = carve<Real>(smem_raw, P, 1, TK == kDenseGauss);
  __syncthreads();
  const int cur = st->cur;
  const Real* S = static_cast<const Real*>(P.S[cur]);
  const Real* x0 = static_cast<const Real*>(P.x0);
  const TapeKey key(P.seed, P.block);
  unsigned long long nacc = 0;
  double min_margin = __longlong_as_double(0x7ff0000000000000ll), max_def = 0.0;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kWarps + warp; t < P.T;
       t += static_cast<int64_t>(gridDim.x) * kWarps) {
    const Real* xcol = t == 0 ? x0 : S + (t - 1) * Dp;
    const Real* scol = S + t * Dp;
    Col<Real, QPL> col;
    column_forward<Real, TK, QPL>(P, sm, key, xcol, static_cast<int>(t), col);
    const double logu = P.logu[t];
    const bool acc = logu < col.la;
    double def = 0.0, lp = 0.0;
    double* vd = TK == kDenseGauss ? sm.Vd + warp * Dp : nullptr;
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + 32 * q;
      if (4 * j < D) {
        Real s4[4];
        load4(scol + 4 * j, s4);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          if (4 * j + e >= D) continue;
          const Real f = acc ? col.y[q][e] : col.x[q][e];
          def = max(def, static_cast<double>(fabs(s4[e] - f)));
          const double sd = static_cast<double>(s4[e]) - P.mean_d[4 * j + e];
          if constexpr (TK == kDiagGauss) lp += -0.5 * P.prec_d[4 * j + e] * sd * sd;
          else vd[4 * j + e] = sd;
          if (t < P.ncols_out) {
            static_cast<Real*>(P.S_out)[t * D + 4 * j + e] = s4[e];
            if (t == P.ncols_out - 1) static_cast<Real*>(P.x_next)[4 * j + e] = s4[e];
          }
        }
      }
    }
    if constexpr (TK == kDenseGauss) {
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
    lp = warp_sum(lp);
    def = warp_max(def);
    if (lane == 0) {
      if (t < P.ncols_out) {
        if (P.logp_out) static_cast<Real*>(P.logp_out)[t] = static_cast<Real>(lp);
        if (P.accept_out) P.accept_out[t] = acc ? 1 : 0;
      }
      nacc += acc ? 1 : 0;
      min_margin = min(min_margin, fabs(col.la - logu));
      max_def = max(max_def, def);
    }
  }
  // one atomic per CTA and quantity (same-address atomics from every warp serialise)
  __shared__ unsigned long long r_acc[kWarps];
  __shared__ double r_mm[kWarps], r_def[kWarps];
  if (lane == 0) {
    r_acc[warp] = nacc;
    r_mm[warp] = min_margin;
    r_def[warp] = max_def;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kWarps; ++w) {
      nacc = r_acc[0] += r_acc[w];
      min_margin = r_mm[0] = min(r_mm[0], r_mm[w]);
      max_def = r_def[0] = max(r_def[0], r_def[w]);
    }
    if (r_acc[0]) atomicAdd(&st->n_accept, r_acc[0]);
    atomicMin(&st->min_margin_bits, dbits(r_mm[0]));
    if (r_def[0] > 0) atomicMax(&st->max_defect_bits, dbits(r_def[0]));
  }
}

// ---------------------------------------------------------------------------
// Unfused evaluation for the plain path: A and B for every column written to
// HBM (the shape of deer_update!'s batched branch, DEER.jl:398-419).
// ---------------------------------------------------------------------------
template <typename Real, int TK, int JAC, int QPL>
__global__ void __launch_bounds__(kThreads)
    deer_eval_kernel(const DevParams* __restrict__ Pg, const Real* __restrict__ Sold, int iter,
                     int from_x0, Real* __restrict__ A, Real* __restrict__ B) {
  __shared__ DevParams P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  load_params(Pg, P);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  Smem<Real> sm = carve<Real>(smem_raw, P, 1, TK == kDenseGauss);
  __syncthreads();
  const Real* x0 = static_cast<const Real*>(P.x0);
  const TapeKey key(P.seed, P.block);
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kWarps + warp; t < P.T;
       t += static_cast<int64_t>(gridDim.x) * kWarps) {
    const Real* xcol = (t == 0 || from_x0) ? x0 : Sold + (t - 1) * Dp;
    Col<Real, QPL> col;
    column_forward<Real, TK, QPL>(P, sm, key, xcol, static_cast<int>(t), col);
    const double logu = P.logu[t];
    const bool acc = logu < col.la;
    const double gd = 1.0 / (1.0 + exp(-(col.la - logu)));
    const Real gp = static_cast<Real>(gd * (1.0 - gd));
    Real Aq[QPL][4];
    column_jacobian<Real, TK, JAC, QPL>(P, sm, key, static_cast<int>(t + P.t_off), iter, acc, gp,
                                         col, Aq);
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + 32 * q;
      if (4 * j < D) {
        Real a4[4], b4[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const Real f = acc ? col.y[q][e] : col.x[q][e];
          a4[e] = (4 * j + e < D) ? Aq[q][e] : Real(0);
          b4[e] = (4 * j + e < D) ? f - Aq[q][e] * col.x[q][e] : Real(0);
        }
        store4(A + t * Dp + 4 * j, a4);
        store4(B + t * Dp + 4 * j, b4);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Logistic target with probes > 1: after the passes of probe k < probes - 1,
// lg_acc += z_k .* J z_k (lg_acc = for k = 0), one warp a column.  The last
// probe is added, and the sum divided by the probe count, in the sweep.
// ---------------------------------------------------------------------------
template <typename Real, int QPL>
__global__ void __launch_bounds__(kThreads)
    lg_probe_accum_kernel(const DevParams* __restrict__ Pg, const DevState* __restrict__ st,
                          int probe) {
  __shared__ DevParams P;
  load_params(Pg, P);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int Dp = static_cast<int>(P.Dp), D = static_cast<int>(P.D);
  const int iter = st->iter;
  const bool from_x0 = iter == 0;
  const Real* S = static_cast<const Real*>(P.S[st->cur]);
  const Real* x0 = static_cast<const Real*>(P.x0);
  Real* accv = static_cast<Real*>(P.lg_acc);
  const TapeKey key(P.seed, P.block);
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kWarps + warp; t < P.T;
       t += static_cast<int64_t>(gridDim.x) * kWarps) {
    const Real* xcol = (from_x0 || t == 0) ? x0 : S + (t - 1) * Dp;
    Real A[QPL][4], Bq[QPL][4];
    column_logistic<Real, QPL>(P, key, xcol, static_cast<int>(t), iter, probe,
                               probe > 0 ? accv : nullptr, Real(1), A, Bq);
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + 32 * q;
      if (4 * j < D) {
        Real a4[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) a4[e] = (4 * j + e < D) ? A[q][e] : Real(0);
        store4(accv + t * Dp + 4 * j, a4);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Logistic finalize: copy the kept columns out, logp(S_t) from the likelihood
// sums of the last logp pass (left in lpx) plus the prior, and the accept
// flags / margins of acc_col / la_col: those of the verification pass at the
// returned trajectory (fused path), or of the last sweep (plain path, whose
// max_defect the host reports as NaN).
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void __launch_bounds__(kThreads)
    deer_finalize_logistic_kernel(const DevParams* __restrict__ Pg, DevState* __restrict__ st) {
  __shared__ DevParams P;
  load_params(Pg, P);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  const Real* S = static_cast<const Real*>(P.S[st->cur]);
  unsigned long long nacc = 0;
  double mm = __longlong_as_double(0x7ff0000000000000ll);
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kWarps + warp; t < P.T;
       t += static_cast<int64_t>(gridDim.x) * kWarps) {
    double q = 0.0;
    for (int d = lane; d < D; d += 32) {
      const Real v = S[t * Dp + d];
      q += static_cast<double>(v) * static_cast<double>(v);
      if (t < P.ncols_out) {
        static_cast<Real*>(P.S_out)[t * D + d] = v;
        if (t == P.ncols_out - 1) static_cast<Real*>(P.x_next)[d] = v;
      }
    }
    q = warp_sum(q);
    if (lane == 0) {
      const bool acc = P.acc_col[t] != 0;
      if (t < P.ncols_out) {
        if (P.logp_out) static_cast<Real*>(P.logp_out)[t] = static_cast<Real>(P.lpx[t] - 0.5 * P.tau * q);
        if (P.accept_out) P.accept_out[t] = acc ? 1 : 0;
      }
      nacc += acc ? 1 : 0;
      mm = min(mm, fabs(P.la_col[t]));
    }
  }
  __shared__ unsigned long long r_acc[kWarps];
  __shared__ double r_mm[kWarps];
  if (lane == 0) {
    r_acc[warp] = nacc;
    r_mm[warp] = mm;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kWarps; ++w) {
      r_acc[0] += r_acc[w];
      r_mm[0] = min(r_mm[0], r_mm[w]);
    }
    if (r_acc[0]) atomicAdd(&st->n_accept, r_acc[0]);
    atomicMin(&st->min_margin_bits, dbits(r_mm[0]));
  }
}

// ---------------------------------------------------------------------------
// Host-side dispatch
// ---------------------------------------------------------------------------
template <typename Real, int TK, int JAC, int QPL>
static SweepKernels pick3() {
  SweepKernels k;
  k.sweep = reinterpret_cast<const void*>(&deer_sweep_kernel<Real, TK, JAC, QPL, false>);
  k.sweep_coop = reinterpret_cast<const void*>(&deer_sweep_kernel<Real, TK, JAC, QPL, true>);
  k.finalize = reinterpret_cast<const void*>(&deer_finalize_kernel<Real, TK, QPL>);
  k.init = reinterpret_cast<const void*>(&deer_init_kernel<Real>);
  k.eval = reinterpret_cast<const void*>(&deer_eval_kernel<Real, TK, JAC, QPL>);
  return k;
}

template <typename Real, int TK, int JAC>
static SweepKernels pick2(int qpl) {
  switch (qpl) {
    case 1: return pick3<Real, TK, JAC, 1>();
    case 2: return pick3<Real, TK, JAC, 2>();
    default: return pick3<Real, TK, JAC, 4>();
  }
}

template <typename Real>
static SweepKernels pick1(int tk, int jac, int qpl) {
  if (tk == kDiagGauss)
    return jac == kJacStoch ? pick2<Real, kDiagGauss, kJacStoch>(qpl)
                            : pick2<Real, kDiagGauss, kJacDiag>(qpl);
  return jac == kJacStoch ? pick2<Real, kDenseGauss, kJacStoch>(qpl)
                          : pick2<Real, kDenseGauss, kJacDiag>(qpl);
}

template <typename Real, int QPL, int JAC>
static SweepKernels pick_logistic() {
  SweepKernels k;
  k.sweep = reinterpret_cast<const void*>(&deer_sweep_kernel<Real, kLogistic, JAC, QPL, false>);
  k.sweep_coop = reinterpret_cast<const void*>(&deer_sweep_kernel<Real, kLogistic, JAC, QPL, true>);
  k.finalize = reinterpret_cast<const void*>(&deer_finalize_logistic_kernel<Real>);
  k.init = reinterpret_cast<const void*>(&deer_init_kernel<Real>);
  k.eval = reinterpret_cast<const void*>(&lg_probe_accum_kernel<Real, QPL>);
  return k;
}

template <typename Real, int JAC>
static SweepKernels pick_logistic_q(int qpl) {
  return qpl == 1 ? pick_logistic<Real, 1, JAC>()
                  : (qpl == 2 ? pick_logistic<Real, 2, JAC>() : pick_logistic<Real, 4, JAC>());
}

SweepKernels logistic_sweep_kernels(bool f64, int64_t D, int jac) {
  const int qpl = D <= 128 ? 1 : (D <= 256 ? 2 : 4);
  SweepKernels k;
  if (jac == kJacDiag)
    k = f64 ? pick_logistic_q<double, kJacDiag>(qpl) : pick_logistic_q<float, kJacDiag>(qpl);
  else
    k = f64 ? pick_logistic_q<double, kJacStoch>(qpl) : pick_logistic_q<float, kJacStoch>(qpl);
  k.qpl = qpl;
  return k;
}

SweepKernels gauss_sweep_kernels(bool f64, int tk, int jac, int64_t D) {
  const int qpl = D <= 128 ? 1 : (D <= 256 ? 2 : 4);
  SweepKernels k = f64 ? pick1<double>(tk, jac, qpl) : pick1<float>(tk, jac, qpl);
  k.persist = persist_kernel(f64, tk, jac, D);
  k.qpl = qpl;
  return k;
}

SmemPlan gauss_sweep_smem(bool f64, int64_t Dp, int TT, bool dense) {
  return f64 ? plan_sweep_smem<double>(Dp, TT, dense) : plan_sweep_smem<float>(Dp, TT, dense);
}

}  // namespace pmcmc
