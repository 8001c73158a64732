// deer_persist.cu -- a whole DEER solve of a Gaussian device target in one
// cooperative launch: tape, every Newton sweep and the verification pass.
//
// Same iteration as the per-sweep kernel (deer_sweep.cu, DEER.jl:553-581),
// restructured so that nothing between sweeps leaves the SM:
//  - CTA j owns the trajectory columns [t0, t0 + ncols) (t0 = j * TT) and keeps
//    them in shared memory from the first sweep to the last, together with
//    its tape (xi, log u) for columns t0 .. t0 + ncols, generated once.
//  - Its scan group is the columns t0 + 1 .. t0 + ncols.  Column t of the
//    Newton system depends on S_{t-1} only, so the group is evaluated from the
//    CTA's own columns (no halo from the neighbour).  The group's aggregate
//    maps S_{t0} to S_{t0 + ncols}, the first column of the next CTA.
//  - Column 0 depends on x0 alone: S_0 = f(x0) in every sweep; CTA 0 forms it
//    once and it seeds the scan over the group aggregates.
//  - Per sweep: evaluate + tile scan, grid barrier, per-coordinate scan of the
//    group aggregates (state entering every CTA), grid barrier, apply with
//    damping in shared memory, max|dS| / max|S| atomics, grid barrier, and the
//    convergence test (DEER.jl:567-578) read by every CTA alike.
//  - After the last sweep every CTA verifies its columns (exact MALA step from
//    S_{t-1}, FP64 log-acceptance), writes S, logp(S_t) and the accept flags
//    (_trajectory_logps, interface.jl:517-524), as the finalize kernel does.
// The kernel is used when every CTA is co-resident (cooperative launch), the
// block has no sliding window and the target is a diagonal or dense Gaussian.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "deer_column.cuh"
#include "deer_device.cuh"
#include "deer_launch.h"

namespace cg = cooperative_groups;

namespace pmcmc {

// Shared memory: the sweep plan (columns, A, B, carry, dense-target vectors)
// followed by the CTA's tape, TT + 1 columns of xi (float) and log u (double).
template <typename Real>
__host__ __device__ inline PersistPlan plan_persist_smem(int64_t Dp, int TT, bool dense) {
  auto al = [](size_t x) { return (x + 15) & ~size_t(15); };
  PersistPlan p{};
  p.sweep = plan_sweep_smem<Real>(Dp, TT, dense);
  size_t off = al(p.sweep.total);
  p.xi = off;
  off = al(off + sizeof(float) * (TT + 1) * Dp);
  p.lu = off;
  off = al(off + sizeof(double) * (TT + 1));
  p.total = off;
  return p;
}

PersistPlan persist_smem(bool f64, int64_t Dp, int TT, bool dense) {
  return f64 ? plan_persist_smem<double>(Dp, TT, dense) : plan_persist_smem<float>(Dp, TT, dense);
}

namespace {

template <int QPL>
__device__ __forceinline__ void xi_from_smem(const float* col, int D, float (&n)[QPL][4]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < QPL; ++q) {
    const int j = lane + 32 * q;
    if (4 * j < D) {
      load4(col + 4 * j, n[q]);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) n[q][e] = 0.f;
    }
  }
}

__device__ __forceinline__ unsigned long long ld_l2(const unsigned long long* p) {
  return __ldcg(p);
}

}  // namespace

template <typename Real, int TK, int JAC, int QPL>
__global__ void __launch_bounds__(kThreads)
    deer_persist_kernel(const DevParams* __restrict__ Pg, DevState* __restrict__ st) {
  __shared__ DevParams P;
  __shared__ Real s_sa[kThreads], s_sb[kThreads];
  __shared__ double s_red[3][kWarps];
  __shared__ unsigned long long s_acc[kWarps];
  __shared__ int s_bad;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  load_params(Pg, P);
  cg::grid_group grid = cg::this_grid();

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cta = static_cast<int>(blockIdx.x), nctas = static_cast<int>(gridDim.x);
  const int TT = P.tile_cols;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  const int64_t T = P.T;
  const int64_t t0 = static_cast<int64_t>(cta) * TT;
  const int ncols = static_cast<int>(imin64(TT, T - t0));  // >= 1: one CTA per tile
  const bool has_next = t0 + ncols < T;
  const int ng = has_next ? ncols : ncols - 1;  // columns of the scan group
  constexpr bool kDense = TK == kDenseGauss;
  Smem<Real> sm = carve<Real>(smem_raw, P, TT, kDense);
  const PersistPlan pp = plan_persist_smem<Real>(Dp, TT, kDense);
  float* xis = reinterpret_cast<float*>(smem_raw + pp.xi);
  double* lus = reinterpret_cast<double*>(smem_raw + pp.lu);
  const Real* x0 = static_cast<const Real*>(P.x0);
  Real* agg_a = static_cast<Real*>(P.agg_a);
  Real* agg_b = static_cast<Real*>(P.agg_b);
  Real* incl = static_cast<Real*>(P.incl);
  Real* carry0 = incl + static_cast<size_t>(nctas) * Dp;  // S_0 = f(x0)
  Real* Sb = static_cast<Real*>(P.S[0]);                   // last column of every CTA

  if (cta == 0 && tid == 0) {
    st->iter = 0;
    st->cur = 0;
    st->converged = 0;
    st->status = 0;
    st->t_lo = 0;
    st->t_lo_prev = 0;
    st->dmax_bits = 0;
    st->smax_bits = 0;
    st->metric = __longlong_as_double(0x7ff0000000000000ll);
    st->n_accept = 0;
    st->min_margin_bits = 0x7ff0000000000000ull;  // +inf
    st->max_defect_bits = 0;
  }
  if (tid == 0) s_bad = 0;

  // ---- tape of columns t0 .. t0 + ncols (interface.jl:334-358) and S = x0 ----
  const TapeKey key(P.seed, P.block);
  {
    const int nq = Dp / 4;
    const int ntape = has_next ? ncols + 1 : ncols;
    for (int i = tid; i < ntape * nq; i += kThreads) {
      const int c = i / nq, q = i - c * nq;
      const uint32_t tg = static_cast<uint32_t>(t0 + c + P.t_off);
      float n[4];
      tape_xi4(key, static_cast<uint32_t>(q), tg, n);
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (4 * q + e >= D) n[e] = 0.f;
      store4(xis + c * Dp + 4 * q, n);
      if (q == 0) lus[c] = log(static_cast<double>(tape_u(key, tg)));
    }
    for (int i = tid; i < ncols * nq; i += kThreads) {
      const int c = i / nq, k = 4 * (i - c * nq);
      Real v[4];
      load4(x0 + k, v);
      store4(sm.Xs + c * Dp + k, v);
    }
  }
  __syncthreads();

  // ---- S_0 = f(x0): the same in every sweep ----
  if (cta == 0 && warp == 0) {
    float xic[QPL][4];
    xi_from_smem<QPL>(xis, D, xic);
    Col<Real, QPL> col;
    column_forward<Real, TK, QPL>(P, sm, key, x0, 0, col, xic);
    const bool acc = lus[0] < col.la;
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + 32 * q;
      if (4 * j < D) {
        Real f[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) f[e] = 4 * j + e < D ? (acc ? col.y[q][e] : col.x[q][e]) : Real(0);
        store4(carry0 + 4 * j, f);
      }
    }
  }

  const Real dmp = static_cast<Real>(P.damping), omd = static_cast<Real>(1.0 - P.damping);
  const bool undamped = P.damping == 1.0;
  int iter = 0, converged = 0;
  double metric = 0.0;
  for (;;) {
    // ---- evaluate the scan group: column t0 + c + 1 from S_{t0 + c} ----
    for (int c = warp; c < ng; c += kWarps) {
      const int t = static_cast<int>(t0 + c + 1);
      float xic[QPL][4];
      xi_from_smem<QPL>(xis + (c + 1) * Dp, D, xic);
      Col<Real, QPL> col;
      column_forward<Real, TK, QPL>(P, sm, key, sm.Xs + c * Dp, t, col, xic);
      const double logu = lus[c + 1];
      const bool acc = logu < col.la;
      const double gd = 1.0 / (1.0 + exp(-(col.la - logu)));
      const Real gp = static_cast<Real>(gd * (1.0 - gd));
      Real A[QPL][4];
      column_jacobian<Real, TK, JAC, QPL>(P, sm, key, t + P.t_off, iter, acc, gp, col, A);
#pragma unroll
      for (int q = 0; q < QPL; ++q) {
        const int j = lane + 32 * q;
        if (4 * j < D) {
          Real a4[4], b4[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const Real f = acc ? col.y[q][e] : col.x[q][e];
            a4[e] = (4 * j + e < D) ? A[q][e] : Real(0);
            b4[e] = (4 * j + e < D) ? f - A[q][e] * col.x[q][e] : Real(0);
          }
          store4(sm.As + c * Dp + 4 * j, a4);
          store4(sm.Bs + c * Dp + 4 * j, b4);
        }
      }
    }
    __syncthreads();
    tile_scan_inplace<Real>(sm.As, sm.Bs, ng, D, Dp);
    __syncthreads();
    for (int d = tid; d < D; d += kThreads) {
      agg_a[static_cast<size_t>(cta) * Dp + d] = ng > 0 ? sm.As[(ng - 1) * Dp + d] : Real(1);
      agg_b[static_cast<size_t>(cta) * Dp + d] = ng > 0 ? sm.Bs[(ng - 1) * Dp + d] : Real(0);
    }
    grid.sync();
    // every CTA has read the previous sweep's maxima: clear them for this one
    if (cta == 0 && tid == 0) {
      st->dmax_bits = 0;
      st->smax_bits = 0;
    }

    // ---- state entering every CTA: scan of the group aggregates per coordinate ----
    for (int d = cta; d < D; d += nctas)
      carry_scan_tiles<Real>(nctas, d, Dp, agg_a, agg_b, __ldcg(carry0 + d), incl, s_sa, s_sb);
    grid.sync();

    // ---- apply: Newton state of every column, damping, maxima ----
    double my_dmax = 0.0, my_smax = 0.0;
    bool bad = false;
    Real cr[QPL][4];
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + 32 * q;
#pragma unroll
      for (int e = 0; e < 4; ++e)
        cr[q][e] = 4 * j + e < D ? __ldcg(incl + static_cast<size_t>(cta) * Dp + 4 * j + e)
                                 : Real(0);
    }
    for (int c = warp; c < ncols; c += kWarps) {
#pragma unroll
      for (int q = 0; q < QPL; ++q) {
        const int j = lane + 32 * q;
        if (4 * j < D) {
          Real a4[4] = {1, 1, 1, 1}, b4[4] = {0, 0, 0, 0}, o4[4], n4[4];
          if (c > 0) {
            load4(sm.As + (c - 1) * Dp + 4 * j, a4);
            load4(sm.Bs + (c - 1) * Dp + 4 * j, b4);
          }
          load4(sm.Xs + c * Dp + 4 * j, o4);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const Real s = a4[e] * cr[q][e] + b4[e];
            n4[e] = undamped ? s : omd * o4[e] + dmp * s;
            if (4 * j + e < D) {
              my_dmax = max(my_dmax, static_cast<double>(fabs(n4[e] - o4[e])));
              my_smax = max(my_smax, static_cast<double>(fabs(n4[e])));
              bad |= !isfinite(n4[e]);
            } else {
              n4[e] = Real(0);
            }
          }
          store4(sm.Xs + c * Dp + 4 * j, n4);
          if (c == ncols - 1 && has_next) store4(Sb + (t0 + c) * Dp + 4 * j, n4);
        }
      }
    }
    if (bad) s_bad = 1;
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
      if (s_bad) atomicCAS(&st->status, 0, static_cast<int>(kStNonfinite));
    }
    grid.sync();

    // ---- convergence test (DEER.jl:567-578), the same in every CTA ----
    const double dmax = bitsd(ld_l2(&st->dmax_bits));
    const double smax = bitsd(ld_l2(&st->smax_bits));
    const int status = __ldcg(&st->status);
    metric = dmax / (P.tol_abs + P.tol_rel * smax);
    ++iter;
    converged = metric <= 1.0;
    if (converged || iter >= P.maxiter || status != 0) break;
  }

  // ---- verification pass and outputs on the CTA's columns ----
  // S_{t0 - 1}, the previous CTA's last column, into shared memory
  for (int d = tid; d < Dp; d += kThreads)
    sm.carry[d] = cta == 0 ? x0[d] : __ldcg(Sb + (t0 - 1) * Dp + d);
  __syncthreads();
  unsigned long long nacc = 0;
  double min_margin = __longlong_as_double(0x7ff0000000000000ll), max_def = 0.0;
  for (int c = warp; c < ncols; c += kWarps) {
    const int64_t t = t0 + c;
    const Real* xcol = c == 0 ? sm.carry : sm.Xs + (c - 1) * Dp;
    const Real* scol = sm.Xs + c * Dp;
    float xic[QPL][4];
    xi_from_smem<QPL>(xis + c * Dp, D, xic);
    Col<Real, QPL> col;
    column_forward<Real, TK, QPL>(P, sm, key, xcol, static_cast<int>(t), col, xic);
    const double logu = lus[c];
    const bool acc = logu < col.la;
    double def = 0.0, lp = 0.0;
    double* vd = kDense ? sm.Vd + warp * Dp : nullptr;
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
    if constexpr (kDense) {
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
  if (lane == 0) {
    s_acc[warp] = nacc;
    s_red[0][warp] = min_margin;
    s_red[2][warp] = max_def;
  }
  __syncthreads();
  if (tid == 0) {
    unsigned long long a = 0;
    double mm = s_red[0][0], md = 0.0;
    for (int w = 0; w < kWarps; ++w) {
      a += s_acc[w];
      mm = min(mm, s_red[0][w]);
      md = max(md, s_red[2][w]);
    }
    if (a) atomicAdd(&st->n_accept, a);
    atomicMin(&st->min_margin_bits, dbits(mm));
    if (md > 0) atomicMax(&st->max_defect_bits, dbits(md));
    if (cta == 0) {
      st->iter = iter;
      st->converged = converged;
      st->metric = metric;
    }
  }
}

namespace {

template <typename Real, int TK, int JAC>
const void* pick_persist(int qpl) {
  switch (qpl) {
    case 1: return reinterpret_cast<const void*>(&deer_persist_kernel<Real, TK, JAC, 1>);
    case 2: return reinterpret_cast<const void*>(&deer_persist_kernel<Real, TK, JAC, 2>);
    default: return reinterpret_cast<const void*>(&deer_persist_kernel<Real, TK, JAC, 4>);
  }
}

template <typename Real>
const void* pick_persist_t(int tk, int jac, int qpl) {
  if (tk == kDiagGauss)
    return jac == kJacStoch ? pick_persist<Real, kDiagGauss, kJacStoch>(qpl)
                            : pick_persist<Real, kDiagGauss, kJacDiag>(qpl);
  return jac == kJacStoch ? pick_persist<Real, kDenseGauss, kJacStoch>(qpl)
                          : pick_persist<Real, kDenseGauss, kJacDiag>(qpl);
}

}  // namespace

const void* persist_kernel(bool f64, int tk, int jac, int qpl) {
  if (tk != kDiagGauss && tk != kDenseGauss) return nullptr;
  return f64 ? pick_persist_t<double>(tk, jac, qpl) : pick_persist_t<float>(tk, jac, qpl);
}

}  // namespace pmcmc
