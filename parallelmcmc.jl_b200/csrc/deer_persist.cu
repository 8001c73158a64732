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
//  - Per sweep: evaluate + tile scan, grid barrier, the previous sweep's
//    convergence test (DEER.jl:567-578) read by every CTA alike, per-coordinate
//    scan of the group aggregates (state entering every CTA), grid barrier,
//    apply with damping in shared memory, max|dS| / max|S| atomics.  Testing a
//    sweep after the next sweep's first barrier saves a barrier a sweep; the
//    evaluation after the last sweep is discarded.  Sweep 0 is tested at once
//    after a third barrier, so a one-sweep solve evaluates once.
//  - After the last sweep every CTA verifies its columns (exact MALA step from
//    S_{t-1}, FP64 log-acceptance), writes S, logp(S_t) and the accept flags
//    (_trajectory_logps, interface.jl:517-524), as the finalize kernel does.
// The kernel is used when every CTA is co-resident (cooperative launch), the
// block has no sliding window and the target is a diagonal or dense Gaussian.
// Its parameters come by value in the launch, so a solve is one launch and
// the state readback.
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
  p.x0 = off;
  off = al(off + sizeof(Real) * Dp);
  p.total = off;
  return p;
}

PersistPlan persist_smem(bool f64, int64_t Dp, int TT, bool dense) {
  return f64 ? plan_persist_smem<double>(Dp, TT, dense) : plan_persist_smem<float>(Dp, TT, dense);
}

namespace {

template <int QPL, int LPC>
__device__ __forceinline__ void xi_from_smem(const float* col, int D, float (&n)[QPL][4]) {
  const int lane = threadIdx.x & (LPC - 1);
#pragma unroll
  for (int q = 0; q < QPL; ++q) {
    const int j = lane + LPC * q;
    if (4 * j < D) {
      load4(col + 4 * j, n[q]);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) n[q][e] = 0.f;
    }
  }
}

}  // namespace

// Two CTAs per SM (at most 128 registers a thread) where that costs no spills:
// FP32 state with up to two quads a lane, FP64 with one.
template <typename Real, int QPL>
constexpr int kPersistMinBlocks = sizeof(Real) * QPL <= 8 ? 2 : 1;

// Columns are evaluated by LPC lanes each (32 / LPC columns per warp); QPL
// quads per lane cover Dp / 4 <= LPC * QPL.
template <typename Real, int TK, int JAC, int QPL, int LPC>
__global__ void __launch_bounds__(kThreads, kPersistMinBlocks<Real, QPL>)
    deer_persist_kernel(const DevParams Pv, DevState* __restrict__ st) {
  __shared__ DevParams P;
  __shared__ Real s_sa[kThreads], s_sb[kThreads];
  __shared__ double s_red[3][kWarps];
  __shared__ unsigned long long s_acc[kWarps];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (threadIdx.x == 0) P = Pv;  // parameters by value: no upload before the launch
  __syncthreads();
  cg::grid_group grid = cg::this_grid();
  // this sweep's maxima max|dS|, max|S| and the non-finite flag, as ordered
  // bits of non-negative doubles, in two slots by sweep parity (P.part[0..5])
  unsigned long long* red = reinterpret_cast<unsigned long long*>(P.part);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int CPW = 32 / LPC;                  // columns per warp
  const int lq = lane & (LPC - 1), half = lane / LPC;  // quad lane, column slot
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
  Real* agg_a = static_cast<Real*>(P.agg_a);
  Real* agg_b = static_cast<Real*>(P.agg_b);
  Real* incl = static_cast<Real*>(P.incl);
  Real* carry0 = incl + static_cast<size_t>(nctas) * Dp;  // S_0 = f(x0)
  Real* Sb = static_cast<Real*>(P.S[0]);                   // last column of every CTA

  Real* x0s = reinterpret_cast<Real*>(smem_raw + pp.x0);
  const int nblk = P.nblk > 1 ? static_cast<int>(P.nblk) : 1;
  for (int bi = 0; bi < nblk; ++bi) {  // blocks of one call, back to back
    const int64_t ncols_out = bi + 1 < nblk ? T : P.ncols_out;
    Real* const S_out = static_cast<Real*>(P.S_out) + static_cast<size_t>(bi) * T * D;
    Real* const logp_out =
        P.logp_out ? static_cast<Real*>(P.logp_out) + static_cast<size_t>(bi) * T : nullptr;
    uint8_t* const accept_out = P.accept_out ? P.accept_out + static_cast<size_t>(bi) * T : nullptr;
    DevState* const st_host = P.st_host ? P.st_host + bi : nullptr;
    // totals of the verification pass, folded in by every CTA as it finishes,
    // the arrival counter and the sweep maxima (the grid barriers in between
    // order these resets before every update, and after the previous block's reads)
    if (cta == 0 && tid == 0) {
      for (int i = 0; i < 6; ++i) red[i] = 0ull;
      st->fin_counter = 0;
      st->n_accept = 0;
      st->min_margin_bits = dbits(INFINITY);
      st->max_defect_bits = 0;
    }
    // start state, zero-padded to Dp: the call's x0, or the previous block's last
    // column; loaded here, stored to shared memory after the tape work below
    const Real* x0src = static_cast<const Real*>(bi > 0 ? P.x_next : P.x0_src ? P.x0_src : P.x0);
    const Real x0r = tid < D ? x0src[tid] : Real(0);

    // ---- tape (interface.jl:334-358) of the CTA's columns, drawn once a block ----
    const TapeKey key(P.seed, P.block + static_cast<uint64_t>(bi));
    // the tape of columns t0 .. t0 + ng (the CTA's own and its scan group's), one
    // (column, quad) pair a thread at a time: every lane busy, however D splits
    {
      const int nq = Dp / 4;
      for (int i = tid; i < (ng + 1) * nq; i += kThreads) {
        const int c = i / nq, q = i - c * nq;
        float n[4];
        tape_xi4(key, static_cast<uint32_t>(q), static_cast<uint32_t>(t0 + c + P.t_off), n);
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (4 * q + e >= D) n[e] = 0.f;
        store4(xis + c * Dp + 4 * q, n);
      }
    }
    // log u of the columns t0 .. t0 + ng (the CTA's own and its scan group's), in
    // FP64, one column a thread: the evaluation reads them from shared memory
    for (int c = tid; c <= ng; c += kThreads)
      lus[c] = log(static_cast<double>(tape_u(key, static_cast<uint32_t>(t0 + c + P.t_off))));
    for (int d = tid; d < Dp; d += kThreads)
      x0s[d] = d == tid ? x0r : d < D ? x0src[d] : Real(0);
    __syncthreads();
    for (int i = tid; i < ncols * (Dp / 4); i += kThreads) {
      const int nq = Dp / 4, c = i / nq, k = 4 * (i - c * nq);
      Real v[4];
      load4(x0s + k, v);
      store4(sm.Xs + c * Dp + k, v);
    }

    // ---- S_0 = f(x0): the same in every sweep ----
    if (cta == 0 && warp == 0) {  // every column slot of warp 0 forms it; slot 0 stores
      float xic[QPL][4];
      xi_from_smem<QPL, LPC>(xis, D, xic);
      Col<Real, QPL> col;
      column_forward<Real, TK, QPL, LPC>(P, sm, key, x0s, 0, col, xic);
      const bool acc = lus[0] < col.la;
#pragma unroll
      for (int q = 0; q < QPL; ++q) {
        const int j = lq + LPC * q;
        if (half == 0 && 4 * j < D) {
          Real f[4];
#pragma unroll
          for (int e = 0; e < 4; ++e)
            f[e] = 4 * j + e < D ? (acc ? col.y[q][e] : col.x[q][e]) : Real(0);
          store4(carry0 + 4 * j, f);
        }
      }
    }

    const Real dmp = static_cast<Real>(P.damping), omd = static_cast<Real>(1.0 - P.damping);
    const bool undamped = P.damping == 1.0;
    int iter = 0, converged = 0, status = 0;
    Real sprev = 0;
    double metric = 0.0;
    // the test of sweep k from its maxima (slot k & 1), after a grid barrier that
    // follows sweep k's apply; on a stop, S_{t0 - 1} (the previous CTA's last
    // column) is read for the verification
    auto stop_test = [&](int k) {
      const unsigned long long* sl = red + 3 * (k & 1);
      const double dmax = __longlong_as_double(static_cast<long long>(__ldcg(sl)));
      const double smax = __longlong_as_double(static_cast<long long>(__ldcg(sl + 1)));
      const bool nonfinite = __ldcg(sl + 2) != 0ull;
      metric = dmax / (P.tol_abs + P.tol_rel * smax);
      converged = metric <= 1.0;
      status = nonfinite ? static_cast<int>(kStNonfinite) : 0;
      const bool stop = converged || iter >= P.maxiter || status != 0;
      if (stop && cta > 0 && tid < Dp) sprev = __ldcg(Sb + (t0 - 1) * Dp + tid);
      return stop;
    };
    for (;;) {
      // ---- evaluate the scan group: column t0 + c + 1 from S_{t0 + c} ----
      // (warp-uniform loop over groups of CPW columns; a slot past the end
      // repeats the group's first column and stores nothing).  The previous
      // sweep's convergence test comes after the next grid barrier, so this
      // evaluation runs before it is known whether another sweep is needed: a
      // solve of more than one sweep evaluates once more than it sweeps, and a
      // sweep has two grid barriers instead of three.  At maxiter nothing is
      // evaluated.
      const bool sweep = iter < P.maxiter;
      for (int cb = warp * CPW; sweep && cb < ng; cb += kWarps * CPW) {
        const bool valid = cb + half < ng;
        const int c = valid ? cb + half : cb;
        const int t = static_cast<int>(t0 + c + 1);
        float xic[QPL][4];
        xi_from_smem<QPL, LPC>(xis + (c + 1) * Dp, D, xic);
        const double logu = lus[c + 1];
        Col<Real, QPL> col;
        column_forward<Real, TK, QPL, LPC>(P, sm, key, sm.Xs + c * Dp, t, col, xic);
        const bool acc = logu < col.la;
        const Real gp = sigmoid_slope<Real>(col.la - logu);
        Real A[QPL][4];
        column_jacobian<Real, TK, JAC, QPL, LPC>(P, sm, key, t + P.t_off, iter, acc, gp, col, A);
#pragma unroll
        for (int q = 0; q < QPL; ++q) {
          const int j = lq + LPC * q;
          if (valid && 4 * j < D) {
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
      if (sweep) {
        __syncthreads();
        tile_scan_inplace<Real>(sm.As, sm.Bs, ng, D, Dp);
        __syncthreads();
        for (int d = tid; d < D; d += kThreads) {
          agg_a[static_cast<size_t>(cta) * Dp + d] = ng > 0 ? sm.As[(ng - 1) * Dp + d] : Real(1);
          agg_b[static_cast<size_t>(cta) * Dp + d] = ng > 0 ? sm.Bs[(ng - 1) * Dp + d] : Real(0);
        }
      }
      grid.sync();

      // ---- convergence test of the previous sweep (DEER.jl:567-578), the same in
      // every CTA: its maxima are complete, every CTA having applied it.  Sweep 0
      // was tested at once, after a barrier of its own (below) ----
      if (iter >= 2 && stop_test(iter - 1)) break;
      // this sweep's slot was last read in the test of sweep iter - 2, which
      // every CTA finished before the previous sweep's second barrier: clear it
      // (the next barrier orders the clear before this sweep's atomics)
      if (cta == 0 && tid == 0)
        for (int i = 0; i < 3; ++i) red[3 * (iter & 1) + i] = 0ull;

      // ---- state entering every CTA: scan of the group aggregates per coordinate ----
      for (int d = cta; d < D; d += nctas)
        carry_scan_tiles<Real>(nctas, d, Dp, agg_a, agg_b, __ldcg(carry0 + d), incl, s_sa, s_sb);
      grid.sync();

      // ---- apply: Newton state of every column, damping, maxima ----
      Real my_dmax = 0, my_smax = 0;  // maxima are exact in the state's precision
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
                my_dmax = max(my_dmax, fabs(n4[e] - o4[e]));
                my_smax = max(my_smax, fabs(n4[e]));
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
      // this CTA's maxima into the sweep's slot (max is exact in any order; the
      // CTAs arrive spread over the apply phase, so the atomics rarely meet)
      my_dmax = warp_max(my_dmax);
      my_smax = warp_max(my_smax);
      bad = __any_sync(0xffffffffu, bad);
      if (lane == 0) {
        s_red[0][warp] = static_cast<double>(my_dmax);
        s_red[1][warp] = static_cast<double>(my_smax);
        s_red[2][warp] = bad ? 1.0 : 0.0;
      }
      __syncthreads();
      unsigned long long* slot = red + 3 * (iter & 1);
      if (tid == 0) {
        double a = 0, b = 0, c = 0;
        for (int w = 0; w < kWarps; ++w)
          a = max(a, s_red[0][w]), b = max(b, s_red[1][w]), c = max(c, s_red[2][w]);
        atomicMax(slot, dbits(a));
        atomicMax(slot + 1, dbits(b));
        if (c != 0.0) atomicMax(slot + 2, 1ull);
      }
      ++iter;
      // the first sweep is tested at once: a block that converges in one sweep
      // (no accepted move) then evaluates nothing more
      if (iter == 1) {
        grid.sync();
        if (stop_test(0)) break;
      }
    }

    // ---- verification pass and outputs on the CTA's columns ----
    // S_{t0 - 1}, the previous CTA's last column, into shared memory
    for (int d = tid; d < Dp; d += kThreads)
      sm.carry[d] = cta == 0 ? x0s[d] : d == tid ? sprev : __ldcg(Sb + (t0 - 1) * Dp + d);
    // the CTA's rows of S_out (row t = column t, D entries) in one coalesced copy
    {
      const int64_t nrows = imin64(ncols, ncols_out - t0);
      if (nrows > 0) {
        Real* dst = S_out + t0 * D;
        const int64_t n = nrows * D;
        if (D == Dp && reinterpret_cast<uintptr_t>(dst) % (4 * sizeof(Real)) == 0) {
          for (int64_t i = tid; i < n / 4; i += kThreads) {
            Real v[4];
            load4(sm.Xs + 4 * i, v);
            store4(dst + 4 * i, v);
          }
        } else {
          for (int64_t i = tid; i < n; i += kThreads) {
            const int64_t r = i / D;
            dst[i] = sm.Xs[r * Dp + (i - r * D)];
          }
        }
      }
    }
    __syncthreads();
    unsigned long long nacc = 0;
    double min_margin = __longlong_as_double(0x7ff0000000000000ll), max_def = 0.0;
    for (int cb = warp * CPW; cb < ncols; cb += kWarps * CPW) {
      const bool valid = cb + half < ncols;
      const int c = valid ? cb + half : cb;
      const int64_t t = t0 + c;
      const Real* xcol = c == 0 ? sm.carry : sm.Xs + (c - 1) * Dp;
      const Real* scol = sm.Xs + c * Dp;
      float xic[QPL][4];
      xi_from_smem<QPL, LPC>(xis + c * Dp, D, xic);
      Col<Real, QPL> col;
      // log alpha reduced below with the log density and the defect (one pass)
      column_forward<Real, TK, QPL, LPC, false>(P, sm, key, xcol, static_cast<int>(t), col, xic);
      const double logu = lus[c];
      const bool out = valid && t < ncols_out;
      // the recursion defect max|S_t - f_t| for both outcomes, selected after the
      // reductions (which then run alongside the log-density's)
      Real dx = 0, dy = 0;  // exact maxima
      double lp = 0.0;
      double* vd = kDense ? sm.Vd + warp * Dp : nullptr;
#pragma unroll
      for (int q = 0; q < QPL; ++q) {
        const int j = lq + LPC * q;
        if (4 * j < D) {
          Real s4[4];
          load4(scol + 4 * j, s4);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            if (4 * j + e >= D) continue;
            dx = max(dx, fabs(s4[e] - col.x[q][e]));
            dy = max(dy, fabs(s4[e] - col.y[q][e]));
            const double sd = static_cast<double>(s4[e]) - P.mean_d[4 * j + e];
            if constexpr (TK == kDiagGauss) lp += -0.5 * P.prec_d[4 * j + e] * sd * sd;
            else vd[4 * j + e] = sd;
            if (out && t == ncols_out - 1) static_cast<Real*>(P.x_next)[4 * j + e] = s4[e];
          }
        }
      }
      if constexpr (kDense) {
        __syncwarp();
#pragma unroll
        for (int q = 0; q < QPL; ++q) {
          const int j = lq + LPC * q;
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
#pragma unroll
      for (int o = LPC / 2; o > 0; o >>= 1) {
        col.la += __shfl_xor_sync(0xffffffffu, col.la, o);
        lp += __shfl_xor_sync(0xffffffffu, lp, o);
        dx = max(dx, __shfl_xor_sync(0xffffffffu, dx, o));
        dy = max(dy, __shfl_xor_sync(0xffffffffu, dy, o));
      }
      const bool acc = logu < col.la;
      if (valid && lq == 0) {
        if (out) {
          if (logp_out) logp_out[t] = static_cast<Real>(lp);
          if (accept_out) accept_out[t] = acc ? 1 : 0;
        }
        nacc += acc ? 1 : 0;
        min_margin = min(min_margin, fabs(col.la - logu));
        max_def = max(max_def, static_cast<double>(acc ? dy : dx));
      }
    }
    // per warp: the column slots' totals
    nacc = warp_sum(nacc);
    max_def = warp_max(max_def);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      min_margin = min(min_margin, __shfl_xor_sync(0xffffffffu, min_margin, o));
    __syncthreads();  // s_red was last read in the convergence test
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
      // accepted count, smallest margin and largest defect into the totals
      // (margins and defects are non-negative: their bits order like the values,
      // and a NaN defect sorts above every number); the last CTA to arrive writes
      // the final state, the others leave without waiting at a grid barrier
      atomicAdd(&st->n_accept, a);
      atomicMin(&st->min_margin_bits, dbits(mm));
      atomicMax(&st->max_defect_bits, dbits(md));
      __threadfence();
      const bool last = atomicAdd(&st->fin_counter, 1u) == static_cast<unsigned>(nctas - 1);
      if (last) {
        __threadfence();

        // ---- last CTA: the final state ----
        const unsigned long long* tot = &st->n_accept;
        DevState f{};
        f.epoch = st->epoch;  // look-back epochs of the per-sweep path continue
        f.iter = iter;
        f.converged = converged;
        f.status = status;
        f.metric = metric;
        f.n_accept = __ldcg(tot);
        f.min_margin_bits = __ldcg(&st->min_margin_bits);
        f.max_defect_bits = __ldcg(&st->max_defect_bits);
        *st = f;
        if (st_host) {
          *st_host = f;
          __threadfence_system();
        }
      }
    }
    // the next block starts from this block's last column (x_next) once every
    // CTA has finished this one
    if (bi + 1 < nblk) grid.sync();
  }  // blocks
}

namespace {

template <typename Real, int TK, int JAC>
const void* pick_persist(int64_t D) {
  const void* k = nullptr;
  if constexpr (TK == kDiagGauss) {  // two columns per warp while D <= 128
    if (D <= 64) return reinterpret_cast<const void*>(&deer_persist_kernel<Real, TK, JAC, 1, 16>);
    if (D <= 128) return reinterpret_cast<const void*>(&deer_persist_kernel<Real, TK, JAC, 2, 16>);
  }
  if (D <= 128) k = reinterpret_cast<const void*>(&deer_persist_kernel<Real, TK, JAC, 1, 32>);
  else if (D <= 256) k = reinterpret_cast<const void*>(&deer_persist_kernel<Real, TK, JAC, 2, 32>);
  else k = reinterpret_cast<const void*>(&deer_persist_kernel<Real, TK, JAC, 4, 32>);
  return k;
}

template <typename Real>
const void* pick_persist_t(int tk, int jac, int64_t D) {
  if (tk == kDiagGauss)
    return jac == kJacStoch ? pick_persist<Real, kDiagGauss, kJacStoch>(D)
                            : pick_persist<Real, kDiagGauss, kJacDiag>(D);
  return jac == kJacStoch ? pick_persist<Real, kDenseGauss, kJacStoch>(D)
                          : pick_persist<Real, kDenseGauss, kJacDiag>(D);
}

}  // namespace

const void* persist_kernel(bool f64, int tk, int jac, int64_t D) {
  if (tk != kDiagGauss && tk != kDenseGauss) return nullptr;
  return f64 ? pick_persist_t<double>(tk, jac, D) : pick_persist_t<float>(tk, jac, D);
}

}  // namespace pmcmc
