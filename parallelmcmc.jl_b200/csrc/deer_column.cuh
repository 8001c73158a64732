// deer_column.cuh -- per-column building blocks shared by the sweep kernels:
// vector loads, dense mat-vecs, the shared-memory plan, and the forward MALA
// half and Jacobian-diagonal estimates for one column evaluated by one warp.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "deer_device.cuh"
#include "deer_launch.h"
#include "pmcmc_rng.cuh"

namespace pmcmc {

template <typename Real>
struct Vec4;
template <>
struct Vec4<float> {
  using T = float4;
};
template <>
struct Vec4<double> {
  using T = double4;
};

template <typename Real>
__device__ __forceinline__ void load4(const Real* p, Real v[4]) {
  const auto q = *reinterpret_cast<const typename Vec4<Real>::T*>(p);
  v[0] = q.x;
  v[1] = q.y;
  v[2] = q.z;
  v[3] = q.w;
}
template <typename Real>
__device__ __forceinline__ void store4(Real* p, const Real v[4]) {
  typename Vec4<Real>::T q;
  q.x = v[0];
  q.y = v[1];
  q.z = v[2];
  q.w = v[3];
  *reinterpret_cast<typename Vec4<Real>::T*>(p) = q;
}

template <typename Real>
__device__ __forceinline__ const Real* prec_of(const DevParams& P);
template <>
__device__ __forceinline__ const float* prec_of<float>(const DevParams& P) {
  return P.prec_f;
}
template <>
__device__ __forceinline__ const double* prec_of<double>(const DevParams& P) {
  return P.prec_d;
}
template <typename Real>
__device__ __forceinline__ const Real* mean_of(const DevParams& P);
template <>
__device__ __forceinline__ const float* mean_of<float>(const DevParams& P) {
  return P.mean_f;
}
template <>
__device__ __forceinline__ const double* mean_of<double>(const DevParams& P) {
  return P.mean_d;
}

// out[e] = sum_k M(4j+e, k) v[k]; M column-major, leading dimension Dp,
// padded rows zero; v is a warp-private vector in shared memory.
template <typename M, typename V, typename Acc>
__device__ __forceinline__ void matvec4(const M* __restrict__ Mm, const V* v, int D, int Dp,
                                        int j, Acc out[4]) {
  Acc a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  const M* col = Mm + 4 * j;
  for (int k = 0; k < D; ++k) {
    const Acc vk = static_cast<Acc>(v[k]);
    M m[4];
    load4(col + static_cast<size_t>(k) * Dp, m);
    a0 = fma(static_cast<Acc>(m[0]), vk, a0);
    a1 = fma(static_cast<Acc>(m[1]), vk, a1);
    a2 = fma(static_cast<Acc>(m[2]), vk, a2);
    a3 = fma(static_cast<Acc>(m[3]), vk, a3);
  }
  out[0] = a0;
  out[1] = a1;
  out[2] = a2;
  out[3] = a3;
}

// ---------------------------------------------------------------------------
// Shared memory
// ---------------------------------------------------------------------------
template <typename Real>
struct Smem {
  Real* Xs;     // (TT+1) x Dp : S_old columns t0-1 .. t0+TT-1
  Real* As;     // TT x Dp
  Real* Bs;     // TT x Dp
  Real* carry;  // Dp
  const double* Pd;  // dense precision in double (smem copy or global)
  const Real* Pf;    // dense precision in Real
  double* Vd;        // kWarps x Dp warp-private vectors
  Real* Vf;          // kWarps x Dp
};

template <typename Real>
__host__ __device__ inline SmemPlan plan_sweep_smem(int64_t Dp, int TT, bool dense) {
  SmemPlan s{};
  size_t off = 0;
  auto al = [](size_t x) { return (x + 15) & ~size_t(15); };
  s.xs = off;
  off = al(off + sizeof(Real) * (TT + 1) * Dp);
  s.as = off;
  off = al(off + sizeof(Real) * 2 * TT * Dp);
  s.carry = off;
  off = al(off + sizeof(Real) * Dp);
  s.p_in_smem = 0;
  if (dense) {
    s.vd = off;
    off = al(off + sizeof(double) * kWarps * Dp);
    s.vf = off;
    off = al(off + sizeof(Real) * kWarps * Dp);
    const size_t pbytes = (sizeof(double) + sizeof(Real)) * Dp * Dp + 32;
    if (off + pbytes <= 150 * 1024) {
      s.p_in_smem = 1;
      s.pd = off;
      off = al(off + sizeof(double) * Dp * Dp);
      s.pf = off;
      off = al(off + sizeof(Real) * Dp * Dp);
    }
  }
  s.total = off;
  return s;
}

template <typename Real>
__device__ Smem<Real> carve(unsigned char* base, const DevParams& P, int TT, bool dense) {
  const SmemPlan pl = plan_sweep_smem<Real>(P.Dp, TT, dense);
  Smem<Real> s;
  s.Xs = reinterpret_cast<Real*>(base + pl.xs);
  s.As = reinterpret_cast<Real*>(base + pl.as);
  s.Bs = s.As + static_cast<size_t>(TT) * P.Dp;
  s.carry = reinterpret_cast<Real*>(base + pl.carry);
  s.Vd = nullptr;
  s.Vf = nullptr;
  s.Pd = P.prec_d;
  s.Pf = prec_of<Real>(P);
  if (dense) {
    s.Vd = reinterpret_cast<double*>(base + pl.vd);
    s.Vf = reinterpret_cast<Real*>(base + pl.vf);
    const int nv = static_cast<int>(kWarps * P.Dp);
    for (int i = threadIdx.x; i < nv; i += blockDim.x) {
      s.Vd[i] = 0.0;
      s.Vf[i] = Real(0);
    }
    if (pl.p_in_smem) {
      double* pd = reinterpret_cast<double*>(base + pl.pd);
      Real* pf = reinterpret_cast<Real*>(base + pl.pf);
      const int n = static_cast<int>(P.Dp * P.Dp);
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        pd[i] = P.prec_d[i];
        pf[i] = prec_of<Real>(P)[i];
      }
      s.Pd = pd;
      s.Pf = pf;
    }
  }
  return s;
}

__device__ __forceinline__ void load_params(const DevParams* Pg, DevParams& sp) {
  constexpr int n = sizeof(DevParams) / sizeof(unsigned long long);
  static_assert(sizeof(DevParams) % sizeof(unsigned long long) == 0, "DevParams padding");
  if (threadIdx.x < n)
    reinterpret_cast<unsigned long long*>(&sp)[threadIdx.x] =
        reinterpret_cast<const unsigned long long*>(Pg)[threadIdx.x];
  __syncthreads();
}

// ---------------------------------------------------------------------------
// One column, one warp (or LPC lanes of it: 32 / LPC columns per warp for the
// diagonal target).  Lane owns quads j = lane + LPC q (d = 4j .. 4j+3).
// ---------------------------------------------------------------------------
template <typename Real, int QPL>
struct Col {
  Real x[QPL][4], xi[QPL][4], gx[QPL][4], y[QPL][4], gy[QPL][4];
  double la;
};

// g (1 - g) for g = sigmoid(x) (x = log alpha - log u), the slope of the
// surrogate accept weight in the JVP (MALA.jl:622, 721), as a / (1 + a)^2
// with a = exp(-|x|): no cancellation in either tail.  It scales only the
// Jacobian estimate, so FP32 state takes it in FP32; accept decisions use
// the FP64 log alpha itself.
template <typename Real>
__device__ __forceinline__ Real sigmoid_slope(double x) {
  if constexpr (sizeof(Real) == 4) {
    const float a = __expf(-fabsf(static_cast<float>(x)));
    const float inv = __fdividef(1.f, 1.f + a);
    return a * inv * inv;
  } else {
    const double a = exp(-fabs(x));
    const double inv = 1.0 / (1.0 + a);
    return a * inv * inv;
  }
}

// Forward MALA half (MALA.jl:577-592): gradient, proposal y (Real), gradient
// at y, and the FP64 log acceptance ratio.  The D/2 log(4 pi eps) constants of
// the two logq terms cancel exactly and are not formed; y - x - eps g_x is
// sqrt(2 eps) xi by construction of y.
// xi_pre: the column's tape normals already in registers (prefetched by the
// caller), or nullptr to load them here.
template <typename Real, int QPL>
__device__ __forceinline__ void load_xi(const DevParams& P, int64_t t, float (&n)[QPL][4]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < QPL; ++q) {
    const int j = lane + 32 * q;
    if (4 * j < P.D) {
      load4(P.xi + t * P.Dp + 4 * j, n[q]);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) n[q][e] = 0.f;
    }
  }
}

// kReduce = false leaves c.la as this lane's partial sum, for a caller that
// reduces it together with its own per-lane sums.
template <typename Real, int TK, int QPL, int LPC = 32, bool kReduce = true>
__device__ __forceinline__ void column_forward(const DevParams& P, const Smem<Real>& sm,
                                               const TapeKey& key, const Real* xcol, int t,
                                               Col<Real, QPL>& c,
                                               const float (*xi_pre)[4] = nullptr) {
  static_assert(TK == kDiagGauss || LPC == 32, "dense targets use whole warps per column");
  const int lane = threadIdx.x & (LPC - 1), warp = threadIdx.x >> 5;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  const Real eps = static_cast<Real>(P.eps), c2 = static_cast<Real>(P.sqrt2eps);
  double la = 0.0;
#pragma unroll
  for (int q = 0; q < QPL; ++q) {
    const int j = lane + LPC * q;
    if (4 * j < D) {
      load4(xcol + 4 * j, c.x[q]);
      float n[4];
      if (xi_pre) {
#pragma unroll
        for (int e = 0; e < 4; ++e) n[e] = xi_pre[q][e];
      } else {
        load4(P.xi + static_cast<size_t>(t) * Dp + 4 * j, n);
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) c.xi[q][e] = static_cast<Real>(n[e]);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) c.x[q][e] = c.xi[q][e] = Real(0);
    }
  }
  if constexpr (TK == kDiagGauss) {
    const Real* lamR = prec_of<Real>(P);
    const Real* muR = mean_of<Real>(P);
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + LPC * q;
      if (4 * j >= D) {
        // lanes past the last quad take part in the warp reductions with zeros
#pragma unroll
        for (int e = 0; e < 4; ++e) c.gx[q][e] = c.y[q][e] = c.gy[q][e] = Real(0);
      } else {
        Real lam[4], mu[4];
        double lamd[4], mud[4];
        load4(lamR + 4 * j, lam);
        load4(muR + 4 * j, mu);
        load4(P.prec_d + 4 * j, lamd);
        load4(P.mean_d + 4 * j, mud);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const Real gx = -lam[e] * (c.x[q][e] - mu[e]);
          const Real y = fma(c2, c.xi[q][e], fma(eps, gx, c.x[q][e]));
          c.gx[q][e] = gx;
          c.y[q][e] = y;
          c.gy[q][e] = -lam[e] * (y - mu[e]);
          if (4 * j + e < D) {
            const double xd = static_cast<double>(c.x[q][e]) - mud[e];
            const double yd = static_cast<double>(y) - mud[e];
            const double lp = -0.5 * lamd[e] * (yd * yd - xd * xd);
            const double r1 = P.sqrt2eps * static_cast<double>(c.xi[q][e]);
            const double r2 = (static_cast<double>(c.x[q][e]) - static_cast<double>(y)) +
                              P.eps * lamd[e] * yd;
            la += lp + (r1 * r1 - r2 * r2) * P.inv4eps;
          }
        }
      }
    }
  } else {
    // Dense Gaussian: gradients in FP64 through warp-private shared vectors.
    double* vd = sm.Vd + warp * Dp;
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + LPC * q;
      if (4 * j < D)
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (4 * j + e < D) vd[4 * j + e] = static_cast<double>(c.x[q][e]) - P.mean_d[4 * j + e];
    }
    __syncwarp();
    double gxd[QPL][4];
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + LPC * q;
      if (4 * j < D) {
        double o[4];
        matvec4<double, double, double>(sm.Pd, vd, D, Dp, j, o);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          gxd[q][e] = -o[e];
          c.gx[q][e] = static_cast<Real>(-o[e]);
          c.y[q][e] = fma(c2, c.xi[q][e], fma(eps, c.gx[q][e], c.x[q][e]));
          if (4 * j + e < D)
            la -= 0.5 * (static_cast<double>(c.x[q][e]) - P.mean_d[4 * j + e]) * gxd[q][e];
        }
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) gxd[q][e] = 0.0, c.gx[q][e] = c.y[q][e] = Real(0);
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + LPC * q;
      if (4 * j < D)
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (4 * j + e < D) vd[4 * j + e] = static_cast<double>(c.y[q][e]) - P.mean_d[4 * j + e];
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < QPL; ++q) {
      const int j = lane + LPC * q;
      if (4 * j < D) {
        double o[4];
        matvec4<double, double, double>(sm.Pd, vd, D, Dp, j, o);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          c.gy[q][e] = static_cast<Real>(-o[e]);
          if (4 * j + e < D) {
            const double yd = static_cast<double>(c.y[q][e]) - P.mean_d[4 * j + e];
            la += 0.5 * yd * (-o[e]);
            const double r1 = P.sqrt2eps * static_cast<double>(c.xi[q][e]);
            const double r2 = (static_cast<double>(c.x[q][e]) - static_cast<double>(c.y[q][e])) +
                              P.eps * o[e];
            la += (r1 * r1 - r2 * r2) * P.inv4eps;
          }
        }
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) c.gy[q][e] = Real(0);
      }
    }
    __syncwarp();
  }
  c.la = kReduce ? seg_sum<LPC>(la) : la;
}

// Dense HVP quad: out = -P v (v written to the warp's Real vector first).
template <typename Real, int QPL>
__device__ __forceinline__ void dense_neg_pv(const DevParams& P, const Smem<Real>& sm,
                                             const Real (&v)[QPL][4], Real (&out)[QPL][4]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  Real* vf = sm.Vf + warp * Dp;
#pragma unroll
  for (int q = 0; q < QPL; ++q) {
    const int j = lane + 32 * q;
    if (4 * j < D)
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (4 * j + e < D) vf[4 * j + e] = v[q][e];
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < QPL; ++q) {
    const int j = lane + 32 * q;
    if (4 * j < D) {
      Real o[4];
      matvec4<Real, Real, Real>(sm.Pf, vf, D, Dp, j, o);
#pragma unroll
      for (int e = 0; e < 4; ++e) out[q][e] = -o[e];
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) out[q][e] = Real(0);
    }
  }
  __syncwarp();
}

// Jacobian diagonal estimate A (Real) for one evaluated column.
template <typename Real, int TK, int JAC, int QPL, int LPC = 32>
__device__ __forceinline__ void column_jacobian(const DevParams& P, const Smem<Real>& sm,
                                                const TapeKey& key, int t, int iter, bool acc,
                                                Real gp, const Col<Real, QPL>& c,
                                                Real (&A)[QPL][4]) {
  static_assert(TK == kDiagGauss || LPC == 32, "dense targets use whole warps per column");
  const int lane = threadIdx.x & (LPC - 1);
  const int D = static_cast<int>(P.D);
  const Real eps = static_cast<Real>(P.eps), inv2eps = static_cast<Real>(P.inv2eps);
  const Real* lamR = prec_of<Real>(P);
  if constexpr (JAC == kJacStoch) {
#pragma unroll
    for (int q = 0; q < QPL; ++q)
#pragma unroll
      for (int e = 0; e < 4; ++e) A[q][e] = Real(0);
    for (int k = 0; k < P.probes; ++k) {
      Real z[QPL][4], w[QPL][4], hvy[QPL][4];
#pragma unroll
      for (int q = 0; q < QPL; ++q) {
        const int j = lane + LPC * q;
        if (4 * j < D) {
          const U4 pb = probe_bits(key, static_cast<uint32_t>(j >> 5), static_cast<uint32_t>(t),
                                   k, iter);
          const uint32_t wv = u4_word(pb, (j >> 3) & 3);
          const int sh = (j & 7) * 4;
#pragma unroll
          for (int e = 0; e < 4; ++e) z[q][e] = ((wv >> (sh + e)) & 1u) ? Real(1) : Real(-1);
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e) z[q][e] = Real(0);
        }
      }
      if constexpr (TK == kDiagGauss) {
#pragma unroll
        for (int q = 0; q < QPL; ++q) {
          const int j = lane + LPC * q;
          Real lam[4] = {0, 0, 0, 0};
          if (4 * j < D) load4(lamR + 4 * j, lam);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            w[q][e] = z[q][e] + eps * (-lam[e] * z[q][e]);
            hvy[q][e] = -lam[e] * w[q][e];
          }
        }
      } else {
        Real hvx[QPL][4];
        dense_neg_pv<Real, QPL>(P, sm, z, hvx);
#pragma unroll
        for (int q = 0; q < QPL; ++q)
#pragma unroll
          for (int e = 0; e < 4; ++e) w[q][e] = z[q][e] + eps * hvx[q][e];
        dense_neg_pv<Real, QPL>(P, sm, w, hvy);
      }
      Real dla = 0;
#pragma unroll
      for (int q = 0; q < QPL; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const Real r = c.x[q][e] - c.y[q][e] - eps * c.gy[q][e];
          const Real dr = z[q][e] - w[q][e] - eps * hvy[q][e];
          dla += c.gy[q][e] * w[q][e] - c.gx[q][e] * z[q][e] - inv2eps * r * dr;
        }
      dla = seg_sum<LPC>(dla);
      const Real dg = gp * dla;
#pragma unroll
      for (int q = 0; q < QPL; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const Real jz = (acc ? w[q][e] : z[q][e]) + (c.y[q][e] - c.x[q][e]) * dg;
          A[q][e] += z[q][e] * jz;
        }
    }
    if (P.probes > 1) {
      const Real inv = Real(1) / static_cast<Real>(P.probes);
#pragma unroll
      for (int q = 0; q < QPL; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e) A[q][e] *= inv;
    }
  } else {
    // Exact diagonal: (J e_i)_i = a (1 + eps H_ii) + (1 - a) + (y_i - x_i) g(1-g) dlogalpha(e_i),
    // dlogalpha(e_i) = [(I + eps H) g_y]_i - g_x,i + 1/2 ([H r]_i + [H r]_i + eps [H H r]_i).
    if constexpr (TK == kDiagGauss) {
#pragma unroll
      for (int q = 0; q < QPL; ++q) {
        const int j = lane + LPC * q;
        Real lam[4] = {0, 0, 0, 0};
        if (4 * j < D) load4(lamR + 4 * j, lam);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const Real el = eps * lam[e];
          const Real r = c.x[q][e] - c.y[q][e] - eps * c.gy[q][e];
          const Real dl = (Real(1) - el) * c.gy[q][e] - c.gx[q][e] -
                          lam[e] * r * (Real(1) - Real(0.5) * el);
          A[q][e] = (acc ? Real(1) - el : Real(1)) + (c.y[q][e] - c.x[q][e]) * gp * dl;
        }
      }
    } else {
      Real r[QPL][4], pgy[QPL][4], pr[QPL][4], ppr[QPL][4];
#pragma unroll
      for (int q = 0; q < QPL; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e) r[q][e] = c.x[q][e] - c.y[q][e] - eps * c.gy[q][e];
      dense_neg_pv<Real, QPL>(P, sm, c.gy, pgy);  // -P g_y
      dense_neg_pv<Real, QPL>(P, sm, r, pr);      // -P r
      dense_neg_pv<Real, QPL>(P, sm, pr, ppr);    // P P r
      const int Dp = static_cast<int>(P.Dp);
#pragma unroll
      for (int q = 0; q < QPL; ++q) {
        const int j = lane + LPC * q;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int i = 4 * j + e;
          const Real pii = i < D ? sm.Pf[static_cast<size_t>(i) * Dp + i] : Real(0);
          const Real dl = c.gy[q][e] + eps * pgy[q][e] - c.gx[q][e] + pr[q][e] +
                          Real(0.5) * eps * ppr[q][e];
          A[q][e] = (acc ? Real(1) - eps * pii : Real(1)) + (c.y[q][e] - c.x[q][e]) * gp * dl;
        }
      }
    }
  }
}

}  // namespace pmcmc
