// logistic_adjoint.cu -- gradient of a trajectory objective with respect to
// epsilon for the logistic target, at a returned trajectory with its accept
// decisions held fixed.
//
// The objectives are those of the Gaussian adjoint:
//   esjd    = (1/T) sum_t min(1, alpha_t) |y_t - x_{t-1}|^2
//   mean_sq = (1/T) sum_t |x_t|^2
// with the MALA step of src/MALA/MALA.jl:207-229, 377-411 and the logistic
// model of bayes_logreg.jl:30-86.  The derivative is the reverse recurrence
//   lambda_t = c_t + J_{t+1}^T lambda_{t+1},  J_{t+1} = I + eps H(x_t) (accepted) or I,
//   dL/deps  = direct + sum_{t accepted} lambda_t . (g(x_{t-1}) + xi_t / sqrt(2 eps)),
// where c_t (the objective's gradient in x_t) and `direct` (its partial in eps)
// come from per-step terms.  Those need Hessian-vector products at x_{t-1} and
// y_t for every t, batched as GEMMs:
//   H(z) V = -X^T (p(1 - p) .* (X V)) - tau V,  p = sigmoid(X z).
// J_{t+1} is dense and changes with t, so the recurrence is not one affine scan
// of diagonal maps.  It is solved by Jacobi iterations on its diagonal part:
//   lambda^{k+1}_t = D_{t+1} lambda^{k+1}_{t+1} + c_t + (J_{t+1} - D_{t+1}) lambda^k_{t+1},
// D_{t+1} = 1 + eps diag H(x_t) = 1 - eps (X.*X)^T p(1 - p) - eps tau; each
// iteration is one batched HVP and one diagonal affine scan (the standalone
// look-back scan, run on the time-reversed arrays).  The fixed point is the
// exact recurrence; the iterations stop when max|lambda^{k+1} - lambda^k| <=
// 1e-12 max|lambda^{k+1}|.
//
// Everything runs in FP64 (cuBLAS DGEMM, pedantic math) whatever the state's
// type.  Layouts: D-vectors of column t at t * Dp (zero-padded to Dp); N x T
// matrices column-major (column t at t * N).
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "deer_device.cuh"
#include "logistic.h"
#include "pmcmc_rng.cuh"

namespace pmcmc {
namespace lga {

constexpr int kTh = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  }
  return s;  // valid in thread 0
}

// XB column t = x_{t-1} (x0 for t = 0) from S (T x D rows of Real) and x0; XI
// column t = xi_t and LU[t] = log u_t of the tape (seed, block).
template <typename Real>
__global__ void setup_kernel(const Real* __restrict__ S, const Real* __restrict__ x0, int D,
                             int Dp, int64_t T, uint64_t seed, uint64_t block,
                             double* __restrict__ XB, double* __restrict__ XI,
                             double* __restrict__ LU) {
  const TapeKey key(seed, block);
  const int nq = Dp / 4;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < T * nq;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = i / nq;
    const int j = static_cast<int>(i - t * nq);
    float n[4];
    tape_xi4(key, static_cast<uint32_t>(j), static_cast<uint32_t>(t), n);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int d = 4 * j + e;
      const bool in = d < D;
      XI[t * Dp + d] = in ? static_cast<double>(n[e]) : 0.0;
      XB[t * Dp + d] = in ? static_cast<double>(t == 0 ? x0[d] : S[(t - 1) * D + d]) : 0.0;
    }
    if (j == 0) LU[t] = log(static_cast<double>(tape_u(key, static_cast<uint32_t>(t))));
  }
}

// Per column t of L = X Z (N x T): R = y - p in place, W = p (1 - p), and the
// log-likelihood sum_n y_n L - softplus(L) into ll[t].  One block a column.
__global__ void lik_kernel(double* __restrict__ L, const double* __restrict__ ylab, int64_t N,
                           double* __restrict__ W, double* __restrict__ ll) {
  __shared__ double sh[kTh / 32];
  const int64_t t = blockIdx.x;
  double* col = L + t * N;
  double* wc = W + t * N;
  double s = 0.0;
  for (int64_t n = threadIdx.x; n < N; n += blockDim.x) {
    const double l = col[n];
    const double e = exp(-fabs(l));
    const double p = l >= 0 ? 1.0 / (1.0 + e) : e / (1.0 + e);
    s += ylab[n] * l - (fmax(l, 0.0) + log1p(e));
    col[n] = ylab[n] - p;
    wc[n] = p * (1.0 - p);
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) ll[t] = s;
}

// L .* W elementwise (N x T).
__global__ void mulw_kernel(double* __restrict__ L, const double* __restrict__ W, int64_t n) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    L[i] *= W[i];
}

// out = a * out + b * V over Dp x T (padded rows stay zero: V and out are zero there).
__global__ void axpby_kernel(double* __restrict__ out, double a, const double* __restrict__ V,
                             double b, int64_t n) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = a * out[i] + b * V[i];
}

// GX = G - tau XB;  Y = XB + eps GX + sqrt(2 eps) XI.
__global__ void propose_kernel(const double* __restrict__ XB, const double* __restrict__ XI,
                               double* __restrict__ GX, double* __restrict__ Y, double eps,
                               double tau, int64_t n) {
  const double c = sqrt(2.0 * eps);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double g = GX[i] - tau * XB[i];
    GX[i] = g;
    Y[i] = XB[i] + eps * g + c * XI[i];
  }
}

// Per column t: Q = XB - Y - eps GY, DY = GX + XI / sqrt(2 eps), E = Y - XB; log
// alpha (FP64, the sequential chain's formula), the accept flag, alpha, its
// derivative in log alpha and |E|^2.  One warp a column.
__global__ void local1_kernel(const double* __restrict__ XB, const double* __restrict__ Y,
                              const double* __restrict__ GX, const double* __restrict__ GY,
                              const double* __restrict__ XI, const double* __restrict__ LU,
                              const double* __restrict__ llx, const double* __restrict__ lly,
                              int Dp, int64_t T, double eps, double tau, double* __restrict__ Q,
                              double* __restrict__ DY, double* __restrict__ E,
                              double* __restrict__ sc) {
  const int lane = threadIdx.x & 31;
  const int64_t t = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (t >= T) return;
  const double rs = 1.0 / sqrt(2.0 * eps);
  double xx = 0, yy = 0, qq = 0, ii = 0, ee = 0;
  for (int d = lane; d < Dp; d += 32) {
    const int64_t k = t * Dp + d;
    const double x = XB[k], y = Y[k], xi = XI[k];
    const double q = x - y - eps * GY[k];
    const double e = y - x;
    Q[k] = q;
    DY[k] = GX[k] + xi * rs;
    E[k] = e;
    xx += x * x;
    yy += y * y;
    qq += q * q;
    ii += xi * xi;
    ee += e * e;
  }
  for (int o = 16; o > 0; o >>= 1) {
    xx += __shfl_xor_sync(0xffffffffu, xx, o);
    yy += __shfl_xor_sync(0xffffffffu, yy, o);
    qq += __shfl_xor_sync(0xffffffffu, qq, o);
    ii += __shfl_xor_sync(0xffffffffu, ii, o);
    ee += __shfl_xor_sync(0xffffffffu, ee, o);
  }
  if (lane == 0) {
    const double la = (lly[t] - 0.5 * tau * yy) - (llx[t] - 0.5 * tau * xx) - qq / (4.0 * eps) +
                      0.5 * ii;
    const bool acc = LU[t] < la;
    const double alpha = la < 0.0 ? exp(la) : 1.0;
    double* s = sc + 8 * t;
    s[0] = la;
    s[1] = acc ? 1.0 : 0.0;
    s[2] = alpha;
    s[3] = la < 0.0 ? alpha : 0.0;  // d alpha / d log alpha
    s[4] = ee;
    s[5] = qq;
  }
}

// Per column t (esjd): dq = -(DY + eps H(y) DY) - GY, the partial of log alpha
// in eps, and the direct term s[6] = dalpha dla e2 + alpha 2 E . DY; the vector
// w = Q + eps H(y) Q in place of HQ.  One warp a column.
__global__ void local2_kernel(const double* __restrict__ GY, const double* __restrict__ DY,
                              const double* __restrict__ Q, const double* __restrict__ E,
                              const double* __restrict__ HyDY, double* __restrict__ HyQ, int Dp,
                              int64_t T, double eps, double* __restrict__ sc) {
  const int lane = threadIdx.x & 31;
  const int64_t t = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (t >= T) return;
  double gd = 0, qdq = 0, edy = 0;
  for (int d = lane; d < Dp; d += 32) {
    const int64_t k = t * Dp + d;
    const double dy = DY[k], q = Q[k];
    const double dq = -(dy + eps * HyDY[k]) - GY[k];
    gd += GY[k] * dy;
    qdq += q * dq;
    edy += E[k] * dy;
    HyQ[k] = q + eps * HyQ[k];
  }
  for (int o = 16; o > 0; o >>= 1) {
    gd += __shfl_xor_sync(0xffffffffu, gd, o);
    qdq += __shfl_xor_sync(0xffffffffu, qdq, o);
    edy += __shfl_xor_sync(0xffffffffu, edy, o);
  }
  if (lane == 0) {
    double* s = sc + 8 * t;
    const double dla = gd - qdq / (2.0 * eps) + s[5] / (4.0 * eps * eps);
    s[6] = s[3] * dla * s[4] + s[2] * 2.0 * edy;
  }
}

// c_{t-1} (esjd) for t >= 1: (dalpha e2 v + alpha 2 eps H(x) E) / T with
// v = J_x GY - GX - (Q - J_x w) / (2 eps), J_x = I + eps H(x_{t-1}); c_{T-1} = 0.
__global__ void cvec_esjd_kernel(const double* __restrict__ GY, const double* __restrict__ GX,
                                 const double* __restrict__ Q, const double* __restrict__ Wv,
                                 const double* __restrict__ HxGY, const double* __restrict__ HxW,
                                 const double* __restrict__ HxE, const double* __restrict__ sc,
                                 int Dp, int64_t T, double eps, double* __restrict__ C) {
  const double invT = 1.0 / static_cast<double>(T);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < T * Dp;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = i / Dp + 1;  // the step whose terms land on column t - 1
    if (t >= T) {
      C[i] = 0.0;
      continue;
    }
    const int64_t k = i + Dp;  // column t
    const double* s = sc + 8 * t;
    const double jgy = GY[k] + eps * HxGY[k];
    const double jw = Wv[k] + eps * HxW[k];
    const double v = jgy - GX[k] - (Q[k] - jw) / (2.0 * eps);
    C[i] = (s[3] * s[4] * v + s[2] * 2.0 * eps * HxE[k]) * invT;
  }
}

// c_t (mean_sq) = 2 S_t / T: S_t is XB column t + 1, and the last row of S for t = T - 1.
template <typename Real>
__global__ void cvec_msq_kernel(const double* __restrict__ XB, const Real* __restrict__ S, int D,
                                int Dp, int64_t T, double* __restrict__ C) {
  const double k2 = 2.0 / static_cast<double>(T);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < T * Dp;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = i / Dp;
    const int d = static_cast<int>(i - t * Dp);
    const double st = t + 1 < T ? XB[i + Dp]
                      : d < D   ? static_cast<double>(S[(T - 1) * D + d])
                                : 0.0;
    C[i] = k2 * st;
  }
}

// DJ = 1 + eps (G - tau), G = -(X.*X)^T W computed by the caller.
__global__ void diagj_kernel(double* __restrict__ DJ, int D, int Dp, int64_t T, double eps,
                             double tau) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < T * Dp;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int d = static_cast<int>(i % Dp);
    DJ[i] = d < D ? 1.0 + eps * (-DJ[i] - tau) : 0.0;
  }
}

// The diagonal affine maps of one Jacobi iteration, time-reversed (row s holds
// step t = T - 1 - s): lambda_t = a_t lambda_{t+1} + b_t.  HL column t is
// H(x_t) lambda^k_{t+1} (t < T - 1).
__global__ void revmaps_kernel(const double* __restrict__ C, const double* __restrict__ LAM,
                               const double* __restrict__ HL, const double* __restrict__ DJ,
                               const double* __restrict__ sc, int Dp, int64_t T, double eps,
                               double* __restrict__ Ar, double* __restrict__ Br) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < T * Dp;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = i / Dp, d = i - t * Dp;
    const int64_t r = (T - 1 - t) * Dp + d;
    double a = 0.0, b = C[i];
    if (t + 1 < T) {
      if (sc[8 * (t + 1) + 1] != 0.0) {
        const double dj = DJ[i + Dp], lk = LAM[i + Dp];
        a = dj;
        b += lk + eps * HL[i] - dj * lk;
      } else {
        a = 1.0;
      }
    }
    Ar[r] = a;
    Br[r] = b;
  }
}

// LAM_new column t = Sr row T - 1 - t; per-block maxima of |new - old| and
// |new| into part[2 * block .. ].
__global__ void revgather_kernel(const double* __restrict__ Sr, double* __restrict__ LAM,
                                 int Dp, int64_t T, double* __restrict__ part) {
  __shared__ double sd[kTh], sm[kTh];
  double md = 0.0, mx = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < T * Dp;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = i / Dp, d = i - t * Dp;
    const double v = Sr[(T - 1 - t) * Dp + d];
    md = fmax(md, fabs(v - LAM[i]));
    mx = fmax(mx, fabs(v));
    LAM[i] = v;
  }
  sd[threadIdx.x] = md;
  sm[threadIdx.x] = mx;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sd[threadIdx.x] = fmax(sd[threadIdx.x], sd[threadIdx.x + o]);
      sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sd[0];
    part[2 * blockIdx.x + 1] = sm[0];
  }
}

// out[0] = sum_t direct_t / T (esjd) + sum_{t accepted} LAM_t . DY_t, in a
// fixed order (one block).
__global__ void final_kernel(const double* __restrict__ LAM, const double* __restrict__ DY,
                             const double* __restrict__ sc, int Dp, int64_t T, int esjd,
                             double* __restrict__ out) {
  __shared__ double sh[kTh / 32];
  double s = 0.0;
  for (int64_t t = threadIdx.x; t < T; t += blockDim.x) {
    const double* st = sc + 8 * t;
    if (esjd) s += st[6] / static_cast<double>(T);
    if (st[1] != 0.0) {
      double v = 0.0;
      for (int d = 0; d < Dp; ++d) v += LAM[t * Dp + d] * DY[t * Dp + d];
      s += v;
    }
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) out[0] = s;
}

inline int grid_for(int64_t n) {
  const int64_t g = (n + kTh - 1) / kTh;
  return static_cast<int>(g < 148 * 8 ? (g > 0 ? g : 1) : 148 * 8);
}

}  // namespace lga

namespace {

// The workspace carve of lg_adjoint, in doubles: every array rounded up to 32
// (256 bytes).  The size and the carve both come from here.
struct AdjLayout {
  size_t v, m;  // one Dp x T and one N x T array
  int gpart;
  size_t total;  // doubles
};

inline size_t r32(size_t n) { return (n + 31) & ~size_t(31); }

AdjLayout adj_layout(int64_t N, int64_t Dp, int64_t T) {
  AdjLayout a{};
  a.v = static_cast<size_t>(Dp) * T;
  a.m = static_cast<size_t>(N) * T;
  a.gpart = lga::grid_for(Dp * T);
  const size_t t = static_cast<size_t>(T);
  a.total = 16 * r32(a.v) + 3 * r32(a.m) + 3 * r32(t) + r32(8 * t) +
            r32(2 * static_cast<size_t>(a.gpart)) + r32(8) + r32(static_cast<size_t>(Dp));
  return a;
}

}  // namespace

size_t lg_adjoint_ws_bytes(const LogisticDev& X, int64_t T) {
  return 8 * adj_layout(X.N, X.Dp, T).total;
}

namespace {

// H(z) V for the columns [c0, c0 + n) of V against the W columns [w0, w0 + n):
// out = -X^T (W .* (X V)) - tau V.
int hvp(cudaStream_t s, cublasHandle_t cb, const LogisticDev& X, const double* W, const double* V,
        int64_t n, double* L, double* out) {
  const double one = 1.0, zero = 0.0, mone = -1.0;
  const int N = static_cast<int>(X.N), dp = static_cast<int>(X.Dp), nc = static_cast<int>(n);
  if (cublasDgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, N, nc, dp, &one, X.X64, dp, V, dp, &zero, L, N) !=
      CUBLAS_STATUS_SUCCESS)
    return 3;
  lga::mulw_kernel<<<lga::grid_for(X.N * n), lga::kTh, 0, s>>>(L, W, X.N * n);
  if (cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, dp, nc, N, &mone, X.X64, dp, L, N, &zero, out,
                  dp) != CUBLAS_STATUS_SUCCESS)
    return 3;
  lga::axpby_kernel<<<lga::grid_for(X.Dp * n), lga::kTh, 0, s>>>(out, 1.0, V, -X.tau, X.Dp * n);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

}  // namespace

int lg_adjoint(cudaStream_t s, cublasHandle_t cb, const LogisticDev& X, bool f64,
               const void* x0, const void* S, uint64_t seed, uint64_t block, int64_t T,
               double eps, int esjd, void* ws, int max_iter, double* grad_eps, int* iters,
               ScanFn scan, void* scan_ctx) {
  using namespace lga;
  const int64_t Dp = X.Dp, N = X.N;
  const int D = static_cast<int>(X.D);
  const AdjLayout Ly = adj_layout(N, Dp, T);
  const size_t v = Ly.v, m = Ly.m;
  double* p = static_cast<double*>(ws);
  double* const end = p + Ly.total;
  auto take = [&](size_t n) {
    double* r = p;
    p += r32(n);
    return r;
  };
  double *XB = take(v), *XI = take(v), *GX = take(v), *Y = take(v), *GY = take(v), *Q = take(v),
         *DY = take(v), *E = take(v), *V1 = take(v), *V2 = take(v), *V3 = take(v), *V4 = take(v),
         *C = take(v), *LAM = take(v), *Ar = take(v), *Br = take(v);
  double *Lb = take(m), *Wx = take(m), *Wy = take(m);
  double *LU = take(T), *llx = take(T), *lly = take(T), *sc = take(8 * T);
  const int gpart = Ly.gpart;
  double* part = take(2 * static_cast<size_t>(gpart));
  double* out = take(8);
  double* s0 = take(static_cast<size_t>(Dp));
  if (p > end) return 3;  // the carve must fit the layout it was sized from
  const double one = 1.0, zero = 0.0;
  const int n = static_cast<int>(N), dp = static_cast<int>(Dp), Tc = static_cast<int>(T);
  const int gv = grid_for(static_cast<int64_t>(v));
  if (f64)
    setup_kernel<double><<<gv, kTh, 0, s>>>(static_cast<const double*>(S),
                                            static_cast<const double*>(x0), D, dp, T, seed, block,
                                            XB, XI, LU);
  else
    setup_kernel<float><<<gv, kTh, 0, s>>>(static_cast<const float*>(S),
                                           static_cast<const float*>(x0), D, dp, T, seed, block,
                                           XB, XI, LU);
  // ---- forward quantities at x_{t-1} and y_t ----
  if (cublasDgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, n, Tc, dp, &one, X.X64, dp, XB, dp, &zero, Lb,
                  n) != CUBLAS_STATUS_SUCCESS)
    return 3;
  lik_kernel<<<Tc, kTh, 0, s>>>(Lb, X.y64, N, Wx, llx);
  if (cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, dp, Tc, n, &one, X.X64, dp, Lb, n, &zero, GX,
                  dp) != CUBLAS_STATUS_SUCCESS)
    return 3;
  propose_kernel<<<gv, kTh, 0, s>>>(XB, XI, GX, Y, eps, X.tau, static_cast<int64_t>(v));
  if (cublasDgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, n, Tc, dp, &one, X.X64, dp, Y, dp, &zero, Lb, n) !=
      CUBLAS_STATUS_SUCCESS)
    return 3;
  lik_kernel<<<Tc, kTh, 0, s>>>(Lb, X.y64, N, Wy, lly);
  if (cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, dp, Tc, n, &one, X.X64, dp, Lb, n, &zero, GY,
                  dp) != CUBLAS_STATUS_SUCCESS)
    return 3;
  axpby_kernel<<<gv, kTh, 0, s>>>(GY, 1.0, Y, -X.tau, static_cast<int64_t>(v));
  const int gw = static_cast<int>((32 * T + kTh - 1) / kTh);
  local1_kernel<<<gw, kTh, 0, s>>>(XB, Y, GX, GY, XI, LU, llx, lly, dp, T, eps, X.tau, Q, DY, E,
                                   sc);
  if (cudaGetLastError() != cudaSuccess) return 3;
  // ---- c_t and the direct term ----
  if (esjd) {
    if (hvp(s, cb, X, Wy, DY, T, Lb, V1)) return 3;  // H(y) DY
    if (hvp(s, cb, X, Wy, Q, T, Lb, V2)) return 3;   // H(y) Q
    local2_kernel<<<gw, kTh, 0, s>>>(GY, DY, Q, E, V1, V2, dp, T, eps, sc);  // V2 <- w
    if (hvp(s, cb, X, Wx, GY, T, Lb, V1)) return 3;  // H(x) GY
    if (hvp(s, cb, X, Wx, V2, T, Lb, V3)) return 3;  // H(x) w
    if (hvp(s, cb, X, Wx, E, T, Lb, V4)) return 3;   // H(x) E
    cvec_esjd_kernel<<<gv, kTh, 0, s>>>(GY, GX, Q, V2, V1, V3, V4, sc, dp, T, eps, C);
  } else if (f64) {
    cvec_msq_kernel<double><<<gv, kTh, 0, s>>>(XB, static_cast<const double*>(S), D, dp, T, C);
  } else {
    cvec_msq_kernel<float><<<gv, kTh, 0, s>>>(XB, static_cast<const float*>(S), D, dp, T, C);
  }
  // ---- D_t = diag J_t: 1 + eps diag H(x_{t-1}) ----
  double* DJ = V4;  // H(x) E is consumed
  if (cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, dp, Tc, n, &one, X.X2_64, dp, Wx, n, &zero, DJ,
                  dp) != CUBLAS_STATUS_SUCCESS)
    return 3;
  diagj_kernel<<<gv, kTh, 0, s>>>(DJ, D, dp, T, eps, X.tau);
  // ---- Jacobi iterations on lambda_t = c_t + J_{t+1} lambda_{t+1} ----
  if (cudaMemcpyAsync(LAM, C, 8 * v, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return 3;
  if (cudaMemsetAsync(s0, 0, 8 * Dp, s) != cudaSuccess) return 3;
  if (cudaMemsetAsync(V1, 0, 8 * v, s) != cudaSuccess) return 3;
  double* HL = V1;
  double* Sr = V3;
  int k = 0;
  bool done = false;
  std::vector<double> hp(2 * static_cast<size_t>(gpart));
  for (; k < max_iter && !done; ++k) {
    // HL column t = H(x_t) lambda^k_{t+1}: W column t + 1 (x_t = XB column t + 1)
    if (T > 1 && hvp(s, cb, X, Wx + N, LAM + Dp, T - 1, Lb, HL)) return 3;
    revmaps_kernel<<<gv, kTh, 0, s>>>(C, LAM, HL, DJ, sc, dp, T, eps, Ar, Br);
    if (cudaGetLastError() != cudaSuccess) return 3;
    const int rc = scan(scan_ctx, Dp, T, Ar, Br, s0, Sr);
    if (rc) return rc;
    revgather_kernel<<<gpart, kTh, 0, s>>>(Sr, LAM, dp, T, part);
    if (cudaMemcpyAsync(hp.data(), part, 8 * hp.size(), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return 3;
    double md = 0.0, mx = 0.0;
    for (int b = 0; b < gpart; ++b) {
      md = std::fmax(md, hp[2 * b]);
      mx = std::fmax(mx, hp[2 * b + 1]);
    }
    if (!std::isfinite(md) || !std::isfinite(mx)) return 4;
    done = md <= 1e-12 * mx || mx == 0.0;
  }
  final_kernel<<<1, kTh, 0, s>>>(LAM, DY, sc, dp, T, esjd, out);
  if (cudaMemcpyAsync(grad_eps, out, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return 3;
  *iters = k;
  return done ? 0 : 5;
}

}  // namespace pmcmc
