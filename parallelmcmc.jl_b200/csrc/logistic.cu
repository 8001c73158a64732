// logistic.cu -- Bayesian logistic regression target (bayes_logreg.jl:91-206).
//
// Per Newton sweep (stoch_diag, one probe) the batched fwd + JVP of
// MALA.jl:577-625 needs, for every trajectory column t,
//   pass 1 at x_bar_t and probe z_t:  l = X x_bar, v = X z      (N x 2T)
//                                     r = y - sigmoid(l), s = sigmoid'(l) v
//                                     g_lik = X' r, Hv_lik = -X' s, sum_n loglik
//   pass 2 at y_t and w_t = z + eps H(x) z: the same contractions.
// A pass is GEMM -> elementwise epilogue -> GEMM with an N x 2T intermediate.
// This file holds the data layout, the elementwise kernels around the passes
// and the plain FP32 pass (cuBLAS SGEMM/DGEMM with tensor-op math disabled,
// intermediate materialised in column chunks).  The tensor-core pass lives in
// logistic_tc.cu.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "deer_device.cuh"
#include "logistic.h"

namespace pmcmc {

// ---------------------------------------------------------------------------
// Elementwise kernels
// ---------------------------------------------------------------------------
// Pass modes without tangent columns in the first GEMM, and modes evaluated at y.
__host__ __device__ inline bool lg_value_only(int mode) { return mode == 2 || mode == 3 || mode == 4; }
__host__ __device__ inline bool lg_at_y(int mode) { return mode == 1 || mode == 4 || mode == 5; }

// B (Dp x ncols, column-major) for a column chunk [t0, t0+Tc):
//   mode 0: [x_bar_t | z_t]   (x_bar_t = S_{t-1}, or x0 at t = 0 / first sweep; z_t the
//                              Rademacher probe `probe` of this sweep)
//   mode 1: [y_t | w_t]
//   mode 2: [S_t]             (logp of the returned trajectory)
// and, for the exact diagonal (:diag, see lg_mid_kernel):
//   mode 3: [x_bar_t]         (the tangent half is filled by the epilogue)
//   mode 4: [y_t]
//   mode 5: [y_t | r_t],  r = x_bar - y - eps g_y
//   mode 6: [x_bar_t | u_t], u from lg_acc
// and zero the likelihood accumulators of the chunk.
template <typename Real>
__global__ void lg_prep_kernel(const DevParams* __restrict__ Pg, const DevState* __restrict__ st,
                               int mode, int64_t t0, int Tc, int probe, Real* __restrict__ B) {
  const DevParams& P = *Pg;
  const int64_t Dp = P.Dp, D = P.D;
  const int iter = st->iter;
  const int cur = st->cur;
  const bool from_x0 = iter == 0;
  const Real* S = static_cast<const Real*>(P.S[cur]);
  const Real* x0 = static_cast<const Real*>(P.x0);
  const int ncols = lg_value_only(mode) ? Tc : 2 * Tc;
  const int64_t n = static_cast<int64_t>(ncols) * Dp;
  const TapeKey key(P.seed, P.block);
  const Real eps = static_cast<Real>(P.eps);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(i / Dp);
    const int64_t d = i % Dp;
    const bool tangent = j >= Tc && !lg_value_only(mode);
    const int64_t t = t0 + (tangent ? j - Tc : j);
    Real v = Real(0);
    if (d < D && t < P.T) {
      const Real* xb = (from_x0 || t == 0) ? x0 : S + (t - 1) * Dp;
      if (mode >= 3) {
        const Real* lg1 = static_cast<const Real*>(P.lg[1]);
        if (mode == 3) v = xb[d];
        else if (mode == 4) v = lg1[t * Dp + d];
        else if (mode == 5)
          v = tangent ? xb[d] - lg1[t * Dp + d] -
                            eps * static_cast<const Real*>(P.lg[3])[t * Dp + d]
                      : lg1[t * Dp + d];
        else
          v = tangent ? static_cast<const Real*>(P.lg_acc)[t * Dp + d] : xb[d];
      } else if (mode == 0) {
        if (!tangent) {
          v = (from_x0 || t == 0) ? x0[d] : S[(t - 1) * Dp + d];
        } else {
          const U4 pb = probe_bits(key, static_cast<uint32_t>(d >> 7),
                                   static_cast<uint32_t>(t + P.t_off),
                                   probe, iter);
          v = ((u4_word(pb, static_cast<int>((d >> 5) & 3)) >> (d & 31)) & 1u) ? Real(1)
                                                                              : Real(-1);
        }
      } else if (mode == 1) {
        v = static_cast<const Real*>(P.lg[tangent ? 2 : 1])[t * Dp + d];
      } else {
        v = S[t * Dp + d];
      }
    }
    B[i] = v;
  }
  double* lp = lg_at_y(mode) ? P.lpy : P.lpx;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < Tc;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x)
    if (t0 + j < P.T) lp[t0 + j] = 0.0;
}

// Epilogue of a pass on the chunk intermediate L (N x ncols, column-major):
// value column t -> r = y - sigmoid(l) with loglik = y l - softplus(l) summed
// into lp[t] (FP64); tangent column -> s = sigmoid'(l) v (has_tangent = 1), or
// the weight sigmoid'(l) itself (has_tangent = 2: the diagonal of the Hessian,
// contracted with X .* X).
template <typename Real>
__global__ void lg_epilogue_kernel(const Real* __restrict__ ylab, int64_t N, int Tc,
                                   int has_tangent, Real* __restrict__ L, double* __restrict__ lp,
                                   int64_t tmax) {
  const int t = blockIdx.y;
  if (t >= tmax) return;
  Real* lv = L + static_cast<int64_t>(t) * N;
  Real* lt = L + static_cast<int64_t>(Tc + t) * N;
  double acc = 0.0;
  for (int64_t n = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; n < N;
       n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const Real l = lv[n];
    const Real e = exp(-fabs(l));
    const Real sp = (l > Real(0) ? l : Real(0)) + log1p(e);
    const Real p = l >= Real(0) ? Real(1) / (Real(1) + e) : e / (Real(1) + e);
    const Real yn = ylab[n];
    acc += static_cast<double>(yn * l - sp);
    lv[n] = yn - p;
    if (has_tangent == 1) lt[n] = p * (Real(1) - p) * lt[n];
    else if (has_tangent == 2) lt[n] = p * (Real(1) - p);
  }
  acc = warp_sum(acc);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) a += red[w];
    atomicAdd(lp + t, a);
  }
}

// After a pass: stage 1 -> g_x = X'r - tau x, H(x) z = -X's - tau z,
// y = x + eps g_x + sqrt(2 eps) xi, w = z + eps H(x) z;
// stage 2 -> g_y = X'r - tau y, H(y) w = -X's - tau w.
// G is Dp x 2Tc column-major (value block then tangent block).
//
// The exact diagonal of the surrogate Jacobian (:diag; the diagonal that
// jac_diag_via_jvps, DEER.jl:327-342, gathers from D JVPs of MALA.jl:732-797)
// is, with a the accept decision, g' the slope of the accept weight and
// r = x_bar - y - eps g_y,
//   J_ii = a (1 + eps H_x,ii) + (1 - a) + (y - x_bar)_i g' dla_i,
//   dla = (g_y - g_x) + H_y r / 2 + H_x (eps g_y + r / 2 + eps H_y r / 2),
// from four passes (modes 3-6) and these stages:
//   stage 3 -> g_x, y, diag H_x = -(X.*X)'w - tau       into lg[0], lg[1], lg[2];
//   stage 4 -> g_y                                      into lg[3];
//   stage 5 -> v = H_y r: u = eps g_y + r/2 + eps v/2   into lg_acc,
//              dla = g_y - g_x + v/2 so far              into lg[4];
//   stage 6 -> dla += H_x u                              in lg[4].
template <typename Real>
__global__ void lg_mid_kernel(const DevParams* __restrict__ Pg, const DevState* __restrict__ st,
                              int stage, int64_t t0, int Tc, int probe, const Real* __restrict__ G) {
  const DevParams& P = *Pg;
  const int64_t Dp = P.Dp, D = P.D;
  const int64_t nq = Dp / 4;
  const int iter = st->iter;
  const bool from_x0 = iter == 0;
  const Real* S = static_cast<const Real*>(P.S[st->cur]);
  const Real* x0 = static_cast<const Real*>(P.x0);
  const Real tau = static_cast<Real>(P.tau), eps = static_cast<Real>(P.eps);
  const Real c2 = static_cast<Real>(P.sqrt2eps);
  const TapeKey key(P.seed, P.block);
  const int64_t n = static_cast<int64_t>(Tc) * nq;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(i / nq);
    const int64_t q = i % nq;
    const int64_t t = t0 + j;
    if (t >= P.T) continue;
    const Real* gv = G + static_cast<int64_t>(j) * Dp + 4 * q;
    const Real* gt = G + static_cast<int64_t>(Tc + j) * Dp + 4 * q;
    const size_t o = static_cast<size_t>(t) * Dp + 4 * q;
    if (stage == 1) {
      float xi[4];
      {
        const float4 v = *reinterpret_cast<const float4*>(P.xi + t * Dp + 4 * q);
        xi[0] = v.x;
        xi[1] = v.y;
        xi[2] = v.z;
        xi[3] = v.w;
      }
      const U4 pb = probe_bits(key, static_cast<uint32_t>(q >> 5),
                               static_cast<uint32_t>(t + P.t_off),
                               probe, iter);
      const uint32_t wv = u4_word(pb, static_cast<int>((q >> 3) & 3));
      const int sh = static_cast<int>(q & 7) * 4;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int64_t d = 4 * q + e;
        Real gx = 0, y = 0, w = 0;
        if (d < D) {
          const Real x = (from_x0 || t == 0) ? x0[d] : S[(t - 1) * Dp + d];
          const Real z = ((wv >> (sh + e)) & 1u) ? Real(1) : Real(-1);
          gx = gv[e] - tau * x;
          const Real hvx = -gt[e] - tau * z;
          y = fma(c2, static_cast<Real>(xi[e]), fma(eps, gx, x));
          w = z + eps * hvx;
        }
        static_cast<Real*>(P.lg[0])[o + e] = gx;
        static_cast<Real*>(P.lg[1])[o + e] = y;
        static_cast<Real*>(P.lg[2])[o + e] = w;
      }
    } else if (stage == 2) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int64_t d = 4 * q + e;
        Real gy = 0, hvy = 0;
        if (d < D) {
          const Real y = static_cast<const Real*>(P.lg[1])[o + e];
          const Real w = static_cast<const Real*>(P.lg[2])[o + e];
          gy = gv[e] - tau * y;
          hvy = -gt[e] - tau * w;
        }
        static_cast<Real*>(P.lg[3])[o + e] = gy;
        static_cast<Real*>(P.lg[4])[o + e] = hvy;
      }
    } else {
      Real* lg0 = static_cast<Real*>(P.lg[0]);
      Real* lg1 = static_cast<Real*>(P.lg[1]);
      Real* lg2 = static_cast<Real*>(P.lg[2]);
      Real* lg3 = static_cast<Real*>(P.lg[3]);
      Real* lg4 = static_cast<Real*>(P.lg[4]);
      Real* uacc = static_cast<Real*>(P.lg_acc);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int64_t d = 4 * q + e;
        const bool in = d < D;
        const Real x = in ? ((from_x0 || t == 0) ? x0[d] : S[(t - 1) * Dp + d]) : Real(0);
        if (stage == 3) {
          Real gx = 0, y = 0, hd = 0;
          if (in) {
            gx = gv[e] - tau * x;
            y = fma(c2, static_cast<Real>(P.xi[t * Dp + d]), fma(eps, gx, x));
            hd = -gt[e] - tau;
          }
          lg0[o + e] = gx;
          lg1[o + e] = y;
          lg2[o + e] = hd;
        } else if (stage == 4) {
          lg3[o + e] = in ? gv[e] - tau * lg1[o + e] : Real(0);
        } else if (stage == 5) {
          Real u = 0, dl = 0;
          if (in) {
            const Real y = lg1[o + e], gy = lg3[o + e];
            const Real r = x - y - eps * gy;
            const Real v = -gt[e] - tau * r;
            u = eps * gy + Real(0.5) * r + Real(0.5) * eps * v;
            dl = (gy - lg0[o + e]) + Real(0.5) * v;
          }
          uacc[o + e] = u;
          lg4[o + e] = dl;
        } else {
          if (in) lg4[o + e] += -gt[e] - tau * uacc[o + e];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
int64_t lg_chunk_cols(int64_t N, int64_t T) {
  // keep the N x 2Tc intermediate under ~512 MB (FP32) / 1 GB (FP64)
  int64_t Tc = 1;
  while (Tc * 2 <= T && Tc * 2 * 2 * N * 4 <= (int64_t(512) << 20)) Tc *= 2;
  return Tc;
}

static int grid_for(int64_t n) {
  return static_cast<int>(n / 256 + 1 < 148 * 16 ? n / 256 + 1 : 148 * 16);
}

cudaError_t lg_prep(cudaStream_t s, bool f64, const DevParams* dP, const DevState* dS, int mode,
                    int64_t t0, int Tc, int probe, int64_t Dp, void* B) {
  const int ncols = mode == 2 ? Tc : 2 * Tc;
  const int g = grid_for(static_cast<int64_t>(ncols) * Dp);
  if (f64)
    lg_prep_kernel<double><<<g, 256, 0, s>>>(dP, dS, mode, t0, Tc, probe, static_cast<double*>(B));
  else
    lg_prep_kernel<float><<<g, 256, 0, s>>>(dP, dS, mode, t0, Tc, probe, static_cast<float*>(B));
  return cudaGetLastError();
}

cudaError_t lg_epilogue(cudaStream_t s, bool f64, const void* ylab, int64_t N, int Tc,
                        int has_tangent, void* L, double* lp, int64_t tmax) {
  dim3 grid(static_cast<unsigned>((N + 1023) / 1024 < 8 ? (N + 1023) / 1024 : 8),
            static_cast<unsigned>(Tc));
  if (f64)
    lg_epilogue_kernel<double><<<grid, 256, 0, s>>>(static_cast<const double*>(ylab), N, Tc,
                                                    has_tangent, static_cast<double*>(L), lp, tmax);
  else
    lg_epilogue_kernel<float><<<grid, 256, 0, s>>>(static_cast<const float*>(ylab), N, Tc,
                                                   has_tangent, static_cast<float*>(L), lp, tmax);
  return cudaGetLastError();
}

cudaError_t lg_mid(cudaStream_t s, bool f64, const DevParams* dP, const DevState* dS, int stage,
                   int64_t t0, int Tc, int probe, int64_t Dp, const void* G) {
  const int g = grid_for(static_cast<int64_t>(Tc) * (Dp / 4));
  if (f64)
    lg_mid_kernel<double><<<g, 256, 0, s>>>(dP, dS, stage, t0, Tc, probe,
                                            static_cast<const double*>(G));
  else
    lg_mid_kernel<float><<<g, 256, 0, s>>>(dP, dS, stage, t0, Tc, probe,
                                           static_cast<const float*>(G));
  return cudaGetLastError();
}

// One plain pass over all column chunks: prep -> L = X B -> epilogue -> G = X' L -> mid.
// mode 0/1 = pass 1/2 (mid stage 1/2), mode 2 = logp pass (no tangent, no mid),
// modes 3-6 = the passes of the exact diagonal (mid stages 3-6; mode 3 contracts
// the weights of its tangent half with X2 = X .* X).
int lg_plain_pass(cudaStream_t s, cublasHandle_t cb, const LogisticDev& X, bool f64,
                  const DevParams* dP, const DevState* dS, double* lp, int mode, int64_t T,
                  int64_t Dp, void* Bbuf, void* Lbuf, void* Gbuf, int64_t Tc, int probe) {
  const int64_t N = X.N;
  const int n = static_cast<int>(N), dp = static_cast<int>(Dp);
  // G = op(A) B for the column block [c0, c0 + nc) of L and G (A = X, or X2)
  auto gemm = [&](bool first, const void* A, int c0, int nc) -> bool {
    const size_t es = f64 ? 8 : 4;
    const unsigned char* Bp = static_cast<const unsigned char*>(Bbuf) + es * c0 * Dp;
    unsigned char* Lp = static_cast<unsigned char*>(Lbuf) + es * c0 * N;
    unsigned char* Gp = static_cast<unsigned char*>(Gbuf) + es * c0 * Dp;
    cublasStatus_t st;
    if (f64) {
      const double one = 1.0, zero = 0.0;
      st = first ? cublasDgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, n, nc, dp, &one,
                               static_cast<const double*>(A), dp,
                               reinterpret_cast<const double*>(Bp), dp, &zero,
                               reinterpret_cast<double*>(Lp), n)
                 : cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, dp, nc, n, &one,
                               static_cast<const double*>(A), dp,
                               reinterpret_cast<const double*>(Lp), n, &zero,
                               reinterpret_cast<double*>(Gp), dp);
    } else {
      const float one = 1.f, zero = 0.f;
      st = first ? cublasSgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, n, nc, dp, &one,
                               static_cast<const float*>(A), dp,
                               reinterpret_cast<const float*>(Bp), dp, &zero,
                               reinterpret_cast<float*>(Lp), n)
                 : cublasSgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, dp, nc, n, &one,
                               static_cast<const float*>(A), dp,
                               reinterpret_cast<const float*>(Lp), n, &zero,
                               reinterpret_cast<float*>(Gp), dp);
    }
    return st == CUBLAS_STATUS_SUCCESS;
  };
  const void* Xa = f64 ? static_cast<const void*>(X.X64) : static_cast<const void*>(X.X32);
  const void* X2 = f64 ? static_cast<const void*>(X.X2_64) : static_cast<const void*>(X.X2_32);
  if (mode == 3 && !X2) return 3;
  for (int64_t t0 = 0; t0 < T; t0 += Tc) {
    const int tc = static_cast<int>(Tc);
    const bool vo = lg_value_only(mode);
    if (lg_prep(s, f64, dP, dS, mode, t0, tc, probe, Dp, Bbuf) != cudaSuccess) return 3;
    if (!gemm(true, Xa, 0, vo ? tc : 2 * tc)) return 3;
    const int64_t tmax = T - t0 < Tc ? T - t0 : Tc;
    const int tang = mode == 3 ? 2 : (vo ? 0 : 1);
    if (lg_epilogue(s, f64, f64 ? static_cast<const void*>(X.y64) : static_cast<const void*>(X.y32),
                    N, tc, tang, Lbuf, lp + t0, tmax) != cudaSuccess)
      return 3;
    if (mode == 2) continue;
    if (mode == 3) {
      if (!gemm(false, Xa, 0, tc) || !gemm(false, X2, tc, tc)) return 3;
    } else if (!gemm(false, Xa, 0, vo ? tc : 2 * tc)) {
      return 3;
    }
    const int stage = mode <= 1 ? mode + 1 : mode;
    if (lg_mid(s, f64, dP, dS, stage, t0, tc, probe, Dp, Gbuf) != cudaSuccess) return 3;
  }
  return 0;
}

// X2 = X .* X (the rows and padding of X), for the diagonal of the Hessian.
template <typename Real>
__global__ void lg_square_kernel(const Real* __restrict__ X, Real* __restrict__ X2, int64_t n) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    X2[i] = X[i] * X[i];
}

cudaError_t lg_make_square(cudaStream_t s, LogisticDev& X, bool f64) {
  const int64_t n = X.N * X.Dp;
  const int g = grid_for(n);
  if (f64) {
    if (X.X2_64) return cudaSuccess;
    cudaError_t e = cudaMalloc(&X.X2_64, 8 * n);
    if (e != cudaSuccess) return e;
    lg_square_kernel<double><<<g, 256, 0, s>>>(X.X64, X.X2_64, n);
  } else {
    if (X.X2_32) return cudaSuccess;
    cudaError_t e = cudaMalloc(&X.X2_32, 4 * n);
    if (e != cudaSuccess) return e;
    lg_square_kernel<float><<<g, 256, 0, s>>>(X.X32, X.X2_32, n);
  }
  return cudaGetLastError();
}

}  // namespace pmcmc
