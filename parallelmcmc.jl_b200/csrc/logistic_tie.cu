// logistic_tie.cu -- FP64 decisions for near-tie columns of the logistic target,
// and the verification pass at a returned trajectory.
//
// The accept decision of column t compares log u_t with log alpha_t
// (MALA.jl:402-404, strict <).  With FP32 state and the 22-bit tensor-core
// contractions, log alpha carries an absolute error of about 1e-5 .. 1e-4:
// each of the N log-likelihood terms of lp(x) and lp(y) is rounded on its own,
// and their errors add up over the rows.  A column whose margin
// |log alpha - log u| lies inside that band can change its decision from one
// Newton sweep to the next while the iterate moves only by rounding-level
// amounts; every change moves the trajectory after the column, and the solve
// stalls (N = 10000, D = 256, T = 65536: 369 sweeps where the FP64 solve takes
// 49, and accept flags that differ from the FP64 sequential chain).
//
// The sequential FP64 chain (MALA.jl:377-411, bayes_logreg.jl:37-58) decides
// such a column by its exact log alpha.  So after the contraction passes of a
// sweep:
//   1. tie_margin_kernel: log alpha_t of every column from the sweep's
//      quantities (the value the sweep kernel would use) and |margin_t|;
//   2. tie_select_kernel: the columns whose margin is inside a band, in column
//      order (deterministic), at most kmax of them: the widest of four nested
//      bands whose count fits;
//   3. for those columns, in FP64 from the FP64 design matrix: the gradient at
//      x_bar_t = S_{t-1}, the proposal y_t = x_bar + eps g + sqrt(2 eps) xi_t,
//      lp(x_bar), lp(y), the gradient at y and both log proposal densities
//      (logq_mala, MALA.jl:172-193) -- four DGEMMs over the selected columns
//      with FP64 elementwise kernels between them;
//   4. tie_final_kernel: log alpha_t in FP64 replaces the sweep's value.
// The sweep kernel then reads log alpha from la_ref for every column.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "deer_device.cuh"
#include "logistic.h"

namespace pmcmc {
namespace tie {

constexpr int kSelThreads = 1024;
constexpr int kBands = 4;  // band, band / 4, band / 16, band / 64

__device__ __forceinline__ int grid_cap(int64_t n, int per) {
  const int64_t g = (n + per - 1) / per;
  return static_cast<int>(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

// log alpha_t as the sweep computes it (column_logistic in deer_sweep.cu):
//   sum_d [-tau/2 (y^2 - x^2) + (r1^2 - r2^2) / (4 eps)] + lpy_t - lpx_t,
//   r1 = sqrt(2 eps) xi, r2 = (x - y) - eps g_y, in FP64 from the state's
// precision.  One warp a column.
template <typename Real>
__global__ void tie_margin_kernel(const DevParams* __restrict__ Pg,
                                  const DevState* __restrict__ st, double* __restrict__ la_ref,
                                  float* __restrict__ mg) {
  const DevParams& P = *Pg;
  const int lane = threadIdx.x & 31;
  const int64_t D = P.D, Dp = P.Dp;
  const bool from_x0 = st->iter == 0;
  const Real* S = static_cast<const Real*>(P.S[st->cur]);
  const Real* x0 = static_cast<const Real*>(P.x0);
  const Real* yv = static_cast<const Real*>(P.lg[1]);
  const Real* gyv = static_cast<const Real*>(P.lg[3]);
  const int64_t nw = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
       t < P.T; t += nw) {
    const Real* xb = (from_x0 || t == 0) ? x0 : S + (t - 1) * Dp;
    double la = 0.0;
    for (int64_t d = lane; d < D; d += 32) {
      const double xd = static_cast<double>(xb[d]);
      const double yd = static_cast<double>(yv[t * Dp + d]);
      const double r1 = P.sqrt2eps * static_cast<double>(P.xi[t * Dp + d]);
      const double r2 = (xd - yd) - P.eps * static_cast<double>(gyv[t * Dp + d]);
      la += -0.5 * P.tau * (yd * yd - xd * xd) + (r1 * r1 - r2 * r2) * P.inv4eps;
    }
    la = warp_sum(la) + (P.lpy[t] - P.lpx[t]);
    if (lane == 0) {
      la_ref[t] = la;
      mg[t] = static_cast<float>(fabs(la - P.logu[t]));
    }
  }
}

// Near-tie columns, in column order: the widest of the bands band / 4^i whose
// count is at most kmax (the narrowest one, truncated to its first kmax
// columns, if none fits).  One CTA; thread i owns a contiguous run of columns.
// info[0] = columns selected, info[1] = columns inside the widest band,
// info[2] = band index used.
__global__ void __launch_bounds__(kSelThreads)
    tie_select_kernel(const float* __restrict__ mg, int64_t T, float band, int kmax,
                      int32_t* __restrict__ list, int32_t* __restrict__ info) {
  __shared__ int s_cnt[kBands][kSelThreads / 32];
  __shared__ int s_base[kSelThreads / 32];
  __shared__ int s_band;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t run = (T + kSelThreads - 1) / kSelThreads;
  const int64_t c0 = imin64(T, tid * run), c1 = imin64(T, c0 + run);
  int cnt[kBands] = {0, 0, 0, 0};
  for (int64_t t = c0; t < c1; ++t) {
    const float m = mg[t];
    float b = band;
#pragma unroll
    for (int i = 0; i < kBands; ++i, b *= 0.25f) cnt[i] += m < b ? 1 : 0;
  }
#pragma unroll
  for (int i = 0; i < kBands; ++i) {
    const int s = warp_sum(cnt[i]);
    if (lane == 0) s_cnt[i][warp] = s;
  }
  __syncthreads();
  if (tid == 0) {
    int bi = kBands - 1;
    int tot[kBands];
    for (int i = 0; i < kBands; ++i) {
      tot[i] = 0;
      for (int w = 0; w < kSelThreads / 32; ++w) tot[i] += s_cnt[i][w];
    }
    for (int i = 0; i < kBands; ++i)
      if (tot[i] <= kmax) {
        bi = i;
        break;
      }
    s_band = bi;
    info[0] = tot[bi] < kmax ? tot[bi] : kmax;
    info[1] = tot[0];
    info[2] = bi;
  }
  __syncthreads();
  const int bi = s_band;
  float b = band;
  for (int i = 0; i < bi; ++i) b *= 0.25f;
  // exclusive scan of this thread's count in band bi (warp shuffles, then warps)
  int mine = 0;
#pragma unroll
  for (int i = 0; i < kBands; ++i)
    if (i == bi) mine = cnt[i];
  int incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (tid == 0) {
    int acc = 0;
    for (int w = 0; w < kSelThreads / 32; ++w) {
      s_base[w] = acc;
      acc += s_cnt[bi][w];
    }
  }
  __syncthreads();
  int pos = s_base[warp] + incl - mine;
  for (int64_t t = c0; t < c1 && pos < kmax; ++t)
    if (mg[t] < b) list[pos++] = static_cast<int32_t>(t);
}

// B[k] (Dp doubles) = x_bar of selected column k; zero beyond the selection.
template <typename Real>
__global__ void tie_gather_kernel(const DevParams* __restrict__ Pg,
                                  const DevState* __restrict__ st,
                                  const int32_t* __restrict__ list,
                                  const int32_t* __restrict__ info, int kmax,
                                  double* __restrict__ B) {
  const DevParams& P = *Pg;
  const int64_t Dp = P.Dp;
  const int cnt = info[0];
  const bool from_x0 = st->iter == 0;
  const Real* S = static_cast<const Real*>(P.S[st->cur]);
  const Real* x0 = static_cast<const Real*>(P.x0);
  const int64_t n = static_cast<int64_t>(kmax) * Dp;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(i / Dp);
    const int64_t d = i % Dp;
    double v = 0.0;
    if (k < cnt && d < P.D) {
      const int64_t t = list[k];
      v = static_cast<double>((from_x0 || t == 0) ? x0[d] : S[(t - 1) * Dp + d]);
    }
    B[i] = v;
  }
}

// Column k of L (N logits): r = y - sigmoid(l) in place, lp[k] = sum_n
// y l - softplus(l) (bayes_logreg.jl:37-58 with the stable softplus of
// docs/src/15-gpu.md:91-97), in FP64, summed in a fixed order.
__global__ void tie_loglik_kernel(const double* __restrict__ ylab, int64_t N,
                                  const int32_t* __restrict__ info, double* __restrict__ L,
                                  double* __restrict__ lp) {
  __shared__ double red[32];
  const int k = blockIdx.x;
  double* l = L + static_cast<int64_t>(k) * N;
  if (k >= info[0]) {
    for (int64_t n = threadIdx.x; n < N; n += blockDim.x) l[n] = 0.0;
    if (threadIdx.x == 0) lp[k] = 0.0;
    return;
  }
  double acc = 0.0;
  for (int64_t n = threadIdx.x; n < N; n += blockDim.x) {
    const double z = l[n];
    const double e = exp(-fabs(z));
    const double sp = (z > 0.0 ? z : 0.0) + log1p(e);
    const double p = z >= 0.0 ? 1.0 / (1.0 + e) : e / (1.0 + e);
    acc += ylab[n] * z - sp;
    l[n] = ylab[n] - p;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) a += red[w];
    lp[k] = a;
  }
}

// gx = X'r - tau x_bar (bayes_logreg.jl:48-58), y = x_bar + eps gx + sqrt(2 eps) xi
// (MALA.jl:221-222), column by column over the selection.
__global__ void tie_propose_kernel(const DevParams* __restrict__ Pg,
                                   const int32_t* __restrict__ list,
                                   const int32_t* __restrict__ info, int kmax,
                                   const double* __restrict__ Bx, const double* __restrict__ G,
                                   double* __restrict__ GX, double* __restrict__ By) {
  const DevParams& P = *Pg;
  const int64_t Dp = P.Dp;
  const int cnt = info[0];
  const int64_t n = static_cast<int64_t>(kmax) * Dp;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(i / Dp);
    const int64_t d = i % Dp;
    double gx = 0.0, y = 0.0;
    if (k < cnt && d < P.D) {
      const int64_t t = list[k];
      const double x = Bx[i];
      gx = G[i] - P.tau * x;
      y = x + P.eps * gx + P.sqrt2eps * static_cast<double>(P.xi[t * Dp + d]);
    }
    GX[i] = gx;
    By[i] = y;
  }
}

// log alpha_t = [lp(y) + logq(x|y)] - [lp(x) + logq(y|x)] (MALA.jl:172-193,
// 402) in FP64 for every selected column; one warp a column.
__global__ void tie_final_kernel(const DevParams* __restrict__ Pg,
                                 const int32_t* __restrict__ list,
                                 const int32_t* __restrict__ info, int kmax,
                                 const double* __restrict__ Bx, const double* __restrict__ By,
                                 const double* __restrict__ GX, const double* __restrict__ G,
                                 const double* __restrict__ lpx, const double* __restrict__ lpy,
                                 double* __restrict__ la_ref) {
  const DevParams& P = *Pg;
  const int lane = threadIdx.x & 31;
  const int64_t Dp = P.Dp;
  const int cnt = info[0];
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < cnt; k += nw) {
    const double* x = Bx + static_cast<int64_t>(k) * Dp;
    const double* y = By + static_cast<int64_t>(k) * Dp;
    const double* gx = GX + static_cast<int64_t>(k) * Dp;
    const double* g2 = G + static_cast<int64_t>(k) * Dp;
    double xx = 0.0, yy = 0.0, q1 = 0.0, q2 = 0.0;
    for (int64_t d = lane; d < P.D; d += 32) {
      const double gy = g2[d] - P.tau * y[d];
      const double a = y[d] - (x[d] + P.eps * gx[d]);
      const double b = x[d] - (y[d] + P.eps * gy);
      xx += x[d] * x[d];
      yy += y[d] * y[d];
      q1 += a * a;
      q2 += b * b;
    }
    xx = warp_sum(xx);
    yy = warp_sum(yy);
    q1 = warp_sum(q1);
    q2 = warp_sum(q2);
    if (lane == 0) {
      const double lp_x = lpx[k] - 0.5 * P.tau * xx, lp_y = lpy[k] - 0.5 * P.tau * yy;
      la_ref[list[k]] = (lp_y - q2 * P.inv4eps) - (lp_x - q1 * P.inv4eps);
    }
  }
}

// Verification at a returned trajectory S (after the contraction passes at
// x_bar_t = S_{t-1}): the decision by la_ref, f_t = accept ? y_t : x_bar_t,
// the defect max_d |S_t - f_t| (max into the state), the accept flag and the
// signed margin of every column.
template <typename Real>
__global__ void lg_verify_kernel(const DevParams* __restrict__ Pg, DevState* __restrict__ st,
                                 const double* __restrict__ la_ref) {
  __shared__ double red[32];
  const DevParams& P = *Pg;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t D = P.D, Dp = P.Dp;
  const Real* S = static_cast<const Real*>(P.S[st->cur]);
  const Real* x0 = static_cast<const Real*>(P.x0);
  const Real* yv = static_cast<const Real*>(P.lg[1]);
  const int64_t nw = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  double def = 0.0;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp; t < P.T;
       t += nw) {
    const Real* xb = t == 0 ? x0 : S + (t - 1) * Dp;
    const double la = la_ref[t], logu = P.logu[t];
    const bool acc = logu < la;
    for (int64_t d = lane; d < D; d += 32) {
      const Real f = acc ? yv[t * Dp + d] : xb[d];
      def = fmax(def, fabs(static_cast<double>(S[t * Dp + d]) - static_cast<double>(f)));
    }
    if (lane == 0) {
      P.acc_col[t] = acc ? 1 : 0;
      P.la_col[t] = la - logu;
    }
  }
  def = warp_max(def);
  if (lane == 0) red[warp] = def;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    if (m > 0) atomicMax(&st->max_defect_bits, dbits(m));
  }
}

}  // namespace tie

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {
size_t up256(size_t b) { return (b + 255) & ~size_t(255); }
}  // namespace

size_t lg_tie_ws_bytes(const LogisticDev& X, int64_t T, int kmax) {
  const size_t K = static_cast<size_t>(kmax), Dp = static_cast<size_t>(X.Dp);
  return up256(4 * static_cast<size_t>(T)) + up256(4 * K) + up256(16) +
         5 * up256(8 * Dp * K) + up256(8 * static_cast<size_t>(X.N) * K) + 2 * up256(8 * K);
}

TieBufs lg_tie_carve(void* ws, const LogisticDev& X, int64_t T, int kmax) {
  TieBufs b{};
  const size_t K = static_cast<size_t>(kmax), Dp = static_cast<size_t>(X.Dp);
  unsigned char* p = static_cast<unsigned char*>(ws);
  auto take = [&](size_t bytes) {
    unsigned char* q = p;
    p += up256(bytes);
    return q;
  };
  b.kmax = kmax;
  b.mg = reinterpret_cast<float*>(take(4 * static_cast<size_t>(T)));
  b.list = reinterpret_cast<int32_t*>(take(4 * K));
  b.info = reinterpret_cast<int32_t*>(take(16));
  b.Bx = reinterpret_cast<double*>(take(8 * Dp * K));
  b.By = reinterpret_cast<double*>(take(8 * Dp * K));
  b.GX = reinterpret_cast<double*>(take(8 * Dp * K));
  b.G = reinterpret_cast<double*>(take(8 * Dp * K));
  b.G2 = reinterpret_cast<double*>(take(8 * Dp * K));
  b.L = reinterpret_cast<double*>(take(8 * static_cast<size_t>(X.N) * K));
  b.lpx = reinterpret_cast<double*>(take(8 * K));
  b.lpy = reinterpret_cast<double*>(take(8 * K));
  return b;
}

cudaError_t lg_margin(cudaStream_t s, bool f64, const DevParams* dP, const DevState* dS,
                      int64_t T, double* la_ref, float* mg) {
  const int g = static_cast<int>((T + 7) / 8 < 148 * 16 ? (T + 7) / 8 : 148 * 16);
  if (f64) tie::tie_margin_kernel<double><<<g, 256, 0, s>>>(dP, dS, la_ref, mg);
  else tie::tie_margin_kernel<float><<<g, 256, 0, s>>>(dP, dS, la_ref, mg);
  return cudaGetLastError();
}

int lg_tie_refine(cudaStream_t s, cublasHandle_t cb, const LogisticDev& X, bool f64,
                  const DevParams* dP, const DevState* dS, int64_t T, double* la_ref,
                  const TieBufs& b, float band) {
  const int K = b.kmax;
  const int64_t N = X.N, Dp = X.Dp;
  if (lg_margin(s, f64, dP, dS, T, la_ref, b.mg) != cudaSuccess) return 3;
  tie::tie_select_kernel<<<1, tie::kSelThreads, 0, s>>>(b.mg, T, band, K, b.list, b.info);
  if (cudaGetLastError() != cudaSuccess) return 3;
  const int64_t nk = static_cast<int64_t>(K) * Dp;
  const int ge = static_cast<int>((nk + 255) / 256 < 148 * 16 ? (nk + 255) / 256 : 148 * 16);
  if (f64) tie::tie_gather_kernel<double><<<ge, 256, 0, s>>>(dP, dS, b.list, b.info, K, b.Bx);
  else tie::tie_gather_kernel<float><<<ge, 256, 0, s>>>(dP, dS, b.list, b.info, K, b.Bx);
  if (cudaGetLastError() != cudaSuccess) return 3;
  const double one = 1.0, zero = 0.0;
  const int n = static_cast<int>(N), dp = static_cast<int>(Dp);
  // L = X Bx (N x K), X row-major N x Dp = column-major Dp x N
  if (cublasDgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, n, K, dp, &one, X.X64, dp, b.Bx, dp, &zero, b.L,
                  n) != CUBLAS_STATUS_SUCCESS)
    return 3;
  tie::tie_loglik_kernel<<<K, 256, 0, s>>>(X.y64, N, b.info, b.L, b.lpx);
  if (cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, dp, K, n, &one, X.X64, dp, b.L, n, &zero, b.G,
                  dp) != CUBLAS_STATUS_SUCCESS)
    return 3;
  tie::tie_propose_kernel<<<ge, 256, 0, s>>>(dP, b.list, b.info, K, b.Bx, b.G, b.GX, b.By);
  if (cublasDgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, n, K, dp, &one, X.X64, dp, b.By, dp, &zero, b.L,
                  n) != CUBLAS_STATUS_SUCCESS)
    return 3;
  tie::tie_loglik_kernel<<<K, 256, 0, s>>>(X.y64, N, b.info, b.L, b.lpy);
  if (cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, dp, K, n, &one, X.X64, dp, b.L, n, &zero, b.G2,
                  dp) != CUBLAS_STATUS_SUCCESS)
    return 3;
  const int gf = (K + 7) / 8;
  tie::tie_final_kernel<<<gf, 256, 0, s>>>(dP, b.list, b.info, K, b.Bx, b.By, b.GX, b.G2, b.lpx,
                                           b.lpy, la_ref);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

cudaError_t lg_verify(cudaStream_t s, bool f64, const DevParams* dP, DevState* dS, int64_t T,
                      const double* la_ref) {
  const int g = static_cast<int>((T + 7) / 8 < 148 * 16 ? (T + 7) / 8 : 148 * 16);
  if (f64) tie::lg_verify_kernel<double><<<g, 256, 0, s>>>(dP, dS, la_ref);
  else tie::lg_verify_kernel<float><<<g, 256, 0, s>>>(dP, dS, la_ref);
  return cudaGetLastError();
}

}  // namespace pmcmc
