// Mass-matrix support (M = L L^T, L lower triangular): the two linear maps that
// carry a chain between the target's coordinates x and the whitened ones
// x' = L^-1 x.
//
// The reference applies the Cholesky factor inside every MALA step
// (src/MALA/MALA.jl:29-47: M g = L (L^T g), noise L xi, quadratic form through
// L \ r, log det M): the proposal is y = x + eps M g + sqrt(2 eps) L xi.  With
// x = L x' this is y' = x' + eps L^T g + sqrt(2 eps) xi, and L^T g is the
// gradient of the whitened log density at x'; the proposal densities differ by
// the constant log det M on both sides of log alpha.  So the chain with mass M
// is exactly plain MALA on the whitened target driven by the same tape, and the
// solve runs there: x0 is whitened once, and the trajectory maps back column by
// column.  Both maps are O(D^2) per column against the solve's O(D^2) per
// column per Newton sweep, and run in FP64 whatever the state's type.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "deer_launch.h"

namespace pmcmc {
namespace {

// x' = L^-1 x by forward substitution, one warp per vector (block b solves
// vector b), the lanes splitting each row's dot product; the solved prefix
// stays in shared memory.
template <typename Real>
__global__ void mass_whiten_kernel(const double* __restrict__ L, int64_t D,
                                   const Real* __restrict__ xs, Real* __restrict__ ysout) {
  extern __shared__ double ys[];
  const int lane = threadIdx.x;
  const Real* x = xs + static_cast<int64_t>(blockIdx.x) * D;
  Real* y = ysout + static_cast<int64_t>(blockIdx.x) * D;
  for (int64_t i = 0; i < D; ++i) {
    double s = 0.0;
    for (int64_t k = lane; k < i; k += 32) s += L[k * D + i] * ys[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) ys[i] = (static_cast<double>(x[i]) - s) / L[i * D + i];
    __syncwarp();
  }
  for (int64_t i = lane; i < D; i += 32) y[i] = static_cast<Real>(ys[i]);
}

// S[:, j] <- L S[:, j] in place for every column j: one warp per column, the
// column staged in shared memory before any lane writes, lane i computing
// rows i, i + 32, ... (L is column-major, so the lanes read L coalesced).
template <typename Real>
__global__ void mass_map_kernel(const double* __restrict__ L, int64_t D, int64_t N,
                                Real* __restrict__ S) {
  extern __shared__ double vs_all[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  double* v = vs_all + static_cast<int64_t>(warp) * D;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * wpb + warp; j < N;
       j += static_cast<int64_t>(gridDim.x) * wpb) {
    Real* col = S + j * D;
    for (int64_t i = lane; i < D; i += 32) v[i] = static_cast<double>(col[i]);
    __syncwarp();
    for (int64_t i = lane; i < D; i += 32) {
      double acc = 0.0;
      for (int64_t k = 0; k <= i; ++k) acc += L[k * D + i] * v[k];
      col[i] = static_cast<Real>(acc);
    }
    __syncwarp();
  }
}

}  // namespace

int64_t mass_max_dim() { return 4096; }

cudaError_t mass_whiten(cudaStream_t s, const double* L, int64_t D, int64_t n, const void* x,
                        void* y, bool f64) {
  if (D < 1 || D > mass_max_dim() || n < 1 || n > (int64_t(1) << 31) - 1)
    return cudaErrorInvalidValue;
  const size_t smem = sizeof(double) * static_cast<size_t>(D);
  const unsigned grid = static_cast<unsigned>(n);
  if (f64)
    mass_whiten_kernel<double><<<grid, 32, smem, s>>>(L, D, static_cast<const double*>(x),
                                                     static_cast<double*>(y));
  else
    mass_whiten_kernel<float><<<grid, 32, smem, s>>>(L, D, static_cast<const float*>(x),
                                                    static_cast<float*>(y));
  return cudaGetLastError();
}

cudaError_t mass_map(cudaStream_t s, const double* L, int64_t D, int64_t N, void* S, bool f64,
                     int num_sms) {
  if (D < 1 || D > mass_max_dim() || N < 0) return cudaErrorInvalidValue;
  if (N == 0) return cudaSuccess;
  // warps per block such that the staged columns fit the default 48 KB
  const int wpb = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(8, 6144 / D)));
  const size_t smem = sizeof(double) * static_cast<size_t>(D) * wpb;
  const int64_t want = (N + wpb - 1) / wpb;
  const int grid = static_cast<int>(std::min<int64_t>(want, int64_t(num_sms) * 16));
  if (f64)
    mass_map_kernel<double><<<grid, 32 * wpb, smem, s>>>(L, D, N, static_cast<double*>(S));
  else
    mass_map_kernel<float><<<grid, 32 * wpb, smem, s>>>(L, D, N, static_cast<float*>(S));
  return cudaGetLastError();
}

}  // namespace pmcmc
