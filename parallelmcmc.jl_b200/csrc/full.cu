// full.cu -- the dense-Jacobian (:full) Newton sweep and the adjoint pass for
// the Gaussian device targets.
//
// The reference rejects :full (DEER.jl:465-466, interface.jl:274-275).  Here
// it is Newton with the exact Jacobian of the surrogate step, the matrix whose
// action is the JVP of MALA.jl:768-795.  For a Gaussian with precision
// P = Q diag(lam) Q^T the Hessian is the constant -P, so with M = I - eps P
//     J_t = C_t + u_t v_t^T,   C_t = M (accepted) or I (rejected),
//     u_t = g(1-g) (y_t - x_t),  v_t = grad_x log alpha_t
//         = M g_y - g_x - P r + (eps/2) P^2 r,  r = x - y - eps g_y.
// MALA on N(mu, P^-1) is equivariant under x' = Q^T (x - mu), xi' = Q^T xi:
// in the eigenbasis the target is the diagonal Gaussian N(0, diag(1/lam)) and
//     J'_t = diag(c_t) + u'_t v'_t^T,   c_t = 1 - a_t eps lam.
// The Newton iterate is therefore carried in the eigenbasis (S', with the
// original-basis S kept alongside for the convergence test and the outputs),
// and the step is taken in update form (the same iterates in exact
// arithmetic as the reference's S-form B_t = f_t - J_t x_bar_t, DEER.jl:419):
//     delta'_t = J'_t delta'_{t-1} + (f'_t - S'_t),   S' += damping delta',
//     S += damping Q delta',
// so rounding in the chunk products slows convergence at worst and never
// moves the fixed point.  All sweep buffers use the stride DQ (16, 32, 64 or
// 128, zero-padded) so that the per-step loops have compile-time trip counts.
// Per solve, `rotate` forms xi' and x0'.  A sweep is four launches:
//   eval   one warp per column: the diagonal-target forward step in the
//          eigenbasis, u', v', r' = f'_t - S'_t and the accept flag
//   chunk  one CTA per chunk of L columns: the chunk's map [Phi'|beta'] as an
//          augmented DQ x (DQ+1) matrix in registers; four or eight lanes own a
//          column, whose recursion needs no barrier (column sums by shuffles)
//   carry  one CTA: updates entering each chunk, chunk maps streamed through
//          a cp.async ring
//   apply  one CTA per chunk: exact replay of the chunk from its entering
//          update (the old iterates arrive by cp.async meanwhile), the
//          rotation Q delta' as a warp-tiled product, damping, max|dS| and
//          max|S| in the original basis, and the convergence test +
//          CUDA-graph loop control in the last CTA.
//
// Adjoint (no counterpart in the reference): at a returned trajectory, with
// the accept decisions held fixed, f_t(x) = a_t y_t(x) + (1 - a_t) x has
// Jacobian C_t, so for an objective L(x_1..x_T) the adjoint is the diagonal
// (primed) reverse scan lambda'_t = c'_t + diag(c_{t+1}) lambda'_{t+1} and
//     dL/deps     = explicit + sum_t a_t lambda_t . (g(x_bar_t) + xi_t / sqrt(2 eps)),
//     dL/dlog s_i = sum_t a_t eps lam_i lambda'_{t,i} x_bar'_{t,i}     (s_i = 1 / lam_i).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "deer_column.cuh"
#include "deer_device.cuh"
#include "deer_launch.h"
#include "full.h"

namespace pmcmc {

namespace {

template <typename S>
__device__ __forceinline__ void load_struct(const S* g, S& s) {
  static_assert(sizeof(S) % 8 == 0, "struct size must be a multiple of 8 bytes");
  constexpr int n = sizeof(S) / 8;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    reinterpret_cast<unsigned long long*>(&s)[i] = reinterpret_cast<const unsigned long long*>(g)[i];
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// out = rows 4*lane .. 4*lane+3 of M v for one warp (M in shared memory in
// matvec4's layout, v a shared vector of D entries); zeros past Dp.
__device__ __forceinline__ void warp_rotate(const float* Ms, const float* v, int D, int Dp,
                                            float out[4]) {
  const int lane = threadIdx.x & 31;
  if (4 * lane < Dp) {
    matvec4<float, float, float>(Ms, v, D, Dp, lane, out);
  } else {
    out[0] = out[1] = out[2] = out[3] = 0.f;
  }
}

// Writes the warp's quad of v (masked to D) into a warp-private shared vector.
__device__ __forceinline__ void put_vec(float* vs, const float v[4], int D) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int e = 0; e < 4; ++e)
    if (4 * lane + e < D) vs[4 * lane + e] = v[e];
}

// Rotates a warp quad in place through the warp-private vector vw.
__device__ __forceinline__ void rotate_quad(const float* Qs, float* vw, int D, int Dp, float q[4]) {
  put_vec(vw, q, D);
  __syncwarp();
  warp_rotate(Qs, vw, D, Dp, q);
  __syncwarp();
}

// Warp-tiled product for up to 8 columns at once: acc[c][e] = sum_{k<K}
// Ms(4*lane+e, k) X[c*ldx + k] (Ms column-major at stride DQ, X columns in
// shared memory); each matrix element read serves 8 columns.  Lanes past DQ
// return zeros.
template <int DQ>
__device__ __forceinline__ void warp_tile8(const float* Ms, const float* X, int ldx, int nc, int K,
                                          float acc[8][4]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < 8; ++c)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[c][e] = 0.f;
  if (4 * lane >= DQ) return;
#pragma unroll 4
  for (int k = 0; k < K; ++k) {
    float q[4];
    load4(Ms + k * DQ + 4 * lane, q);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const float x = c < nc ? X[c * ldx + k] : 0.f;
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[c][e] = fmaf(q[e], x, acc[c][e]);
    }
  }
}

// Shared memory of the per-column kernels of the adjoint: the column plan
// (TT = 1), then Q (Dp x Dp, dense target) and kWarps warp-private vectors.
__host__ __device__ inline size_t eval_smem_bytes(int64_t Dp, bool dense) {
  const SmemPlan pl = plan_sweep_smem<float>(Dp, 1, dense);
  return pl.total + sizeof(float) * ((dense ? Dp * Dp : 0) + kWarps * Dp);
}

// Eager mode (no graph): sweeps launched after convergence, maxiter or an
// error are no-ops, like the fused sweep's.
__device__ __forceinline__ bool sweep_done(const DevState* st, int use_cond, int maxiter) {
  if (use_cond) return false;
  return *reinterpret_cast<const volatile int32_t*>(&st->converged) ||
         *reinterpret_cast<const volatile int32_t*>(&st->iter) >= maxiter ||
         *reinterpret_cast<const volatile int32_t*>(&st->status) != 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// rotate (once per solve): xi'_t = Q^T xi_t, x0' = Q^T (x0 - mu), at stride DQ
// ---------------------------------------------------------------------------
template <int DQ>
__global__ void __launch_bounds__(kThreads)
    full_rotate_kernel(const DevParams* __restrict__ Pg, const FullArgs* __restrict__ Fg,
                       DevState* __restrict__, cudaGraphConditionalHandle, int) {
  __shared__ DevParams P;
  __shared__ FullArgs F;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  load_struct(Fg, F);
  load_params(Pg, P);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  float* Qs = reinterpret_cast<float*>(smem_raw);  // Q^T operator at stride DQ
  float* Xw = Qs + DQ * DQ + warp * 8 * Dp;         // 8 staged columns per warp
  for (int i = threadIdx.x; i < DQ * DQ; i += blockDim.x) Qs[i] = F.QrmQ[i];
  __syncthreads();
  float* xi_e = const_cast<float*>(F.Pe->xi);
  if (blockIdx.x == 0 && warp == 0) {
    const float* x0 = static_cast<const float*>(P.x0);
    for (int i = lane; i < Dp; i += 32) Xw[i] = i < D ? static_cast<float>(x0[i] - P.mean_d[i]) : 0.f;
    __syncwarp();
    float acc[8][4];
    warp_tile8<DQ>(Qs, Xw, Dp, 1, D, acc);
    if (4 * lane < DQ) store4(static_cast<float*>(const_cast<void*>(F.Pe->x0)) + 4 * lane, acc[0]);
    __syncwarp();
  }
  const int64_t ntile = (P.T + 7) / 8;
  for (int64_t tile = static_cast<int64_t>(blockIdx.x) * kWarps + warp; tile < ntile;
       tile += static_cast<int64_t>(gridDim.x) * kWarps) {
    const int64_t t0 = tile * 8;
    const int nc = static_cast<int>(imin64(8, P.T - t0));
    for (int i = lane; i < nc * Dp; i += 32) Xw[i] = P.xi[t0 * Dp + i];
    __syncwarp();
    float acc[8][4];
    warp_tile8<DQ>(Qs, Xw, Dp, nc, D, acc);
    if (4 * lane < DQ)
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c < nc) store4(xi_e + (t0 + c) * DQ + 4 * lane, acc[c]);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// eval: per column forward step in the eigenbasis, u', v', r', accept flag
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads)
    full_eval_kernel(const DevParams* __restrict__, const FullArgs* __restrict__ Fg,
                     DevState* __restrict__ st, cudaGraphConditionalHandle, int use_cond) {
  __shared__ DevParams P;  // the eigenbasis view
  __shared__ FullArgs F;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  load_struct(Fg, F);
  __syncthreads();
  load_params(F.Pe, P);
  if (sweep_done(st, use_cond, P.maxiter)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  Smem<float> sm = carve<float>(smem_raw, P, 1, false);
  const float* Sold = static_cast<const float*>(P.S[st->cur]);
  const float* x0 = static_cast<const float*>(P.x0);
  // the first sweep starts from S = x0 broadcast (DEER.jl:538-542), read in place
  const bool first = st->iter == 0;
  const TapeKey key(P.seed, P.block);
  const float eps = static_cast<float>(P.eps);
  float lam[4] = {0.f, 0.f, 0.f, 0.f};
  if (4 * lane < D) load4(P.prec_f + 4 * lane, lam);
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kWarps + warp; t < P.T;
       t += static_cast<int64_t>(gridDim.x) * kWarps) {
    const float* xcol = (t == 0 || first) ? x0 : Sold + (t - 1) * Dp;
    Col<float, 1> c;
    column_forward<float, kDiagGauss, 1>(P, sm, key, xcol, static_cast<int>(t), c);
    const double logu = P.logu[t];
    const bool acc = logu < c.la;
    const float gp = sigmoid_slope<float>(c.la - logu);
    float s4[4] = {0.f, 0.f, 0.f, 0.f};
    if (4 * lane < D) load4(first ? x0 + 4 * lane : Sold + t * Dp + 4 * lane, s4);
    float v[4], u[4], r[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const bool in = 4 * lane + e < D;
      const float el = eps * lam[e];
      const float q = c.x[0][e] - c.y[0][e] - eps * c.gy[0][e];
      v[e] = in ? (1.f - el) * c.gy[0][e] - c.gx[0][e] - lam[e] * q * (1.f - 0.5f * el) : 0.f;
      u[e] = in ? gp * (c.y[0][e] - c.x[0][e]) : 0.f;
      r[e] = in ? (acc ? c.y[0][e] : c.x[0][e]) - s4[e] : 0.f;
    }
    if (4 * lane < Dp) {
      store4(F.U + t * Dp + 4 * lane, u);
      store4(F.V + t * Dp + 4 * lane, v);
      store4(F.R + t * Dp + 4 * lane, r);
    }
    if (lane == 0) F.acc[t] = acc ? 1 : 0;
  }
}

// ---------------------------------------------------------------------------
// chunk: the augmented map [Phi' | beta'] of each chunk.  TPC consecutive
// lanes own column j (j == DQ is beta'), lane q of them rows [q*NR, (q+1)*NR)
// in registers (NR = DQ / TPC).  Per step: w_j = v'^T [Phi'|beta']_{:,j}
// (log2 TPC shuffles), then
// [Phi'|beta'] <- diag(c_t) [Phi'|beta'] + u' w^T + r' e_DQ^T.
// Padded rows and columns stay zero.
// ---------------------------------------------------------------------------
template <int NR, int TPC>
__global__ void __launch_bounds__(544)
    full_chunk_kernel(const DevParams* __restrict__, const FullArgs* __restrict__ Fg,
                      DevState* __restrict__ st, cudaGraphConditionalHandle, int use_cond) {
  constexpr int DQ = TPC * NR;
  static_assert(NR % 4 == 0 && (TPC == 4 || TPC == 8), "chunk tiling");
  __shared__ DevParams P;
  __shared__ FullArgs F;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  load_struct(Fg, F);
  __syncthreads();
  load_params(F.Pe, P);
  if (sweep_done(st, use_cond, P.maxiter)) return;
  const int tid = threadIdx.x;
  const int D = static_cast<int>(P.D);
  const int L = F.L;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * L;
  const int nt = static_cast<int>(imin64(L, P.T - t0));
  float* Us = reinterpret_cast<float*>(smem_raw);
  float* Vs = Us + L * DQ;
  float* Rs = Vs + L * DQ;
  uint8_t* as = reinterpret_cast<uint8_t*>(Rs + L * DQ);
  {
    const int n4 = nt * DQ / 4;
    const float4* gu = reinterpret_cast<const float4*>(F.U + t0 * DQ);
    const float4* gv = reinterpret_cast<const float4*>(F.V + t0 * DQ);
    const float4* gr = reinterpret_cast<const float4*>(F.R + t0 * DQ);
    for (int i = tid; i < n4; i += blockDim.x) {
      reinterpret_cast<float4*>(Us)[i] = gu[i];
      reinterpret_cast<float4*>(Vs)[i] = gv[i];
      reinterpret_cast<float4*>(Rs)[i] = gr[i];
    }
    for (int i = tid; i < nt; i += blockDim.x) as[i] = F.acc[t0 + i];
  }
  const int j = tid / TPC, q = tid % TPC;
  const bool active = j <= DQ;
  const bool bcol = j == DQ;
  const int r0 = q * NR;
  const float eps = static_cast<float>(P.eps);
  float phi[NR], ml[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const int i = r0 + k;
    phi[k] = (active && i == j && i < D) ? 1.f : 0.f;
    ml[k] = i < D ? 1.f - eps * F.lamQ[i] : 0.f;
  }
  __syncthreads();
  for (int s = 0; s < nt; ++s) {
    const float4* v4 = reinterpret_cast<const float4*>(Vs + s * DQ + r0);
    const float4* u4 = reinterpret_cast<const float4*>(Us + s * DQ + r0);
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
    for (int k = 0; k < NR / 4; ++k) {
      const float4 v = v4[k];
      a0 = fmaf(v.x, phi[4 * k], a0);
      a1 = fmaf(v.y, phi[4 * k + 1], a1);
      a2 = fmaf(v.z, phi[4 * k + 2], a2);
      a3 = fmaf(v.w, phi[4 * k + 3], a3);
    }
    float w = (a0 + a1) + (a2 + a3);
    w += __shfl_xor_sync(0xffffffffu, w, 1);
    w += __shfl_xor_sync(0xffffffffu, w, 2);
    if (TPC == 8) w += __shfl_xor_sync(0xffffffffu, w, 4);
    if (as[s]) {  // uniform across the CTA
#pragma unroll
      for (int k = 0; k < NR / 4; ++k) {
        const float4 u = u4[k];
        phi[4 * k] = fmaf(u.x, w, ml[4 * k] * phi[4 * k]);
        phi[4 * k + 1] = fmaf(u.y, w, ml[4 * k + 1] * phi[4 * k + 1]);
        phi[4 * k + 2] = fmaf(u.z, w, ml[4 * k + 2] * phi[4 * k + 2]);
        phi[4 * k + 3] = fmaf(u.w, w, ml[4 * k + 3] * phi[4 * k + 3]);
      }
    } else {
#pragma unroll
      for (int k = 0; k < NR / 4; ++k) {
        const float4 u = u4[k];
        phi[4 * k] = fmaf(u.x, w, phi[4 * k]);
        phi[4 * k + 1] = fmaf(u.y, w, phi[4 * k + 1]);
        phi[4 * k + 2] = fmaf(u.z, w, phi[4 * k + 2]);
        phi[4 * k + 3] = fmaf(u.w, w, phi[4 * k + 3]);
      }
    }
    if (bcol) {
      const float4* r4 = reinterpret_cast<const float4*>(Rs + s * DQ + r0);
#pragma unroll
      for (int k = 0; k < NR / 4; ++k) {
        const float4 r = r4[k];
        phi[4 * k] += r.x;
        phi[4 * k + 1] += r.y;
        phi[4 * k + 2] += r.z;
        phi[4 * k + 3] += r.w;
      }
    }
  }
  if (active) {
    float* dst = bcol ? F.beta + static_cast<size_t>(blockIdx.x) * DQ + r0
                      : F.Phi + (static_cast<size_t>(blockIdx.x) * DQ + j) * DQ + r0;  // column-major
#pragma unroll
    for (int k = 0; k < NR / 4; ++k)
      reinterpret_cast<float4*>(dst)[k] =
          make_float4(phi[4 * k], phi[4 * k + 1], phi[4 * k + 2], phi[4 * k + 3]);
  }
}

// ---------------------------------------------------------------------------
// carry: din_0 = 0, din_{c+1} = Phi'_c din_c + beta'_c (one CTA).  Thread
// (part, row) sums KC terms of row `row` (the map is column-major, so the
// threads of a part read consecutive rows: coalesced), partial sums combined
// through shared memory.  Each thread keeps its KC map entries for the next
// two chunks in registers, loaded from L2 two steps ahead (a three-slot ring),
// so a step waits on no copy.
// ---------------------------------------------------------------------------
template <int DQ, int NST>
__global__ void __launch_bounds__(256)
    full_carry_kernel(const DevParams* __restrict__, const FullArgs* __restrict__ Fg,
                      DevState* __restrict__ st, cudaGraphConditionalHandle, int use_cond) {
  constexpr int PARTS = DQ >= 128 ? 2 : 4;
  constexpr int KC = DQ / PARTS;
  static_assert(PARTS * DQ <= 256, "one thread a (part, row)");
  __shared__ DevParams P;
  __shared__ FullArgs F;
  __shared__ float vec[2][DQ];
  __shared__ float pbuf[PARTS][DQ];
  load_struct(Fg, F);
  __syncthreads();
  load_params(F.Pe, P);
  if (sweep_done(st, use_cond, P.maxiter)) return;
  const int tid = threadIdx.x;
  const int nch = F.nchunks;
  const int row = tid % DQ, part = tid / DQ;
  const bool worker = part < PARTS;
  const int k0 = part * KC;
  for (int i = tid; i < 2 * DQ; i += blockDim.x) (&vec[0][0])[i] = 0.f;
  for (int i = tid; i < DQ; i += blockDim.x) F.din[i] = 0.f;
  float m[3][KC];
  float bt[3] = {0.f, 0.f, 0.f};
  auto fetch = [&](int c, float (&dst)[KC], float& b) {
    if (c < nch - 1) {
      if (worker) {
        const float* Ph = F.Phi + static_cast<size_t>(c) * DQ * DQ + static_cast<size_t>(k0) * DQ + row;
#pragma unroll
        for (int k = 0; k < KC; ++k) dst[k] = __ldcg(Ph + static_cast<size_t>(k) * DQ);
      }
      if (tid < DQ) b = __ldcg(F.beta + static_cast<size_t>(c) * DQ + tid);
    }
  };
  auto step = [&](int c, const float (&cur)[KC], float b) {
    if (worker) {
      const float* x = vec[c & 1] + k0;
      float a0 = 0.f, a1 = 0.f;
#pragma unroll
      for (int k = 0; k < KC; k += 2) {
        a0 = fmaf(cur[k], x[k], a0);
        a1 = fmaf(cur[k + 1], x[k + 1], a1);
      }
      pbuf[part][row] = a0 + a1;
    }
    __syncthreads();
    if (tid < DQ) {
      float y = b;
#pragma unroll
      for (int p = 0; p < PARTS; ++p) y += pbuf[p][tid];
      vec[(c + 1) & 1][tid] = y;
      F.din[static_cast<size_t>(c + 1) * DQ + tid] = y;
    }
    __syncthreads();
  };
  __syncthreads();
  fetch(0, m[0], bt[0]);
  fetch(1, m[1], bt[1]);
  for (int c = 0; c < nch - 1; c += 3) {
    fetch(c + 2, m[2], bt[2]);
    step(c, m[0], bt[0]);
    if (c + 1 >= nch - 1) break;
    fetch(c + 3, m[0], bt[0]);
    step(c + 1, m[1], bt[1]);
    if (c + 2 >= nch - 1) break;
    fetch(c + 4, m[1], bt[1]);
    step(c + 2, m[2], bt[2]);
  }
}

// ---------------------------------------------------------------------------
// apply: replay each chunk from its entering update (warp 0) while the
// cp.async copies of the old iterates land, rotate back (warp-tiled
// Q delta'), damp both iterates, reduce the convergence metric in the
// original basis and run the convergence test in the last CTA.
// ---------------------------------------------------------------------------
template <int DQ>
__global__ void __launch_bounds__(kThreads)
    full_apply_kernel(const DevParams* __restrict__ Pg, const FullArgs* __restrict__ Fg,
                      DevState* __restrict__ st, cudaGraphConditionalHandle cond, int use_cond) {
  __shared__ DevParams P;   // original basis
  __shared__ DevParams Pe;  // eigenbasis
  __shared__ FullArgs F;
  __shared__ double r_dm[kWarps], r_sm[kWarps];
  __shared__ int s_bad, s_last;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  load_struct(Fg, F);
  load_struct(Pg, P);
  __syncthreads();
  load_params(F.Pe, Pe);
  if (sweep_done(st, use_cond, P.maxiter)) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  const int L = F.L;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * L;
  const int nt = static_cast<int>(imin64(L, P.T - t0));
  float* Us = reinterpret_cast<float*>(smem_raw);
  float* Vs = Us + L * DQ;
  float* Rs = Vs + L * DQ;
  float* Qs = Rs + L * DQ;   // DQ x DQ, Q column-major
  float* Eo = Qs + DQ * DQ;  // L x DQ old eigenbasis iterate
  float* So = Eo + L * DQ;   // L x Dp old iterate
  uint8_t* as = reinterpret_cast<uint8_t*>(So + L * Dp);
  const int cur = st->cur;
  const bool first = st->iter == 0;
  {
    const int n4 = nt * DQ / 4;
    const float* gu = F.U + t0 * DQ;
    const float* gv = F.V + t0 * DQ;
    const float* gr = F.R + t0 * DQ;
    for (int i = tid; i < n4; i += blockDim.x) {
      cp_async16(Us + 4 * i, gu + 4 * i);
      cp_async16(Vs + 4 * i, gv + 4 * i);
      cp_async16(Rs + 4 * i, gr + 4 * i);
    }
    for (int i = tid; i < DQ * DQ / 4; i += blockDim.x) cp_async16(Qs + 4 * i, F.QcmQ + 4 * i);
    cp_async_commit();
    if (!first) {
      const float* go = static_cast<const float*>(P.S[cur]) + t0 * Dp;
      const float* ge = static_cast<const float*>(Pe.S[cur]) + t0 * DQ;
      for (int i = tid; i < nt * Dp / 4; i += blockDim.x) cp_async16(So + 4 * i, go + 4 * i);
      for (int i = tid; i < n4; i += blockDim.x) cp_async16(Eo + 4 * i, ge + 4 * i);
    }
    cp_async_commit();
    for (int i = tid; i < nt; i += blockDim.x) as[i] = F.acc[t0 + i];
    if (tid == 0) s_bad = 0;
  }
  cp_async_wait<1>();
  __syncthreads();
  if (warp == 0) {
    // lanes past DQ carry zeros through the warp reduction
    const bool in = 4 * lane < DQ;
    const float eps = static_cast<float>(P.eps);
    float d[4] = {0.f, 0.f, 0.f, 0.f}, lc[4] = {0.f, 0.f, 0.f, 0.f};
    if (in) {
      load4(F.din + static_cast<size_t>(blockIdx.x) * DQ + 4 * lane, d);
      float l4[4];
      load4(F.lamQ + 4 * lane, l4);
#pragma unroll
      for (int e = 0; e < 4; ++e) lc[e] = 4 * lane + e < D ? 1.f - eps * l4[e] : 0.f;
    }
    // step s's u', v', r' and accept flag are loaded during step s - 1
    float u[4] = {0.f, 0.f, 0.f, 0.f}, v[4] = {0.f, 0.f, 0.f, 0.f}, r[4] = {0.f, 0.f, 0.f, 0.f};
    bool a = false;
    if (nt > 0) {
      if (in) {
        load4(Us + 4 * lane, u);
        load4(Vs + 4 * lane, v);
        load4(Rs + 4 * lane, r);
      }
      a = as[0] != 0;
    }
    for (int s = 0; s < nt; ++s) {
      float un[4] = {0.f, 0.f, 0.f, 0.f}, vn[4] = {0.f, 0.f, 0.f, 0.f}, rn[4] = {0.f, 0.f, 0.f, 0.f};
      bool an = false;
      if (s + 1 < nt) {
        if (in) {
          load4(Us + (s + 1) * DQ + 4 * lane, un);
          load4(Vs + (s + 1) * DQ + 4 * lane, vn);
          load4(Rs + (s + 1) * DQ + 4 * lane, rn);
        }
        an = as[s + 1] != 0;
      }
      const float dot = warp_sum((v[0] * d[0] + v[1] * d[1]) + (v[2] * d[2] + v[3] * d[3]));
#pragma unroll
      for (int e = 0; e < 4; ++e) d[e] = fmaf(u[e], dot, (a ? lc[e] : 1.f) * d[e]) + r[e];
      if (in) store4(Rs + s * DQ + 4 * lane, d);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        u[e] = un[e];
        v[e] = vn[e];
        r[e] = rn[e];
      }
      a = an;
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  float* Snew = static_cast<float*>(P.S[cur ^ 1]);
  float* Enew = static_cast<float*>(Pe.S[cur ^ 1]);
  const float* x0 = static_cast<const float*>(P.x0);
  const float* x0e = static_cast<const float*>(Pe.x0);
  const float dmp = static_cast<float>(P.damping);
  float dm = 0.f, smx = 0.f;  // maxima are exact in FP32
  bool bad = false;
  for (int tile = warp; 8 * tile < nt; tile += kWarps) {
    const int c0 = 8 * tile;
    const int nc = min(8, nt - c0);
    float acc[8][4];
    warp_tile8<DQ>(Qs, Rs + c0 * DQ, DQ, nc, DQ, acc);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (c >= nc) break;
      const int64_t t = t0 + c0 + c;
      if (4 * lane < D) {
        float o[4], n[4];
        load4(first ? x0 + 4 * lane : So + (c0 + c) * Dp + 4 * lane, o);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          if (4 * lane + e < D) {
            n[e] = fmaf(dmp, acc[c][e], o[e]);
            dm = fmaxf(dm, fabsf(n[e] - o[e]));
            smx = fmaxf(smx, fabsf(n[e]));
            bad |= !isfinite(n[e]);
          } else {
            n[e] = 0.f;
          }
        }
        store4(Snew + t * Dp + 4 * lane, n);
      }
      if (4 * lane < DQ) {
        float de[4], eo[4], en[4];
        load4(Rs + (c0 + c) * DQ + 4 * lane, de);
        load4(first ? x0e + 4 * lane : Eo + (c0 + c) * DQ + 4 * lane, eo);
#pragma unroll
        for (int e = 0; e < 4; ++e) en[e] = fmaf(dmp, de[e], eo[e]);
        store4(Enew + t * DQ + 4 * lane, en);
      }
    }
  }
  dm = warp_max(dm);
  smx = warp_max(smx);
  bad = __any_sync(0xffffffffu, bad);
  if (lane == 0) {
    r_dm[warp] = static_cast<double>(dm);
    r_sm[warp] = static_cast<double>(smx);
    if (bad) s_bad = 1;
  }
  __syncthreads();
  if (tid == 0) {
    // this CTA's maxima into its own slot (no contended atomics)
    for (int w = 1; w < kWarps; ++w) {
      r_dm[0] = fmax(r_dm[0], r_dm[w]);
      r_sm[0] = fmax(r_sm[0], r_sm[w]);
    }
    F.part[2 * blockIdx.x] = r_dm[0];
    F.part[2 * blockIdx.x + 1] = r_sm[0];
    if (s_bad) atomicCAS(&st->status, 0, static_cast<int>(kStNonfinite));
    __threadfence();
    const unsigned prev = atomicAdd(&st->done_counter, 1u);
    s_last = prev == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  // last CTA: reduce every CTA's slot, the convergence test (DEER.jl:567-578)
  // and loop control
  __threadfence();
  double pd = 0.0, ps = 0.0;
  for (int i = tid; i < static_cast<int>(gridDim.x); i += blockDim.x) {
    pd = fmax(pd, __ldcg(F.part + 2 * i));
    ps = fmax(ps, __ldcg(F.part + 2 * i + 1));
  }
  pd = warp_max(pd);
  ps = warp_max(ps);
  __syncthreads();
  if (lane == 0) {
    r_dm[warp] = pd;
    r_sm[warp] = ps;
  }
  __syncthreads();
  if (tid != 0) return;
  double dmax = 0.0, smax = 0.0;
  for (int w = 0; w < kWarps; ++w) dmax = fmax(dmax, r_dm[w]), smax = fmax(smax, r_sm[w]);
  const double metric = dmax / (P.tol_abs + P.tol_rel * smax);
  const int status = atomicAdd(&st->status, 0);
  const int iter = st->iter;
  const int converged = metric <= 1.0;
  st->metric = metric;
  st->iter = iter + 1;
  st->cur = cur ^ 1;
  st->converged = converged;
  st->done_counter = 0;
  st->dmax_bits = 0;
  st->smax_bits = 0;
  __threadfence();
  const bool more = !converged && (iter + 1 < P.maxiter) && status == 0;
  if (use_cond) cudaGraphSetConditional(cond, more ? 1u : 0u);
}

// ---------------------------------------------------------------------------
// Adjoint kernels
// ---------------------------------------------------------------------------

// Per column t: accept flag of the returned trajectory, the reversed-scan
// multiplier Arev[T - t] = c_t (primed, diagonal) and the objective terms in
// reversed order.  Objective 1: c_t = 2 S_t / T.  Objective 0 (ESJD,
// Rao-Blackwellised): L = (1/T) sum_t alpha_t e_t, e_t = |y_t - x_bar_t|^2,
// alpha_t = min(1, exp(log alpha_t)); term t contributes
//   dL_t/dx_bar_t = (1/T)[alpha' e_t v_t + alpha_t 2 eps H (y_t - x_bar_t)]   to c_{t-1}
//   (1/T)[alpha' e_t dla/deps + alpha_t de_t/deps]                          to the explicit eps term
// with alpha' = d alpha / d log alpha and H = -P.
template <int TK>
__global__ void __launch_bounds__(kThreads)
    adjoint_terms_kernel(const DevParams* __restrict__ Pg, const FullArgs* __restrict__ Fg,
                         int objective, const float* __restrict__ S, float* __restrict__ Brev,
                         float* __restrict__ Arev, double* __restrict__ direct) {
  __shared__ DevParams P;
  __shared__ FullArgs F;
  __shared__ double r_dir[kWarps];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  load_struct(Fg, F);
  load_params(Pg, P);
  constexpr bool dense = TK == kDenseGauss;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  const int64_t T = P.T;
  Smem<float> sm = carve<float>(smem_raw, P, 1, dense);
  float* Qs = reinterpret_cast<float*>(smem_raw + plan_sweep_smem<float>(Dp, 1, dense).total);
  float* vw = Qs + (dense ? Dp * Dp : 0) + warp * Dp;
  if (dense)
    for (int i = threadIdx.x; i < Dp * Dp; i += blockDim.x) Qs[i] = F.Qrm[i];
  for (int i = lane; i < Dp; i += 32) vw[i] = 0.f;
  __syncthreads();
  const float* x0 = static_cast<const float*>(P.x0);
  const TapeKey key(P.seed, P.block);
  const float eps = static_cast<float>(P.eps);
  const double epsd = P.eps;
  const double invT = 1.0 / static_cast<double>(T);
  float lamq[4] = {0.f, 0.f, 0.f, 0.f};
  if (4 * lane < D) load4(F.lam + 4 * lane, lamq);
  double dir = 0.0;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kWarps + warp; t < T;
       t += static_cast<int64_t>(gridDim.x) * kWarps) {
    const float* xcol = t == 0 ? x0 : S + (t - 1) * Dp;
    Col<float, 1> c;
    column_forward<float, TK, 1>(P, sm, key, xcol, static_cast<int>(t), c);
    const double logu = P.logu[t];
    const bool acc = logu < c.la;
    if (lane == 0) F.acc[t] = acc ? 1 : 0;
    if (4 * lane < Dp) {
      float m[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) m[e] = t == 0 ? 1.f : (acc ? 1.f - eps * lamq[e] : 1.f);
      // C_t links lambda_{t-1} (reversed index T - t) to lambda_t; index 0 has no predecessor
      store4(Arev + (t == 0 ? 0 : T - t) * Dp + 4 * lane, m);
    }
    float cvec[4] = {0.f, 0.f, 0.f, 0.f};
    int64_t dst = -1;
    if (objective == 1) {
      if (4 * lane < D) {
        float s4[4];
        load4(S + t * Dp + 4 * lane, s4);
#pragma unroll
        for (int e = 0; e < 4; ++e)
          cvec[e] = 4 * lane + e < D ? static_cast<float>(2.0 * invT * s4[e]) : 0.f;
      }
      dst = T - 1 - t;
    } else {
      const double la = c.la;
      const double alpha = la < 0.0 ? exp(la) : 1.0;
      const double dalpha = la < 0.0 ? alpha : 0.0;
      const float inv_s2e = static_cast<float>(1.0 / P.sqrt2eps);
      float dyx[1][4], dy[1][4], q[1][4], npdy[1][4], npdyx[1][4], v[4];
      double e2 = 0.0, dede = 0.0, qq = 0.0;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const bool in = 4 * lane + e < D;
        dyx[0][e] = in ? c.y[0][e] - c.x[0][e] : 0.f;              // y - x
        dy[0][e] = in ? c.gx[0][e] + c.xi[0][e] * inv_s2e : 0.f;  // dy/deps
        q[0][e] = in ? c.x[0][e] - c.y[0][e] - eps * c.gy[0][e] : 0.f;
        e2 += static_cast<double>(dyx[0][e]) * dyx[0][e];
        dede += 2.0 * static_cast<double>(dyx[0][e]) * dy[0][e];
        qq += static_cast<double>(q[0][e]) * q[0][e];
      }
      if constexpr (dense) {
        float pgy[1][4], pr[1][4], ppr[1][4];
        dense_neg_pv<float, 1>(P, sm, dy, npdy);    // -P dy
        dense_neg_pv<float, 1>(P, sm, dyx, npdyx);  // -P (y - x)
        dense_neg_pv<float, 1>(P, sm, c.gy, pgy);
        dense_neg_pv<float, 1>(P, sm, q, pr);
        dense_neg_pv<float, 1>(P, sm, pr, ppr);
#pragma unroll
        for (int e = 0; e < 4; ++e)
          v[e] = c.gy[0][e] + eps * pgy[0][e] - c.gx[0][e] + pr[0][e] + 0.5f * eps * ppr[0][e];
      } else {
        float lam[4] = {0.f, 0.f, 0.f, 0.f};
        if (4 * lane < D) load4(P.prec_f + 4 * lane, lam);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float el = eps * lam[e];
          npdy[0][e] = -lam[e] * dy[0][e];
          npdyx[0][e] = -lam[e] * dyx[0][e];
          v[e] = (1.f - el) * c.gy[0][e] - c.gx[0][e] - lam[e] * q[0][e] * (1.f - 0.5f * el);
        }
      }
      // dla/deps = g_y.dy - q.dq/(2 eps) + |q|^2/(4 eps^2),  dq = -(dy - eps P dy) - g_y
      double dla = 0.0;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (4 * lane + e >= D) continue;
        const double dq = -(static_cast<double>(dy[0][e]) + epsd * npdy[0][e]) - c.gy[0][e];
        dla += static_cast<double>(c.gy[0][e]) * dy[0][e] -
               static_cast<double>(q[0][e]) * dq / (2 * epsd);
      }
      dla = warp_sum(dla) + warp_sum(qq) / (4 * epsd * epsd);
      e2 = warp_sum(e2);
      dede = warp_sum(dede);
      if (lane == 0) dir += invT * (dalpha * dla * e2 + alpha * dede);
#pragma unroll
      for (int e = 0; e < 4; ++e)
        cvec[e] = 4 * lane + e < D ? static_cast<float>(invT * (dalpha * e2 * v[e] +
                                                                alpha * 2.0 * epsd * npdyx[0][e]))
                                   : 0.f;
      dst = t >= 1 ? T - t : -1;  // c_{t-1} sits at reversed index T - 1 - (t - 1)
      if (t == 0 && 4 * lane < Dp) {
        const float z[4] = {0.f, 0.f, 0.f, 0.f};
        store4(Brev + 4 * lane, z);  // c_{T-1} = 0: the last state enters no term
      }
    }
    if (dense) rotate_quad(Qs, vw, D, Dp, cvec);
    if (dst >= 0 && 4 * lane < Dp) store4(Brev + dst * Dp + 4 * lane, cvec);
  }
  if (lane == 0) r_dir[warp] = dir;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kWarps; ++w) s += r_dir[w];
    if (s != 0.0) atomicAdd(direct, s);
  }
}

// dL/deps and dL/dlog s from the reversed primed adjoint Lrev.
template <int TK>
__global__ void __launch_bounds__(kThreads)
    adjoint_reduce_kernel(const DevParams* __restrict__ Pg, const FullArgs* __restrict__ Fg,
                          int objective, const float* __restrict__ S,
                          const float* __restrict__ Lrev, double* __restrict__ out) {
  __shared__ DevParams P;
  __shared__ FullArgs F;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  load_struct(Fg, F);
  load_params(Pg, P);
  constexpr bool dense = TK == kDenseGauss;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int D = static_cast<int>(P.D), Dp = static_cast<int>(P.Dp);
  const int64_t T = P.T;
  double* red = reinterpret_cast<double*>(smem_raw);  // kWarps x (Dp + 1)
  float* Qs = reinterpret_cast<float*>(red + kWarps * (Dp + 1));
  float* vw = Qs + (dense ? Dp * Dp : 0) + warp * Dp;
  if (dense)
    for (int i = threadIdx.x; i < Dp * Dp; i += blockDim.x) Qs[i] = F.Qrm[i];
  for (int i = lane; i < Dp; i += 32) vw[i] = 0.f;
  __syncthreads();
  const float* x0 = static_cast<const float*>(P.x0);
  const double inv_s2e = 1.0 / P.sqrt2eps;
  float lamq[4] = {0.f, 0.f, 0.f, 0.f};
  if (4 * lane < D) load4(F.lam + 4 * lane, lamq);
  double ge = 0.0, gs[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kWarps + warp; t < T;
       t += static_cast<int64_t>(gridDim.x) * kWarps) {
    if (!F.acc[t]) continue;  // warp-uniform
    const float* xcol = t == 0 ? x0 : S + (t - 1) * Dp;
    float xm[4] = {0.f, 0.f, 0.f, 0.f}, xi[4] = {0.f, 0.f, 0.f, 0.f};
    if (4 * lane < D) {
      load4(xcol + 4 * lane, xm);
      load4(P.xi + t * Dp + 4 * lane, xi);
#pragma unroll
      for (int e = 0; e < 4; ++e)
        xm[e] = 4 * lane + e < D ? static_cast<float>(xm[e] - P.mean_d[4 * lane + e]) : 0.f;
    }
    if (dense) {
      rotate_quad(Qs, vw, D, Dp, xm);
      rotate_quad(Qs, vw, D, Dp, xi);
    }
    float lm[4] = {0.f, 0.f, 0.f, 0.f};
    if (4 * lane < Dp) load4(Lrev + (T - 1 - t) * Dp + 4 * lane, lm);
    double g = 0.0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (4 * lane + e >= D) continue;
      g += static_cast<double>(lm[e]) *
           (-static_cast<double>(lamq[e]) * xm[e] + static_cast<double>(xi[e]) * inv_s2e);
      if (objective == 1) gs[e] += P.eps * static_cast<double>(lamq[e]) * lm[e] * xm[e];
    }
    ge += warp_sum(g);
  }
  if (4 * lane < Dp)
#pragma unroll
    for (int e = 0; e < 4; ++e) red[warp * (Dp + 1) + 4 * lane + e] = gs[e];
  if (lane == 0) red[warp * (Dp + 1) + Dp] = ge;
  __syncthreads();
  for (int i = threadIdx.x; i <= Dp; i += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < kWarps; ++w) s += red[w * (Dp + 1) + i];
    if (s != 0.0) {
      if (i == Dp) atomicAdd(out, s);
      else if (i < D) atomicAdd(out + 1 + i, s);
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

size_t chunk_smem(int Dq, int L) { return sizeof(float) * 3 * static_cast<size_t>(L) * Dq + L + 16; }
size_t apply_smem(int Dq, int64_t Dp, int L) {
  return sizeof(float) * (4 * static_cast<size_t>(L) * Dq + static_cast<size_t>(Dq) * Dq + L * Dp) +
         L + 16;
}
int carry_stages(int Dq) { return Dq <= 64 ? 8 : 2; }

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// lanes per column of the chunk kernel: 8 where NR stays a multiple of 4 and
// the CTA within 544 threads
constexpr int chunk_tpc(int DQ) { return (DQ == 32 || DQ == 64) ? 8 : 4; }

template <int DQ>
void pick_kernels(FullPlan* fp) {
  constexpr int NST = DQ <= 64 ? 8 : 2;
  constexpr int TPC = chunk_tpc(DQ);
  fp->chunk = reinterpret_cast<const void*>(&full_chunk_kernel<DQ / TPC, TPC>);
  fp->carry = reinterpret_cast<const void*>(&full_carry_kernel<DQ, NST>);
  fp->apply = reinterpret_cast<const void*>(&full_apply_kernel<DQ>);
  fp->rotate = reinterpret_cast<const void*>(&full_rotate_kernel<DQ>);
}

}  // namespace

int full_stride(int64_t Dp) {
  for (int q = 16; q <= 128; q <<= 1)
    if (Dp <= q) return q;
  return 0;
}

bool full_plan(int64_t Dp, int64_t T, int tkind, int num_sms, int chunks_override, FullPlan* fp) {
  (void)tkind;
  const int Dq = full_stride(Dp);
  if (Dq == 0 || T < 1) return false;
  fp->Dq = Dq;
  const size_t budget = 200 * 1024;
  int Lmax = 1;
  while (Lmax < 4096 && chunk_smem(Dq, Lmax + 1) <= budget && apply_smem(Dq, Dp, Lmax + 1) <= budget)
    ++Lmax;
  // the sequential depth of a sweep is ~L chunk steps + L replay steps +
  // nchunks carry steps, a carry step about a quarter of the cost of the other
  // two together: about sqrt(2 T) chunks balances them (128 at T = 8192:
  // 121 us a sweep against 139 us at 64 chunks, D = 64)
  int nch = chunks_override > 0
                ? chunks_override
                : std::min(num_sms, static_cast<int>(std::sqrt(2.0 * static_cast<double>(T)) + 0.5));
  nch = std::max(1, nch);
  int64_t L = (T + nch - 1) / nch;
  if (L > Lmax) L = Lmax;
  fp->L = static_cast<int>(L);
  fp->nchunks = static_cast<int>((T + L - 1) / L);
  fp->smem_chunk = chunk_smem(Dq, fp->L);
  fp->smem_apply = apply_smem(Dq, Dp, fp->L);
  const int nst = carry_stages(Dq);
  const int parts = Dq >= 128 ? 2 : 4;
  fp->smem_carry = 0;  // static shared memory only
  (void)nst;
  (void)parts;
  fp->smem_eval = plan_sweep_smem<float>(Dq, 1, false).total;
  fp->eval_grid =
      static_cast<int>(std::min<int64_t>((T + kWarps - 1) / kWarps, int64_t(num_sms) * 4));
  fp->threads_chunk = ((chunk_tpc(Dq) * (Dq + 1) + 31) / 32) * 32;
  fp->eval = reinterpret_cast<const void*>(&full_eval_kernel);
  switch (Dq) {
    case 16: pick_kernels<16>(fp); break;
    case 32: pick_kernels<32>(fp); break;
    case 64: pick_kernels<64>(fp); break;
    default: pick_kernels<128>(fp); break;
  }
  fp->smem_rotate = sizeof(float) * (static_cast<size_t>(Dq) * Dq + kWarps * 8 * Dp);
  fp->rotate_grid = static_cast<int>(
      std::max<int64_t>(1, std::min<int64_t>((T + 8 * kWarps - 1) / (8 * kWarps), num_sms)));
  return true;
}

cudaError_t full_sweep(cudaStream_t s, const FullPlan& fp, const DevParams* Pg, const FullArgs* Fg,
                       DevState* st, cudaGraphConditionalHandle cond, int use_cond) {
  void* args[] = {const_cast<DevParams**>(&Pg), const_cast<FullArgs**>(&Fg), &st, &cond,
                  &use_cond};
  const void* fns[4] = {fp.eval, fp.chunk, fp.carry, fp.apply};
  const size_t sm[4] = {fp.smem_eval, fp.smem_chunk, fp.smem_carry, fp.smem_apply};
  const int grid[4] = {fp.eval_grid, fp.nchunks, 1, fp.nchunks};
  const int thr[4] = {kThreads, fp.threads_chunk, 256, kThreads};
  for (int i = 0; i < 4; ++i) {
    const cudaError_t e = cudaLaunchKernel(fns[i], dim3(grid[i]), dim3(thr[i]), args, sm[i], s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// scratch: counter (256 B) | zero vector | flags | agg_a | agg_b | incl
size_t full_adjoint_scratch_bytes(int64_t Dp, int64_t T) {
  const int TT = scan_tile_cols(Dp, T);
  const int64_t nt = (T + TT - 1) / TT;
  return 256 + al256(4 * Dp) + al256(4 * static_cast<size_t>(nt)) + 3 * al256(4 * nt * Dp);
}

cudaError_t full_adjoint(cudaStream_t s, const DevParams* Pg, const FullArgs* Fg,
                         const FullArgs& Fh, int64_t D, int64_t Dp, int64_t T, int tkind,
                         int num_sms, int objective, const float* S, double* out, void* scratch,
                         uint32_t epoch) {
  const bool dense = tkind == kDenseGauss;
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * (1 + D), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(Fh.direct, 0, sizeof(double), s);
  if (e != cudaSuccess) return e;
  const int grid =
      static_cast<int>(std::min<int64_t>((T + kWarps - 1) / kWarps, int64_t(num_sms) * 2));
  const size_t st = eval_smem_bytes(Dp, dense);
  const void* tk = dense ? reinterpret_cast<const void*>(&adjoint_terms_kernel<kDenseGauss>)
                         : reinterpret_cast<const void*>(&adjoint_terms_kernel<kDiagGauss>);
  if (st > 0) {
    e = raise_smem_limit(reinterpret_cast<const void*>(tk), st);
    if (e != cudaSuccess) return e;
  }
  float* Brev = Fh.cterm;
  float* Arev = Fh.arev;
  double* dir = Fh.direct;
  void* targs[] = {const_cast<DevParams**>(&Pg), const_cast<FullArgs**>(&Fg), &objective,
                   const_cast<float**>(&S), &Brev, &Arev, &dir};
  e = cudaLaunchKernel(tk, dim3(grid), dim3(kThreads), targs, st, s);
  if (e != cudaSuccess) return e;
  // reverse scan in reversed time: Lrev_tau = Arev_tau * Lrev_{tau-1} + Brev_tau, Lrev_{-1} = 0
  unsigned char* w = static_cast<unsigned char*>(scratch);
  const int TT = scan_tile_cols(Dp, T);
  const int64_t ntl = (T + TT - 1) / TT;
  ScanScratch scr;
  scr.counter = reinterpret_cast<uint32_t*>(w);
  size_t off = 256;
  float* zero = reinterpret_cast<float*>(w + off);
  off += al256(4 * Dp);
  scr.flags = reinterpret_cast<uint32_t*>(w + off);
  off += al256(4 * static_cast<size_t>(ntl));
  scr.agg_a = w + off;
  off += al256(4 * ntl * Dp);
  scr.agg_b = w + off;
  off += al256(4 * ntl * Dp);
  scr.incl = w + off;
  e = cudaMemsetAsync(zero, 0, sizeof(float) * Dp, s);
  // the workspace may hold other data where the flags live: clear them (epoch 0 is never used)
  if (e == cudaSuccess) e = cudaMemsetAsync(scr.flags, 0, 4 * static_cast<size_t>(ntl), s);
  if (e != cudaSuccess) return e;
  e = launch_affine_scan(s, false, Dp, T, Arev, Brev, zero, Fh.lam_adj, scr, epoch);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(out, Fh.direct, sizeof(double), cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return e;
  const size_t sr = sizeof(double) * kWarps * (Dp + 1) +
                    sizeof(float) * ((dense ? Dp * Dp : 0) + kWarps * Dp);
  const void* rk = dense ? reinterpret_cast<const void*>(&adjoint_reduce_kernel<kDenseGauss>)
                         : reinterpret_cast<const void*>(&adjoint_reduce_kernel<kDiagGauss>);
  if (sr > 0) {
    e = raise_smem_limit(reinterpret_cast<const void*>(rk), sr);
    if (e != cudaSuccess) return e;
  }
  const float* Lrev = Fh.lam_adj;
  void* rargs[] = {const_cast<DevParams**>(&Pg), const_cast<FullArgs**>(&Fg), &objective,
                   const_cast<float**>(&S), const_cast<float**>(&Lrev), &out};
  return cudaLaunchKernel(rk, dim3(grid), dim3(kThreads), rargs, sr, s);
}

}  // namespace pmcmc
