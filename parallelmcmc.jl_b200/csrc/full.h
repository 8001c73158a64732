// full.h -- host view of the dense-Jacobian (:full) sweep and the adjoint pass.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace pmcmc {

struct DevParams;
struct DevState;

// Device-resident arguments of the :full sweep (one copy per handle, refreshed
// per solve, so that a captured graph stays valid across solves).  The
// Gaussian precision is P = Q diag(lam) Q^T; every Jacobian quantity is kept in
// the eigenbasis (primed).
struct FullArgs {
  const DevParams* Pe;  // the eigenbasis view: prec = lam, mean = 0, xi' = Q^T xi, x0', S'
                        // (its Dp is the sweep stride Dq)
  const float* lam;     // Dp eigenvalues of P (0 in the padding)
  const float* Qrm;     // Dp x Dp, Q row-major: matvec4 with it applies Q^T
  const float* Qcm;     // Dp x Dp, Q column-major: matvec4 with it applies Q
  const float* lamQ;    // the same three padded to the sweep stride Dq (16, 32, 64 or 128)
  const float* QrmQ;
  const float* QcmQ;
  float* U;             // T x Dq  u'_t = Q^T g(1-g)(y_t - x_t)
  float* V;             // T x Dq  v'_t = Q^T grad log alpha_t
  float* R;             // T x Dq  r'_t = f'_t - S'_t   (Newton residual)
  uint8_t* acc;         // T       accept flags of the current sweep
  float* Phi;           // nchunks x Dq x Dq chunk maps (column-major)
  float* beta;          // nchunks x Dq      chunk offsets
  float* din;           // nchunks x Dq      primed update entering each chunk
  double* part;         // nchunks x 2       each apply CTA's max|dS|, max|S|
  int32_t L, nchunks;
  int32_t rot, Dq;
  // adjoint
  float* lam_adj;       // T x Dp  reversed primed adjoint
  float* cterm;         // T x Dp  reversed primed objective terms
  float* arev;          // T x Dp  reversed scan multipliers
  double* direct;       // [1]     explicit d/deps of the objective
};

// Stride of the :full sweep buffers: the smallest of 16, 32, 64, 128 >= Dp
// (0 when Dp > 128).
int full_stride(int64_t Dp);

struct FullPlan {
  int Dq = 0;
  int L = 0, nchunks = 0;
  int eval_grid = 0;
  size_t smem_eval = 0, smem_chunk = 0, smem_carry = 0, smem_apply = 0;
  int threads_chunk = 0;
  const void* eval = nullptr;
  const void* chunk = nullptr;
  const void* carry = nullptr;
  const void* apply = nullptr;
  const void* rotate = nullptr;
  int rotate_grid = 0;
  size_t smem_rotate = 0;
};

// Chunking and kernel choice for padded dimension Dp (<= 128) and length T;
// returns false when the dimension is outside the built range.
bool full_plan(int64_t Dp, int64_t T, int tkind, int num_sms, int chunks_override, FullPlan* fp);

// One sweep = eval, chunk maps, carry, replay + damping + convergence test.
// Kernel signatures: (const DevParams*, const FullArgs*, DevState*, cudaGraphConditionalHandle, int use_cond).
// `rotate` (same signature, grid rotate_grid) fills the eigenbasis tape xi' and
// x0' once per solve, after the tape kernel.
cudaError_t full_sweep(cudaStream_t s, const FullPlan& fp, const DevParams* Pg, const FullArgs* Fg,
                       DevState* st, cudaGraphConditionalHandle cond, int use_cond);

// Adjoint of an objective at a converged trajectory S (T x Dp, padded), with
// the accept decisions of that trajectory held fixed.  objective 0 = mean
// Rao-Blackwellised squared jump (ESJD), 1 = mean |x_t|^2.  out[0] = dL/deps,
// out[1 + i] = dL/dlog s_i for the covariance eigenvalues s_i = 1/lam_i
// (objective 1 only; zeros for objective 0).
// `scratch` holds full_adjoint_scratch_bytes(Dp, T) bytes; `epoch` must differ
// from every earlier call on it.
cudaError_t full_adjoint(cudaStream_t s, const DevParams* Pg, const FullArgs* Fg,
                         const FullArgs& Fh, int64_t D, int64_t Dp, int64_t T, int tkind,
                         int num_sms, int objective, const float* S, double* out,
                         void* scratch, uint32_t epoch);

size_t full_adjoint_scratch_bytes(int64_t Dp, int64_t T);

}  // namespace pmcmc
