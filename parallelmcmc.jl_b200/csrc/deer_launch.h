// deer_launch.h -- host-side view of the kernels (no torch types, plain CUDA runtime).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace pmcmc {

struct SmemPlan {
  size_t xs, as, carry, pd, pf, vd, vf, total;
  int p_in_smem;
};

struct SweepKernels {
  const void* sweep = nullptr;     // (const DevParams*, DevState*, cudaGraphConditionalHandle, int)
  const void* sweep_coop = nullptr;  // same signature, cooperative launch (all tiles resident)
  const void* finalize = nullptr;  // (const DevParams*, DevState*)
  const void* init = nullptr;      // (const DevParams*, DevState*)
  const void* eval = nullptr;      // (const DevParams*, const Real* Sold, int iter, int from_x0, Real* A, Real* B);
                                   // logistic: the probe accumulation (const DevParams*, const DevState*, int probe)
  const void* persist = nullptr;   // (const DevParams*, DevState*): whole solve, cooperative
  int qpl = 1;
};

// Shared memory of the persistent solve kernel (deer_persist.cu): the sweep
// plan at TT columns plus the CTA's tape (TT + 1 columns of xi and log u).
struct PersistPlan {
  SmemPlan sweep;
  size_t xi, lu, x0, total;
};
PersistPlan persist_smem(bool f64, int64_t Dp, int TT, bool dense);
const void* persist_kernel(bool f64, int tk, int jac, int64_t D);

// Raises a kernel's dynamic shared-memory limit to at least `bytes`, never
// lowering it: the attribute is global per function, and handles on other
// host threads (the fleet) launch the same kernels with other sizes.
cudaError_t raise_smem_limit(const void* fn, size_t bytes);

SweepKernels gauss_sweep_kernels(bool f64, int tk, int jac, int64_t D);
SweepKernels logistic_sweep_kernels(bool f64, int64_t D, int jac);
SmemPlan gauss_sweep_smem(bool f64, int64_t Dp, int TT, bool dense);

// Independent sequential MALA chains, one warp a chain (mala_chains.cu): chain c
// from x0[c * D ..] with the tape of (seeds[c], P.block); S is nchains x T x D.
// With ad.active every chain adapts its step size by dual averaging from
// epsilon_init = P.eps; eps_out (nchains x T, or nullptr) gets the step size of
// every step and state_out (nchains x 3, or nullptr) the final (epsilon,
// epsilon_bar, H_bar).
struct DevParams;
struct ChainAdapt {
  int active;
  int64_t n_warmup;
  double target_accept, gamma, t0, kappa;
};
size_t mala_chains_smem(bool f64, int64_t Dp, bool dense);
cudaError_t launch_mala_chains(cudaStream_t s, bool f64, int tk, const DevParams& P,
                               const ChainAdapt& ad, int64_t nchains, const void* x0,
                               const uint64_t* seeds, void* S, void* logp, uint8_t* acc,
                               double* eps_out, double* state_out);

// Tape materialisation (tape.cu).
cudaError_t launch_tape(cudaStream_t s, int64_t D, int64_t T, uint64_t seed, uint64_t block,
                        float* Xi, float* u);

// Standalone diagonal affine scan (scan_diag.cu).  Scratch: flags[ntiles],
// agg_a/agg_b/incl[ntiles * Dp] of the element type, counter[1].
struct ScanScratch {
  uint32_t* flags;
  void* agg_a;
  void* agg_b;
  void* incl;
  uint32_t* counter;
};
int scan_tile_cols(int64_t D, int64_t T);
size_t scan_scratch_bytes(bool f64, int64_t D, int64_t T);
cudaError_t launch_affine_scan(cudaStream_t s, bool f64, int64_t D, int64_t T, const void* A,
                               const void* B, const void* s0, void* S, const ScanScratch& scr,
                               uint32_t epoch);

// Plain path (tape_scan.cu): the reference's Hillis-Steele doubling scan
// (DEERScan.jl:102-173) as one launch per level over buffers of T x Dp
// elements, and damping + max-reductions into red[2] (double bits).
cudaError_t launch_doubling_scan(cudaStream_t s, bool f64, int64_t Dp, int64_t T, const void* A,
                                 const void* B, const void* s0, void* S, void* al0, void* be0,
                                 void* al1, void* be1);
cudaError_t launch_damp_metric(cudaStream_t s, bool f64, int64_t D, int64_t Dp, int64_t T,
                               const void* S_old, void* S_new, double damping,
                               unsigned long long* red);

// One look-back over `flags` (>= 1 zero word) that nothing publishes; err[0] =
// 1 when the wait reached its bound (bound check of the scans' waits).
cudaError_t launch_lookback_bound(cudaStream_t s, const uint32_t* flags, int* err);

cudaError_t launch_broadcast(cudaStream_t s, bool f64, int64_t Dp, int64_t T, const void* x0,
                             void* S);

// Mass matrix M = L L^T (mass.cu), L column-major lower triangular in FP64:
// y = L^-1 x for n D-vectors and S[:, j] <- L S[:, j] for N columns, in place.
int64_t mass_max_dim();
cudaError_t mass_whiten(cudaStream_t s, const double* L, int64_t D, int64_t n, const void* x,
                        void* y, bool f64);
cudaError_t mass_map(cudaStream_t s, const double* L, int64_t D, int64_t N, void* S, bool f64,
                     int num_sms);

}  // namespace pmcmc
