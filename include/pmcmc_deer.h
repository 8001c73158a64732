/*
 * pmcmc_deer.h -- C ABI of libpmcmc_deer.so, the B200 (sm_100a) DEER hot path of
 * ParallelMCMC.jl.
 *
 * The library replaces everything below `_deer_solve_new_tape`
 * (src/interface.jl:475-515): tape generation, the batched MALA forward +
 * Jacobian estimate (src/MALA/MALA.jl:556-628), the Newton loop of
 * `DEER.solve` (src/DEER/DEER.jl:506-595) with `deer_update!`
 * (src/DEER/DEER.jl:375-475) and the diagonal affine scan
 * (src/DEER/DEERScan.jl:102-173).  Callers keep `mcmcsample`, `step` and the
 * FlexiChains bundling; a Julia `ccall` (or Python ctypes) binding calls these
 * functions with plain pointers.
 *
 * Conventions
 *  - Trajectories are D x T column-major, column t (state t) contiguous, like
 *    the reference's Julia matrices (src/DEER/DEER.jl:451-452).
 *  - Every data pointer is either host or device memory; `mem` flags
 *    (PMCMC_MEM_*) say which.  Device pointers must belong to the handle's
 *    device.  Host buffers need not be pinned.
 *  - Element type of state buffers follows `pmcmc_deer_params.dtype`
 *    (PMCMC_F32 -> float, PMCMC_F64 -> double), as the reference's working
 *    precision follows typeof(epsilon) (src/interface.jl:276-277).
 *  - Return value: PMCMC_OK or an error code; pmcmc_last_error() gives the
 *    message.  ArgumentError / DimensionMismatch of the reference map to
 *    PMCMC_ERR_ARGUMENT / PMCMC_ERR_DIMENSION.  Non-convergence is not an
 *    error (the reference accepts it silently, src/interface.jl:501-513); it
 *    is reported in pmcmc_info.converged.
 *  - Threading: one handle per host thread / stream.  Calls on distinct
 *    handles are independent (AbstractMCMC MCMCThreads, test-DEER-Interface.jl:300-318).
 */
#ifndef PMCMC_DEER_H
#define PMCMC_DEER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PMCMC_ABI_VERSION 1

typedef enum {
  PMCMC_OK = 0,
  PMCMC_ERR_ARGUMENT = 1,    /* reference: ArgumentError */
  PMCMC_ERR_DIMENSION = 2,   /* reference: DimensionMismatch */
  PMCMC_ERR_CUDA = 3,        /* CUDA runtime error */
  PMCMC_ERR_NONFINITE = 4,   /* NaN/Inf reached the trajectory */
  PMCMC_ERR_TIMEOUT = 5,     /* a bounded device wait gave up (never hangs) */
  PMCMC_ERR_UNSUPPORTED = 6, /* valid request this build does not implement */
  PMCMC_ERR_NOMEM = 7
} pmcmc_status;

typedef enum { PMCMC_JAC_STOCH_DIAG = 0, PMCMC_JAC_DIAG = 1, PMCMC_JAC_FULL = 2 } pmcmc_jacobian;
typedef enum { PMCMC_F32 = 0, PMCMC_F64 = 1 } pmcmc_dtype;
typedef enum { PMCMC_MEM_HOST = 0, PMCMC_MEM_DEVICE = 1 } pmcmc_mem;

/* Execution strategy of a solve.
 * PMCMC_EXEC_FUSED: the product path.  Gaussian targets: a whole solve in one
 *   persistent launch, or one fused kernel per Newton sweep with the loop in a
 *   CUDA graph and a device-side convergence test.  Logistic targets: the
 *   tensor-core contraction passes and one fused finish-and-scan kernel per
 *   sweep, the state read by the host after each sweep.
 * PMCMC_EXEC_PLAIN: the reference's structure on the GPU -- separate
 *   broadcast-style kernels, Hillis-Steele doubling scan, host-synchronised
 *   convergence check every iteration, FP32 SIMT only (the "plain GPU DEER"
 *   that the batched, mixed-precision path is measured against). */
typedef enum { PMCMC_EXEC_FUSED = 0, PMCMC_EXEC_PLAIN = 1 } pmcmc_exec;

typedef struct pmcmc_handle pmcmc_handle;
typedef struct pmcmc_target pmcmc_target;

/* ParallelMALASampler fields (src/interface.jl:248-290) plus the modes this
 * library adds (:full, window) and execution controls. */
typedef struct {
  double epsilon;   /* step size, > 0 */
  int64_t T;        /* trajectory length per block (reference default 64) */
  int32_t maxiter;  /* Newton iterations (default 200) */
  double tol_abs;   /* default 1e-6 */
  double tol_rel;   /* default 1e-5 */
  int32_t jacobian; /* pmcmc_jacobian (default STOCH_DIAG) */
  double damping;   /* in (0, 1] (default 0.5) */
  int32_t probes;   /* Hutchinson probes >= 1 (default 1) */
  int64_t window;   /* sliding window width; 0 = whole block */
  int32_t dtype;    /* pmcmc_dtype of state buffers */
  int32_t exec;     /* pmcmc_exec */
} pmcmc_deer_params;

/* DEER.solve info (src/DEER/DEER.jl:585-594) plus parity diagnostics. */
typedef struct {
  int32_t iters;       /* Newton sweeps run */
  int32_t converged;   /* metric <= 1 reached */
  double metric;       /* max|dS| / (tol_abs + tol_rel max|S|), FP64 */
  int64_t n_accept;    /* accepted proposals on the returned trajectory */
  double min_margin;   /* min_t |logalpha_t - log u_t| (FP64) */
  double max_defect;   /* max_t |S_t - f_t(S_{t-1})|_inf of the returned trajectory, from a
                          verification pass at the returned S (accept flags and margins come
                          from the same pass); NaN on the plain logistic path
                          (PMCMC_EXEC_PLAIN), whose flags are those of its last sweep */
  int32_t status;      /* pmcmc_status of the device work */
  int32_t path;        /* PMCMC_PATH_* bits: which kernels ran */
} pmcmc_info;

#define PMCMC_PATH_FUSED_SWEEP 1  /* one fused kernel per Newton sweep */
#define PMCMC_PATH_COOPERATIVE 2  /* cooperative sweep (grid-wide carry scan) */
#define PMCMC_PATH_GRAPH 4        /* Newton loop in a CUDA graph while-node */
#define PMCMC_PATH_TENSOR_CORE 8  /* logistic passes on tcgen05 tensor cores */
#define PMCMC_PATH_FULL_JACOBIAN 16 /* :full mode (dense Jacobian, eigenbasis chunk scan) */
#define PMCMC_PATH_PERSISTENT 32  /* whole solve in one cooperative launch, state in shared memory */
#define PMCMC_PATH_TIE_FP64 64    /* logistic, FP32 state: near-tie accept decisions taken from an
                                     FP64 evaluation of log alpha in every sweep */

/* ---- handle ------------------------------------------------------------ */
/* Replaces DEERWorkspace (src/DEER/DEER.jl:47-90): owns all device workspace,
 * reused across blocks and solves.  `stream` may be NULL (handle creates one). */
int pmcmc_create(int device, void* stream, pmcmc_handle** out);
int pmcmc_destroy(pmcmc_handle* h);
const char* pmcmc_last_error(const pmcmc_handle* h);
int pmcmc_abi_version(void);

/* ---- targets -------------------------------------------------------------
 * Replace the user closures of DensityModel (src/interface.jl:36-70) with
 * built-in device targets.  Parameters are copied to the device at creation.
 * Diagonal Gaussian: logp = -1/2 sum_i prec_i (x_i - mean_i)^2
 *   (test-DEER-Interface.jl:13-16, test-GPU-MALA.jl:34-44).
 * Dense Gaussian: logp = -1/2 (x-mean)' P (x-mean), P symmetric D x D.
 * Logistic regression (bayes_logreg.jl:30-86, 91-206): X is N x D
 *   column-major (Julia), y in {0,1}, prior N(0, prior_prec^-1 I).
 * `mean` may be NULL (zero).  All pointers are host memory. */
int pmcmc_target_diag_gauss(pmcmc_handle* h, int64_t D, const double* mean, const double* prec,
                            pmcmc_target** out);
int pmcmc_target_dense_gauss(pmcmc_handle* h, int64_t D, const double* mean,
                             const double* prec, pmcmc_target** out);
int pmcmc_target_logistic(pmcmc_handle* h, int64_t N, int64_t D, const double* X,
                          const double* y, double prior_prec, pmcmc_target** out);
/* Mass matrix M = L L^T: replaces the `cholM = cholesky(M)` keyword of
 * MALASampler / ParallelMALASampler / AdaptiveMALASampler (src/interface.jl:
 * 84-100, 241-287, 899-930) that MALA.jl applies in every step (src/MALA/MALA.jl:
 * 29-47).  `L` is the D x D lower Cholesky factor, column-major host memory
 * (entries above the diagonal are ignored; the diagonal must be positive).
 * Returns a new target, independent of `base` (which may be destroyed), whose
 * solves, samples and sequential chains (pmcmc_deer_solve, pmcmc_sample,
 * pmcmc_fleet_solve, pmcmc_mala_chains) run the chain with mass M, outputs in
 * the base target's coordinates; internally it is the whitened Gaussian
 * x' = L^-1 x (precision L^T P L, mean L^-1 mean), where the same tape gives the
 * same chain, and its `info` defects are in those coordinates.  Gaussian bases
 * with D <= 4096; logistic bases, the adjoint and slices return
 * PMCMC_ERR_UNSUPPORTED. */
int pmcmc_target_mass(pmcmc_handle* h, const pmcmc_target* base, const double* L,
                      pmcmc_target** out);
int pmcmc_target_destroy(pmcmc_target* t);

/* ---- tape ------------------------------------------------------------------
 * Counter-based replacement of _make_mala_tape_block (src/interface.jl:334-358):
 * writes Xi (D x T, float) and u (T, float) for (seed, block). */
int pmcmc_tape(pmcmc_handle* h, int64_t D, int64_t T, uint64_t seed, uint64_t block, float* Xi,
               float* u, int32_t mem);

/* ---- one DEER block ---------------------------------------------------------
 * Replaces _deer_solve_new_tape + DEER.solve + _trajectory_logps
 * (src/interface.jl:475-524, src/DEER/DEER.jl:506-595): draws the tape of
 * (seed, block), solves the T-step trajectory from x0 and writes
 *   S_out    D x T trajectory (dtype), column t = x_{t+1}
 *   logp_out T log densities of the returned columns (dtype), may be NULL
 *   accept_out T accept flags (uint8), may be NULL
 * x0 has dtype and lives in `mem`; outputs live in `mem`. */
int pmcmc_deer_solve(pmcmc_handle* h, const pmcmc_target* t, const pmcmc_deer_params* p,
                     const void* x0, uint64_t seed, uint64_t block, void* S_out, void* logp_out,
                     uint8_t* accept_out, int32_t mem, pmcmc_info* info);

/* ---- block loop ---------------------------------------------------------------
 * Replaces the block loop of _sample_parallel_mala_chain / _blocks
 * (src/interface.jl:557-607, 661-711): ceil(N/T) blocks, block b uses tape
 * block b, keeps min(T, N - nsteps) columns, next x0 = last kept column.
 * vals_out D x N (dtype), logp_out N (dtype, may be NULL), accept_out N (may be NULL).
 * info accumulates: iters = total sweeps, converged = all blocks converged,
 * metric = worst block metric.
 * The blocks run back to back with no host round trip between them; with device
 * outputs on the persistent path (Gaussian targets) they are one launch.  A block
 * that fails (non-finite state) does not stop the blocks after it, whose outputs
 * are then meaningless; the call returns the first failing block's status and info
 * counts the blocks up to it. */
int pmcmc_sample(pmcmc_handle* h, const pmcmc_target* t, const pmcmc_deer_params* p,
                 const void* x0, uint64_t seed, int64_t N, void* vals_out, void* logp_out,
                 uint8_t* accept_out, int32_t mem, pmcmc_info* info);

/* ---- dense-Jacobian mode and the adjoint -------------------------------------
 * jacobian = PMCMC_JAC_FULL has no counterpart in the reference, which rejects
 * :full (src/DEER/DEER.jl:465-466, src/interface.jl:274-275).  Here it is
 * Newton with the exact Jacobian of the surrogate step (the matrix whose action
 * is the JVP of src/MALA/MALA.jl:768-795), built for the Gaussian targets with
 * FP32 state, D <= 128 and no sliding window; other requests return
 * PMCMC_ERR_UNSUPPORTED.
 *
 * pmcmc_target_eigen: the eigendecomposition P = Q diag(lam) Q^T of a
 * Gaussian target's precision that the :full mode and the adjoint work in.
 * lam has D entries (ascending for the dense target, the given order for the
 * diagonal one); Q (D x D column-major, may be NULL) holds the eigenvectors.
 * Host pointers. */
int pmcmc_target_eigen(pmcmc_target* t, double* lam, double* Q);

/* pmcmc_deer_adjoint (no counterpart in the reference): gradient of an
 * objective of a solved trajectory with the accept decisions of that
 * trajectory held fixed, by a reverse scan.  S is the D x T trajectory
 * returned by pmcmc_deer_solve for the same (p, x0, seed, block),
 * in `mem`; grad (host, 1 + D doubles) receives dL/depsilon in grad[0] and,
 * for PMCMC_OBJ_MEAN_SQ, dL/dlog s_i in grad[1 + i] for the covariance
 * eigenvalues s_i = 1 / lam_i in pmcmc_target_eigen's order (zeros for
 * PMCMC_OBJ_ESJD).  Objectives:
 *   PMCMC_OBJ_ESJD     (1/T) sum_t min(1, alpha_t) |y_t - x_{t-1}|^2
 *   PMCMC_OBJ_MEAN_SQ  (1/T) sum_t |x_t|^2
 * Gaussian targets: FP32 state, D <= 128, one reverse scan in the eigenbasis.
 * Logistic targets: FP32 or FP64 state (S and x0 of p->dtype), computed in FP64;
 * the reverse recurrence with the dense Jacobians I + eps H(x_t) is solved by
 * Jacobi iterations on its diagonal (at most p->maxiter, to 1e-12 relative;
 * PMCMC_ERR_TIMEOUT if they do not get there); grad[1 .. D] are NaN (no density
 * parameter).  Mass-matrix targets return PMCMC_ERR_UNSUPPORTED. */
typedef enum { PMCMC_OBJ_ESJD = 0, PMCMC_OBJ_MEAN_SQ = 1 } pmcmc_objective;
int pmcmc_deer_adjoint(pmcmc_handle* h, const pmcmc_target* t, const pmcmc_deer_params* p,
                       const void* x0, uint64_t seed, uint64_t block, const void* S,
                       int32_t mem, int32_t objective, double* grad);

/* ---- fleet of independent chains ---------------------------------------------
 * Many independent chains of uneven size (D, N, T) on one GPU.  The reference
 * runs independent chains through AbstractMCMC's MCMCThreads, one chain and
 * one workspace per thread (test/test-DEER-Interface.jl:300-318).  Here
 * `workers` worker handles, each with its own stream and workspace, take
 * chains largest-first (cost ~ D * N * T) so that small chains fill the device
 * beside the large ones; every chain runs its own Newton loop to its own
 * convergence (pmcmc_deer_solve semantics: one block of params.T columns).
 * Targets may be shared by chains (read-only).  Per-chain results land in the
 * array; the return value is the first failing chain's status, or PMCMC_OK. */
typedef struct {
  const pmcmc_target* target;
  pmcmc_deer_params params;
  const void* x0;        /* D, dtype, in `mem` */
  uint64_t seed, block;
  void* S_out;           /* D x T, in `mem` */
  void* logp_out;        /* T, may be NULL */
  uint8_t* accept_out;   /* T, may be NULL */
  pmcmc_info info;       /* out */
  int32_t status;        /* out: pmcmc_status of this chain */
  int32_t pad0;
} pmcmc_fleet_chain;
int pmcmc_fleet_solve(pmcmc_handle* h, pmcmc_fleet_chain* chains, int64_t n, int32_t workers,
                      int32_t mem);

/* ---- T-split slices (multi-GPU) ------------------------------------------------
 * One long chain split into contiguous slices of the block, one per rank, with
 * one exchange per Newton sweep.  The reference solves a block on one device
 * (src/DEER/DEER.jl:506-595); these entry points run its deer_update! (DEER.jl:
 * 398-475) on columns [t0, t0 + W) so that a caller can compose the slices'
 * affine maps across ranks (the associativity of DEERScan.jl:102-173).  Per
 * sweep, on every rank:
 *   1. xbar0 = last column of rank r-1's iterate (x0 on rank 0) -- exchanged;
 *   2. pmcmc_slice_local: A, B on the slice, agg = [prod_t A_t ; b] (2 x D) with
 *      b the slice scanned from zero;
 *   3. carry = maps of ranks 0..r-1 applied to x0 in order (s = a .* s + b);
 *   4. pmcmc_slice_finish: the slice scanned from carry, damped against the
 *      previous iterate; red = {max|dS|, max|S|} for the caller's max-reduction
 *      and the convergence test; last_out = the new last column.
 * pmcmc_slice_result runs the verification pass on the final iterate (accept
 * flags, logp, S).  Gaussian targets, :diag / :stoch_diag; state dtype and mem
 * as in pmcmc_deer_solve.  The slice lives in the handle until the next begin. */
int pmcmc_slice_begin(pmcmc_handle* h, const pmcmc_target* t, const pmcmc_deer_params* p,
                      const void* x0, uint64_t seed, uint64_t block, int64_t t0, int64_t W,
                      int32_t mem);
int pmcmc_slice_local(pmcmc_handle* h, const void* xbar0, void* agg, int32_t mem);
int pmcmc_slice_finish(pmcmc_handle* h, const void* carry_in, void* last_out, double* red,
                       int32_t mem);
int pmcmc_slice_result(pmcmc_handle* h, const void* xbar0, void* S_out, void* logp_out,
                       uint8_t* accept_out, pmcmc_info* info, int32_t mem);

/* ---- diagonal affine scan ----------------------------------------------------
 * Replaces DEERScan.solve_affine_scan_diag! (src/DEER/DEERScan.jl:102-173):
 * S[:,t] = A[:,t] .* S[:,t-1] + B[:,t], S[:,0-1] = s0.  Single-pass
 * decoupled-lookback scan.  S may not alias A or B (DEERScan.jl:124-125). */
int pmcmc_affine_scan_diag(pmcmc_handle* h, int32_t dtype, int64_t D, int64_t T, const void* A,
                           const void* B, const void* s0, void* S, int32_t mem);

/* ---- diagonal affine scan without allocation ----------------------------------
 * No counterpart in the reference.  For callers that may not call cudaMalloc
 * once running (a process whose own pool already owns the device memory, such
 * as a Julia session with CUDA.jl's pool or a serving process with a fixed
 * memory budget, or a latency-critical loop that cannot take an allocation's
 * implicit synchronisation): the same scan as pmcmc_affine_scan_diag, with A,
 * B, s0 and S device pointers on the current device and no handle.  The
 * look-back scratch is a static device array of PMCMC_NOALLOC_SCRATCH_BYTES
 * (4 MiB) that every GPU loading the library holds until the process exits;
 * no cudaMalloc, cudaFree or allocating library routine is called.  A size
 * whose scratch exceeds the array returns PMCMC_ERR_NOMEM (the scratch needed
 * is about 3 * sizeof(element) * D * ceil(T / tile) bytes, tile <= 64 columns).
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture.  The array takes its device memory
 * when the library's device code is loaded on a device: under lazy module
 * loading (CUDA_MODULE_LOADING=LAZY, the CUDA 12 default) that is this first
 * call, so a caller that later hands all free memory to its own pool should
 * make one call (D = T = 1 will do) before reserving the pool.  Calls share the array: calls that
 * overlap on the GPU (other streams or host threads) race and must be
 * serialised by the caller.  Synchronises `stream` before returning. */
#define PMCMC_NOALLOC_SCRATCH_BYTES (4u << 20)
int pmcmc_affine_scan_diag_noalloc(int32_t dtype, int64_t D, int64_t T, const void* A,
                                   const void* B, const void* s0, void* S, void* stream);

/* ---- profiling ------------------------------------------------------------
 * With profiling on, solves run their Newton loop as individual launches with
 * CUDA events around every sweep and finalize kernel (no graph); the device
 * times accumulate until pmcmc_get_profile is called with reset = 1.  Used by
 * bench.py to time the dominant kernel; no counterpart in the reference
 * (its benchmarks time whole solves, benchmarks/.../profile_deer_logreg_components.jl). */
typedef struct {
  int64_t sweep_launches;
  double sweep_ms;      /* one Newton sweep (the fused kernel; the four :full kernels) */
  int64_t finalize_launches;
  double finalize_ms;
  int64_t pass_launches;
  double pass_ms;       /* logistic target: one gradient/HVP contraction pass */
  int64_t solve_launches;
  double solve_ms;      /* persistent kernel: a whole solve (tape, sweeps, verification) */
  int64_t solve_sweeps; /* Newton sweeps inside those launches */
} pmcmc_profile;
int pmcmc_set_profiling(pmcmc_handle* h, int32_t on);
int pmcmc_get_profile(pmcmc_handle* h, pmcmc_profile* out, int32_t reset);

/* pmcmc_mala_chains (no counterpart entry point in the reference, which runs
 * such chains one by one on the CPU, src/MALA/MALA.jl:322-346, 377-411): n independent
 * sequential MALA chains of p->T steps each, one warp a chain.  Chain c starts
 * at x0[c*D .. c*D+D) and uses the tape of (seeds[c], block), the tape a DEER
 * solve with that seed and block uses, so its trajectory is the one DEER
 * converges to.  Outputs: S_out n x T x D (step t of chain c at
 * (c*T + t)*D), logp_out n x T and accept_out n x T (either may be NULL).
 * Element type per p->dtype; Gaussian targets only (others return
 * PMCMC_ERR_UNSUPPORTED); p is validated as for a solve, and only its
 * epsilon, T and dtype are used. */
int pmcmc_mala_chains(pmcmc_handle* h, const pmcmc_target* t, const pmcmc_deer_params* p,
                      int64_t n, const void* x0, const uint64_t* seeds, uint64_t block,
                      void* S_out, void* logp_out, uint8_t* accept_out, int32_t mem);

/* pmcmc_mala_chains_adaptive: the same chains as AdaptiveMALASampler runs them
 * (src/interface.jl:899-933 settings, 1024-1065 step): chain c carries its own
 * step size, epsilon_init = p->epsilon.  Step m (0-based) uses epsilon while
 * m < n_warmup and epsilon_bar after, and during warmup is followed by the
 * dual-averaging update _dual_average_update (src/interface.jl:962-984) with
 * that step's log alpha and m + 1.  The settings are checked as the
 * reference's constructor checks them (PMCMC_ERR_ARGUMENT).  Extra outputs
 * (either may be NULL; host or device per mem): eps_out n x T, the step size
 * of every step (the transition's step_size; is_warmup = m < n_warmup), and
 * state_out n x 3, the final (epsilon, epsilon_bar, H_bar) of every chain.
 * The adaptation is computed in FP64 whatever p->dtype. */
typedef struct pmcmc_adapt {
  int64_t n_warmup;     /* 1000 in the reference */
  double target_accept; /* 0.574 */
  double gamma;         /* 0.05 */
  double t0;            /* 10.0 */
  double kappa;         /* 0.75 */
} pmcmc_adapt;
int pmcmc_mala_chains_adaptive(pmcmc_handle* h, const pmcmc_target* t,
                               const pmcmc_deer_params* p, int64_t n, const void* x0,
                               const uint64_t* seeds, uint64_t block, const pmcmc_adapt* ad,
                               void* S_out, void* logp_out, uint8_t* accept_out,
                               double* eps_out, double* state_out, int32_t mem);

/* pmcmc_autotune (no counterpart in the reference): times the candidate
 * shapes of the kernels that would solve (t, p) on x0 and keeps the fastest
 * for every later solve of the same shape (target kind, Jacobian, precision, D,
 * T), process-wide.  Candidates: CTAs a SM of the persistent solve (1..4, as
 * fit), or the :full chunk count (about sqrt(f T), f = 1/2, 1, 2, 4).  Each
 * candidate solves tape block 0 of `seed` three times (the first warms up).
 * *choice gets the kept value (0 when the path has nothing to tune) and
 * *best_ms its time.  Allocates and frees its own scratch. */
int pmcmc_autotune(pmcmc_handle* h, const pmcmc_target* t, const pmcmc_deer_params* p,
                   const void* x0, uint64_t seed, int32_t mem, int32_t* choice,
                   double* best_ms);

/* ---- bound check of the device waits (no counterpart in the reference, whose
 * device code never waits on another block) ------------------------------------
 * Runs one of the library's bounded waits on a flag that nothing sets: the
 * look-back spin of the scans and sweeps (PMCMC_WAIT_LOOKBACK), or the
 * mbarrier wait of the tensor-core pass (PMCMC_WAIT_MBARRIER).  The wait
 * gives up at its bound, the kernel returns normally and the call returns
 * PMCMC_ERR_TIMEOUT with the device time in *wait_ms; the handle and its
 * context stay usable.  PMCMC_OK would mean the wait ended without its flag. */
typedef enum { PMCMC_WAIT_LOOKBACK = 0, PMCMC_WAIT_MBARRIER = 1 } pmcmc_wait_kind;
int pmcmc_check_wait_bound(pmcmc_handle* h, int32_t kind, double* wait_ms);

#ifdef __cplusplus
}
#endif
#endif /* PMCMC_DEER_H */
