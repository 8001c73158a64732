/*
 * pmcmc_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of ParallelMCMC.jl's DEER hot path (sequential MALA,
 * surrogate JVP, batched fwd+JVP, DEER update/solve, affine scans), used by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
 * as the checker.  It is never linked into, loaded by, or called from the
 * product library (libpmcmc_deer.so).
 *
 * Parity status: "parity unpinned" against reference outputs.  The reference
 * (pure Julia) ships no golden vectors and Julia is not installed here, so the
 * restatement is pinned by (a) the reference's own property tests restated
 * (tests/test_oracle_*.py), (b) an independent NumPy restatement on small
 * cases, and (c) the published Philox4x32-10 known-answer vectors for the
 * tape generator.
 *
 * Layout conventions follow the reference (Julia, column-major): a D x T
 * trajectory S stores column t (one state) contiguously at S + t*D.
 * The logistic design matrix X is N x D column-major (X[n,i] = X[i*N+n]),
 * exactly as `X * beta` in bayes_logreg.jl.
 */
#ifndef PMCMC_ORACLE_H
#define PMCMC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_DIAG_GAUSS = 0, ORC_DENSE_GAUSS = 1, ORC_LOGISTIC = 2 };
enum { ORC_JAC_STOCH_DIAG = 0, ORC_JAC_DIAG = 1, ORC_JAC_FULL = 2 };

typedef struct {
    int32_t kind;
    int64_t D;
    int64_t N;             /* logistic rows */
    const double* mean;    /* gaussians: length D (may be NULL = 0) */
    const double* prec;    /* diag: D values; dense: D*D column-major */
    const double* X;       /* logistic: N x D column-major */
    const double* y;       /* logistic: N labels in {0,1} */
    double prior_prec;     /* logistic prior N(0, prior_prec^-1 I) */
} orc_target;

typedef struct {
    double eps;
    double tol_abs, tol_rel;
    int32_t maxiter;
    int32_t jacobian;      /* ORC_JAC_* */
    double damping;
    int32_t probes;
    int32_t batched;       /* 1: batched fwd+JVP branch (DEER.jl:398-419) for stoch_diag */
    int32_t scan_doubling; /* 1: Hillis-Steele doubling scan (DEERScan.jl:102-173); 0: sequential */
    int64_t window;        /* 0 = whole trajectory; else sliding-window width */
    int32_t nthreads;      /* OpenMP threads (0 = default) */
} orc_deer_params;

typedef struct {
    int32_t iters;
    int32_t converged;
    double metric;
} orc_deer_info;

/* ---- tape generator (Philox4x32-10 + Box-Muller, FP32, bit-identical to the device) ---- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
float orc_u01(uint32_t bits);
float orc_logf(float x);
void orc_sincos2pi(float u, float* s, float* c);
void orc_tape(uint64_t seed, uint64_t block, int64_t D, int64_t T, float* Xi, float* u);
void orc_probe(uint64_t seed, uint64_t block, int32_t iter, int32_t probe, int64_t D,
               int64_t T, double* Z);

/* ---- targets (bayes_logreg.jl:30-86, test-DEER-Interface.jl:13-16) ---- */
double orc_logp(const orc_target* tg, const double* x);
void orc_grad(const orc_target* tg, const double* x, double* g);
void orc_hvp(const orc_target* tg, const double* x, const double* v, double* out);

/* ---- MALA (MALA.jl) ---- */
double orc_logq(const orc_target* tg, const double* y, const double* x, const double* gx,
                double eps);
double orc_mala_step(const orc_target* tg, double eps, const double* x, const double* xi,
                     double u, double* x_next, int32_t* accepted);
void orc_mala_sequential(const orc_target* tg, double eps, const double* x0, const double* Xi,
                         const double* u, int64_t T, double* S, int32_t* accepted,
                         double* logalpha);
/* orc_mala_sequential for the logistic target, the accepted proposal's log density and
 * gradient carried to the next step, the target's sums split over threads with their
 * order kept: the same results bit for bit, fast enough for full-size chains. */
void orc_mala_sequential_logistic(const orc_target* tg, double eps, const double* x0,
                                  const double* Xi, const double* u, int64_t T, double* S,
                                  int32_t* accepted, double* logalpha, int32_t nthreads);
/* Sequential MALA with mass matrix M = L L^T (L lower triangular, D x D column-major). */
void orc_mala_sequential_mass(const orc_target* tg, double eps, const double* L, const double* x0,
                              const double* Xi, const double* u, int64_t T, double* S,
                              int32_t* accepted, double* logalpha);
void orc_fwd_and_jvp(const orc_target* tg, double eps, const double* x, const double* xi,
                     double u, const double* v, double* f, double* jv);
void orc_fwd_and_jvp_batched(const orc_target* tg, double eps, int64_t T, const double* X,
                             const double* Xi, const double* u, const double* Z, double* FT,
                             double* Jt, int32_t nthreads);
void orc_jac_full(const orc_target* tg, double eps, const double* x, const double* xi,
                  double u, double* f, double* J);

/* ---- affine scans (DEERScan.jl) ---- */
void orc_scan_seq(int64_t D, int64_t T, const double* A, const double* B, const double* s0,
                  double* S);
void orc_scan_doubling(int64_t D, int64_t T, const double* A, const double* B,
                       const double* s0, double* S, double* ws /* 4*D*T */);
double orc_scan_residual(int64_t D, int64_t T, const double* S, const double* A,
                         const double* B, const double* s0);
void orc_scan_dense_seq(int64_t D, int64_t T, const double* J, const double* B,
                        const double* s0, double* S);

/* ---- DEER (DEER.jl) ---- */
int orc_deer_update(const orc_target* tg, const orc_deer_params* p, int64_t T,
                    const double* s0, const double* S_in, const double* Xi, const double* u,
                    uint64_t seed, uint64_t block, int32_t iter, double* S_out,
                    double* A_out, double* B_out);
int orc_deer_solve(const orc_target* tg, const orc_deer_params* p, int64_t T,
                   const double* s0, const double* Xi, const double* u, uint64_t seed,
                   uint64_t block, double* S_out, orc_deer_info* info);

#ifdef __cplusplus
}
#endif
#endif
