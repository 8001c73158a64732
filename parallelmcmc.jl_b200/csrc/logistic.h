// logistic.h -- host-side interface of the logistic-regression target.
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <cuda_fp16.h>

#include <cstdint>

#include "deer_device.cuh"

namespace pmcmc {

// Device copies of the data: X row-major N x Dp (padded columns zero), labels.
struct LogisticDev {
  int64_t N = 0, D = 0, Dp = 0;
  float* X32 = nullptr;
  double* X64 = nullptr;
  float* y32 = nullptr;
  double* y64 = nullptr;
  double tau = 1.0;
  // tensor-core operands: X as FP16 hi + lo, Np x Dk (rows padded to 128,
  // columns padded to 128); only built when D <= 256
  int64_t Np = 0, Dk = 0;
  __half* Xh = nullptr;
  __half* Xl = nullptr;
  // X .* X for the exact diagonal (:diag), made on first use (lg_make_square)
  float* X2_32 = nullptr;
  double* X2_64 = nullptr;
};

int64_t lg_chunk_cols(int64_t N, int64_t T);
// `probe` picks the Rademacher probe of the tangent columns (mode 0; DEER.jl:412-416).
int lg_plain_pass(cudaStream_t s, cublasHandle_t cb, const LogisticDev& X, bool f64,
                  const DevParams* dP, const DevState* dS, double* lp, int mode, int64_t T,
                  int64_t Dp, void* Bbuf, void* Lbuf, void* Gbuf, int64_t Tc, int probe);

cudaError_t lg_mid(cudaStream_t s, bool f64, const DevParams* dP, const DevState* dS, int stage,
                   int64_t t0, int Tc, int probe, int64_t Dp, const void* G);
// X2 = X .* X in the state's precision (once; the caller serialises first uses).
cudaError_t lg_make_square(cudaStream_t s, LogisticDev& X, bool f64);

// Tensor-core pass (logistic_tc.cu): mode 0/1/2 as in lg_plain_pass; writes G
// (Dp x 2T FP32, value block then tangent block) and lp.  ws holds the FP16
// operand arrays and an error word (lg_tc_ws_bytes).
bool lg_tc_supported(const LogisticDev& X);
size_t lg_tc_ws_bytes(const LogisticDev& X, int64_t T);
int lg_tc_pass(cudaStream_t s, const LogisticDev& X, const DevParams* dP, const DevState* dS,
               double* lp, int mode, int64_t T, void* ws, float* G, int probe);
int* lg_tc_err_word(void* ws, const LogisticDev& X, int64_t T);
// One bounded mbarrier wait that nothing completes (bound check); err[0] = 1
// when it gave up.
cudaError_t lg_tc_mbar_bound(cudaStream_t s, int* err);

// Near-tie decisions in FP64 and the verification pass (logistic_tie.cu).
// Scratch of one refinement over at most kmax columns.
struct TieBufs {
  int kmax = 0;
  float* mg = nullptr;      // [T] |log alpha - log u| of the sweep
  int32_t* list = nullptr;  // [kmax] selected columns, ascending
  int32_t* info = nullptr;  // [4] selected, inside the widest band, band index
  double *Bx = nullptr, *By = nullptr, *GX = nullptr, *G = nullptr, *G2 = nullptr;  // [kmax x Dp]
  double* L = nullptr;                                                            // [kmax x N]
  double *lpx = nullptr, *lpy = nullptr;                                          // [kmax]
};
size_t lg_tie_ws_bytes(const LogisticDev& X, int64_t T, int kmax);
TieBufs lg_tie_carve(void* ws, const LogisticDev& X, int64_t T, int kmax);
// log alpha of every column as the sweep forms it -> la_ref, |margin| -> mg.
cudaError_t lg_margin(cudaStream_t s, bool f64, const DevParams* dP, const DevState* dS,
                      int64_t T, double* la_ref, float* mg);
// lg_margin, then FP64 log alpha for the columns whose margin is below `band`
// (or a quarter, sixteenth, sixty-fourth of it, the widest that fits kmax),
// written over their la_ref entries.  cb must be on stream s.
int lg_tie_refine(cudaStream_t s, cublasHandle_t cb, const LogisticDev& X, bool f64,
                  const DevParams* dP, const DevState* dS, int64_t T, double* la_ref,
                  const TieBufs& b, float band);
// Accept flags, margins and the recursion defect at the returned trajectory from
// la_ref and the passes' proposals (into acc_col, la_col, max_defect_bits).
cudaError_t lg_verify(cudaStream_t s, bool f64, const DevParams* dP, DevState* dS, int64_t T,
                      const double* la_ref);


// Adjoint of a trajectory objective in epsilon (logistic_adjoint.cu), FP64:
// x0 (D) and S (T x D rows) of the state's type on the device, the tape of
// (seed, block); esjd = 1 for the expected squared jump distance, 0 for the
// mean of |x_t|^2; `scan` runs a diagonal affine scan of T rows of Dp doubles
// on the device (S_t = A_t S_{t-1} + B_t from s0).  Returns 0, 3 (CUDA or
// cuBLAS error), 4 (non-finite) or 5 (the Jacobi iterations did not reach
// 1e-12 within max_iter); *iters gets the iterations run.
typedef int (*ScanFn)(void* ctx, int64_t D, int64_t T, const double* A, const double* B,
                      const double* s0, double* S);
size_t lg_adjoint_ws_bytes(const LogisticDev& X, int64_t T);
int lg_adjoint(cudaStream_t s, cublasHandle_t cb, const LogisticDev& X, bool f64,
               const void* x0, const void* S, uint64_t seed, uint64_t block, int64_t T,
               double eps, int esjd, void* ws, int max_iter, double* grad_eps, int* iters,
               ScanFn scan, void* scan_ctx);

}  // namespace pmcmc
