// logistic.h -- host-side interface of the logistic-regression target.
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>

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
};

int64_t lg_chunk_cols(int64_t N, int64_t T);
int lg_plain_pass(cudaStream_t s, cublasHandle_t cb, const LogisticDev& X, bool f64,
                  const DevParams* dP, const DevState* dS, double* lp, int mode, int64_t T,
                  int64_t Dp, void* Bbuf, void* Lbuf, void* Gbuf, int64_t Tc);

}  // namespace pmcmc
