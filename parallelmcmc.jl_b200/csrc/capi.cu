// capi.cu -- the extern "C" boundary of libpmcmc_deer.so (see include/pmcmc_deer.h).
//
// Host-side runtime: handle (device, stream, workspace, cached CUDA graph),
// device targets, argument validation with the reference's error classes, the
// Newton loop driver and the block loop of the sampler.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pmcmc_deer.h"
#include "deer_device.cuh"
#include "deer_launch.h"
#include "logistic.h"

using namespace pmcmc;

struct GraphKey {
  const void* sweep = nullptr;
  bool coop = false;
  int ntiles = 0, fin_grid = 0, init_grid = 0;
  size_t smem_sweep = 0, smem_fin = 0;
  bool operator==(const GraphKey& o) const {
    return sweep == o.sweep && coop == o.coop && ntiles == o.ntiles && fin_grid == o.fin_grid &&
           init_grid == o.init_grid && smem_sweep == o.smem_sweep && smem_fin == o.smem_fin;
  }
};

struct pmcmc_handle {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  DevParams* d_params = nullptr;
  DevState* d_state = nullptr;
  DevState* h_state = nullptr;  // pinned
  unsigned char* ws = nullptr;
  size_t ws_bytes = 0;
  unsigned char* scan_ws = nullptr;
  size_t scan_ws_bytes = 0;
  uint32_t scan_epoch = 0;
  cudaGraphExec_t gexec = nullptr;
  cudaGraphConditionalHandle cond = 0;
  GraphKey gkey;
  bool force_eager = false;
  bool no_coop = false;
  int tile_override = 0;
  unsigned long long* h_red = nullptr;  // pinned, plain-path metric readback
  cublasHandle_t cublas = nullptr;
  bool profiling = false;
  pmcmc_profile prof{};
  cudaEvent_t ev[2] = {nullptr, nullptr};
};

struct pmcmc_target {
  pmcmc_handle* h = nullptr;
  int kind = 0;
  int64_t D = 0, N = 0, Dp = 0;
  double* mean_d = nullptr;
  double* prec_d = nullptr;
  float* mean_f = nullptr;
  float* prec_f = nullptr;
  LogisticDev lg;
};

namespace {

int fail(pmcmc_handle* h, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (h) h->err = buf;
  return code;
}

#define CK(call)                                                                           \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(h, PMCMC_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                     \
  } while (0)

int64_t round4(int64_t d) { return (d + 3) & ~int64_t(3); }

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int ensure_ws(pmcmc_handle* h, size_t bytes) {
  if (bytes <= h->ws_bytes) return PMCMC_OK;
  if (h->ws) {
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaFree(h->ws));
    h->ws = nullptr;
    h->ws_bytes = 0;
  }
  const size_t want = std::max(bytes, h->ws_bytes * 3 / 2);
  if (cudaMalloc(&h->ws, want) != cudaSuccess) {
    cudaGetLastError();
    return fail(h, PMCMC_ERR_NOMEM, "device workspace allocation of %zu bytes failed", want);
  }
  CK(cudaMemsetAsync(h->ws, 0, want, h->stream));
  h->ws_bytes = want;
  return PMCMC_OK;
}

// Reference argument validation (DEER.jl:387-393, 525-528; interface.jl:273-275).
int validate(pmcmc_handle* h, const pmcmc_target* t, const pmcmc_deer_params* p) {
  if (!p) return fail(h, PMCMC_ERR_ARGUMENT, "params must not be NULL");
  if (!t) return fail(h, PMCMC_ERR_ARGUMENT, "target must not be NULL");
  if (!(p->epsilon > 0) || !std::isfinite(p->epsilon))
    return fail(h, PMCMC_ERR_ARGUMENT, "epsilon must be > 0, got %g", p->epsilon);
  if (p->T < 1) return fail(h, PMCMC_ERR_ARGUMENT, "T must be >= 1, got %lld", (long long)p->T);
  if (p->T > (int64_t(1) << 31) - 1)
    return fail(h, PMCMC_ERR_ARGUMENT, "T must be < 2^31 (counter-based tape)");
  if (p->maxiter < 1) return fail(h, PMCMC_ERR_ARGUMENT, "maxiter must be >= 1");
  if (p->maxiter >= (1 << 20)) return fail(h, PMCMC_ERR_ARGUMENT, "maxiter must be < 2^20");
  if (!(p->tol_abs >= 0)) return fail(h, PMCMC_ERR_ARGUMENT, "tol_abs must be >= 0");
  if (!(p->tol_rel >= 0)) return fail(h, PMCMC_ERR_ARGUMENT, "tol_rel must be >= 0");
  if (!(p->damping > 0 && p->damping <= 1))
    return fail(h, PMCMC_ERR_ARGUMENT, "damping must be in (0,1]");
  if (p->probes < 1) return fail(h, PMCMC_ERR_ARGUMENT, "probes must be >= 1");
  if (p->probes > 255) return fail(h, PMCMC_ERR_ARGUMENT, "probes must be <= 255");
  if (p->jacobian != PMCMC_JAC_STOCH_DIAG && p->jacobian != PMCMC_JAC_DIAG &&
      p->jacobian != PMCMC_JAC_FULL)
    return fail(h, PMCMC_ERR_ARGUMENT, "jacobian must be :stoch_diag, :diag or :full");
  if (p->window < 0) return fail(h, PMCMC_ERR_ARGUMENT, "window must be >= 0");
  if (p->dtype != PMCMC_F32 && p->dtype != PMCMC_F64)
    return fail(h, PMCMC_ERR_ARGUMENT, "dtype must be PMCMC_F32 or PMCMC_F64");
  if (p->exec != PMCMC_EXEC_FUSED && p->exec != PMCMC_EXEC_PLAIN)
    return fail(h, PMCMC_ERR_ARGUMENT, "exec must be PMCMC_EXEC_FUSED or PMCMC_EXEC_PLAIN");
  if (t->h != h) return fail(h, PMCMC_ERR_ARGUMENT, "target belongs to another handle");
  return PMCMC_OK;
}

struct TilePlan {
  int TT = 8;
  bool coop = false;
};

// Smallest tile (most parallelism) whose every CTA is co-resident -> the
// cooperative sweep; otherwise the decoupled look-back sweep with a tile that
// keeps about two CTAs per SM busy.
TilePlan choose_tile(pmcmc_handle* h, const SweepKernels& k, bool f64, int64_t Dp, int64_t W,
                     bool dense) {
  TilePlan tp;
  if (h->tile_override > 0) {
    tp.TT = h->tile_override;
    tp.coop = false;
    return tp;
  }
  if (!h->no_coop && k.sweep_coop) {
    for (int TT = 8; TT <= 256; TT <<= 1) {
      const size_t smem = gauss_sweep_smem(f64, Dp, TT, dense).total;
      if (smem > 200 * 1024) break;
      cudaFuncSetAttribute(k.sweep_coop, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem));
      int nb = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k.sweep_coop, kThreads, smem) !=
          cudaSuccess) {
        cudaGetLastError();
        break;
      }
      if (nb > 0 && (W + TT - 1) / TT <= static_cast<int64_t>(nb) * h->num_sms) {
        tp.TT = TT;
        tp.coop = true;
        return tp;
      }
    }
  }
  int TT = 64;
  while (TT > 8 && gauss_sweep_smem(f64, Dp, TT, dense).total > 100 * 1024) TT >>= 1;
  while (TT > 8 && (W + TT - 1) / TT < 2 * h->num_sms) TT >>= 1;
  tp.TT = TT;
  return tp;
}

cudaError_t launch_sweep(const void* fn, bool coop, int grid, size_t smem, void** args,
                         cudaStream_t s) {
  if (coop)
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, smem, s);
  return cudaLaunchKernel(fn, dim3(grid), dim3(kThreads), args, smem, s);
}

// Workspace carve-up for one solve.
struct SolveLayout {
  size_t S0, S1, x0a, x0b, flags, agg_a, agg_b, incl, colmax, out_S, out_lp, out_acc;
  size_t pA, pB, al0, be0, al1, be1, red;  // plain path only
  size_t lg[5], lpx, lpy, acc_col, la_col, Bb, Lb, Gb;  // logistic only
  size_t xi, logu;
  size_t tcws, Gtc;  // tensor-core logistic path
  size_t total;
};

SolveLayout layout(int64_t D, int64_t Dp, int64_t T, int ntiles, size_t es, bool plain,
                   int64_t N = 0, int64_t Tc = 0, size_t tc_bytes = 0) {
  SolveLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = (off + bytes + 255) & ~size_t(255);
    return o;
  };
  L.S0 = take(es * T * Dp);
  L.S1 = take(es * T * Dp);
  L.x0a = take(es * Dp);
  L.x0b = take(es * Dp);
  L.flags = take(4 * static_cast<size_t>(ntiles));
  L.agg_a = take(es * ntiles * Dp);
  L.agg_b = take(es * ntiles * Dp);
  L.incl = take(es * ntiles * Dp);
  L.colmax = take(4 * static_cast<size_t>(T));
  L.out_S = take(es * T * D);
  L.out_lp = take(es * T);
  L.out_acc = take(static_cast<size_t>(T));
  L.xi = take(4 * T * Dp);
  L.logu = take(8 * static_cast<size_t>(T));
  if (plain) {
    L.pA = take(es * T * Dp);
    L.pB = take(es * T * Dp);
    L.al0 = take(es * T * Dp);
    L.be0 = take(es * T * Dp);
    L.al1 = take(es * T * Dp);
    L.be1 = take(es * T * Dp);
    L.red = take(4 * sizeof(unsigned long long));
  }
  if (N > 0) {
    for (int i = 0; i < 5; ++i) L.lg[i] = take(es * T * Dp);
    L.lpx = take(8 * static_cast<size_t>(T));
    L.lpy = take(8 * static_cast<size_t>(T));
    L.acc_col = take(static_cast<size_t>(T));
    L.la_col = take(8 * static_cast<size_t>(T));
    L.Bb = take(es * Dp * 2 * Tc);
    L.Lb = take(es * N * 2 * Tc);
    L.Gb = take(es * Dp * 2 * Tc);
  }
  if (tc_bytes) {
    L.tcws = take(tc_bytes);
    L.Gtc = take(4 * Dp * 2 * static_cast<size_t>(T));
  }
  L.total = off;
  return L;
}

int build_graph(pmcmc_handle* h, const SweepKernels& k, const GraphKey& key, int init_grid) {
  if (h->gexec && h->gkey == key) return PMCMC_OK;
  if (h->gexec) {
    cudaGraphExecDestroy(h->gexec);
    h->gexec = nullptr;
  }
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle cond = 0;
  cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(h, PMCMC_ERR_CUDA, "cudaGraphConditionalHandleCreate: %s", cudaGetErrorString(e));
  }
  h->cond = cond;
  int one = 1;
  void* init_args[] = {&h->d_params, &h->d_state};
  void* sweep_args[] = {&h->d_params, &h->d_state, &h->cond, &one};
  void* fin_args[] = {&h->d_params, &h->d_state};

  cudaKernelNodeParams kp{};
  kp.func = const_cast<void*>(k.init);
  kp.gridDim = dim3(init_grid);
  kp.blockDim = dim3(256);
  kp.sharedMemBytes = 0;
  kp.kernelParams = init_args;
  cudaGraphNode_t n_init, n_while, n_sweep, n_fin;
  e = cudaGraphAddKernelNode(&n_init, g, nullptr, 0, &kp);
  cudaGraphNodeParams cp{};
  if (e == cudaSuccess) {
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&n_while, g, &n_init, 1, &cp);
  }
  if (e == cudaSuccess) {
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaKernelNodeParams sp{};
    sp.func = const_cast<void*>(key.sweep);
    sp.gridDim = dim3(key.ntiles);
    sp.blockDim = dim3(kThreads);
    sp.sharedMemBytes = static_cast<unsigned>(key.smem_sweep);
    sp.kernelParams = sweep_args;
    e = cudaGraphAddKernelNode(&n_sweep, body, nullptr, 0, &sp);
    if (e == cudaSuccess && key.coop) {
      cudaLaunchAttributeValue v{};
      v.cooperative = 1;
      e = cudaGraphKernelNodeSetAttribute(n_sweep, cudaLaunchAttributeCooperative, &v);
    }
  }
  if (e == cudaSuccess) {
    cudaKernelNodeParams fp{};
    fp.func = const_cast<void*>(k.finalize);
    fp.gridDim = dim3(key.fin_grid);
    fp.blockDim = dim3(kThreads);
    fp.sharedMemBytes = static_cast<unsigned>(key.smem_fin);
    fp.kernelParams = fin_args;
    e = cudaGraphAddKernelNode(&n_fin, g, &n_while, 1, &fp);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&h->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->gexec = nullptr;
    return fail(h, PMCMC_ERR_CUDA, "CUDA graph construction failed: %s", cudaGetErrorString(e));
  }
  h->gkey = key;
  return PMCMC_OK;
}

// One DEER block on the fused path.  Outputs go to the pointers in `P`
// (already filled by the caller); the state of the solve stays in d_state.
int run_fused(pmcmc_handle* h, const SweepKernels& k, bool coop, const DevParams& P,
              size_t smem_sweep, size_t smem_fin, int fin_grid, int init_grid) {
  const void* sweep_fn = coop ? k.sweep_coop : k.sweep;
  CK(cudaMemcpyAsync(h->d_params, &P, sizeof(DevParams), cudaMemcpyHostToDevice, h->stream));
  if (smem_sweep > 48 * 1024)
    CK(cudaFuncSetAttribute(sweep_fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(smem_sweep)));
  if (smem_fin > 48 * 1024)
    CK(cudaFuncSetAttribute(k.finalize, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(smem_fin)));
  if (!h->force_eager && !h->profiling) {
    GraphKey key;
    key.sweep = sweep_fn;
    key.coop = coop;
    key.ntiles = P.ntiles;
    key.fin_grid = fin_grid;
    key.init_grid = init_grid;
    key.smem_sweep = smem_sweep;
    key.smem_fin = smem_fin;
    const int rc = build_graph(h, k, key, init_grid);
    if (rc == PMCMC_OK) {
      CK(cudaGraphLaunch(h->gexec, h->stream));
      return PMCMC_OK;
    }
    // fall through to the eager loop if graphs with conditional nodes are unavailable
    h->force_eager = true;
  }
  void* init_args[] = {&h->d_params, &h->d_state};
  CK(cudaLaunchKernel(k.init, dim3(init_grid), dim3(256), init_args, 0, h->stream));
  cudaGraphConditionalHandle none = 0;
  int zero = 0;
  void* sweep_args[] = {&h->d_params, &h->d_state, &none, &zero};
  for (int it = 0; it < P.maxiter; ++it) {
    if (h->profiling) CK(cudaEventRecord(h->ev[0], h->stream));
    CK(launch_sweep(sweep_fn, coop, P.ntiles, smem_sweep, sweep_args, h->stream));
    if (h->profiling) {
      // one sweep at a time so that only real sweeps are timed
      CK(cudaEventRecord(h->ev[1], h->stream));
      CK(cudaMemcpyAsync(h->h_state, h->d_state, sizeof(DevState), cudaMemcpyDeviceToHost,
                         h->stream));
      CK(cudaStreamSynchronize(h->stream));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
      h->prof.sweep_launches += 1;
      h->prof.sweep_ms += ms;
      if (h->h_state->converged || h->h_state->status) break;
      continue;
    }
    if ((it & 7) == 7 || it + 1 == P.maxiter) {
      CK(cudaMemcpyAsync(h->h_state, h->d_state, sizeof(DevState), cudaMemcpyDeviceToHost,
                         h->stream));
      CK(cudaStreamSynchronize(h->stream));
      if (h->h_state->converged || h->h_state->status) break;
    }
  }
  void* fin_args[] = {&h->d_params, &h->d_state};
  if (h->profiling) CK(cudaEventRecord(h->ev[0], h->stream));
  CK(cudaLaunchKernel(k.finalize, dim3(fin_grid), dim3(kThreads), fin_args, smem_fin,
                      h->stream));
  if (h->profiling) {
    CK(cudaEventRecord(h->ev[1], h->stream));
    CK(cudaEventSynchronize(h->ev[1]));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
    h->prof.finalize_launches += 1;
    h->prof.finalize_ms += ms;
  }
  return PMCMC_OK;
}

// One DEER block on the plain path: unfused evaluate -> doubling scan ->
// damping/metric, with the convergence test on the host after every
// iteration (two reductions read back, as DEER.jl:567-570 does).
int run_plain(pmcmc_handle* h, const SweepKernels& k, const DevParams& P, const SolveLayout& L,
              size_t es, size_t smem_fin, int fin_grid, int init_grid) {
  unsigned char* ws = h->ws;
  const bool f64 = es == 8;
  CK(cudaMemcpyAsync(h->d_params, &P, sizeof(DevParams), cudaMemcpyHostToDevice, h->stream));
  if (smem_fin > 48 * 1024) {
    CK(cudaFuncSetAttribute(k.finalize, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(smem_fin)));
    CK(cudaFuncSetAttribute(k.eval, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(smem_fin)));
  }
  void* init_args[] = {&h->d_params, &h->d_state};
  CK(cudaLaunchKernel(k.init, dim3(init_grid), dim3(256), init_args, 0, h->stream));
  CK(launch_broadcast(h->stream, f64, P.Dp, P.T, P.x0, P.S[0]));
  void* A = ws + L.pA;
  void* B = ws + L.pB;
  int cur = 0, iters = 0, converged = 0, status = 0;
  double metric = INFINITY;
  for (int it = 0; it < P.maxiter; ++it) {
    iters = it + 1;
    const void* Sold = P.S[cur];
    void* Snew = P.S[cur ^ 1];
    int from_x0 = 0;
    void* eval_args[] = {&h->d_params, const_cast<void**>(&Sold), &it, &from_x0, &A, &B};
    CK(cudaLaunchKernel(k.eval, dim3(fin_grid), dim3(kThreads), eval_args, smem_fin, h->stream));
    CK(launch_doubling_scan(h->stream, f64, P.Dp, P.T, A, B, P.x0, Snew, ws + L.al0,
                            ws + L.be0, ws + L.al1, ws + L.be1));
    auto* red = reinterpret_cast<unsigned long long*>(ws + L.red);
    CK(launch_damp_metric(h->stream, f64, P.D, P.Dp, P.T, Sold, Snew, P.damping, red));
    CK(cudaMemcpyAsync(h->h_red, red, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double dmax, smax;
    std::memcpy(&dmax, &h->h_red[0], 8);
    std::memcpy(&smax, &h->h_red[1], 8);
    metric = dmax / (P.tol_abs + P.tol_rel * smax);
    cur ^= 1;
    if (h->h_red[2]) {
      status = kStNonfinite;
      break;
    }
    if (metric <= 1) {
      converged = 1;
      break;
    }
  }
  CK(cudaMemcpyAsync(h->h_state, h->d_state, sizeof(DevState), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  DevState st = *h->h_state;
  st.cur = cur;
  st.iter = iters;
  st.converged = converged;
  st.metric = metric;
  st.status = status;
  *h->h_state = st;
  CK(cudaMemcpyAsync(h->d_state, h->h_state, sizeof(DevState), cudaMemcpyHostToDevice,
                     h->stream));
  void* fin_args[] = {&h->d_params, &h->d_state};
  CK(cudaLaunchKernel(k.finalize, dim3(fin_grid), dim3(kThreads), fin_args, smem_fin,
                      h->stream));
  return PMCMC_OK;
}

// One DEER block for the logistic target: per Newton iteration two GEMM
// passes (pass 1 at [x_bar | z], pass 2 at [y | w]) feed the fused
// finish + scan sweep kernel; then a logp pass over the returned trajectory.
int run_logistic(pmcmc_handle* h, const pmcmc_target* tg, const SweepKernels& k, bool coop,
                 const DevParams& P, const SolveLayout& L, size_t es, size_t smem_sweep,
                 int fin_grid, int init_grid, int64_t Tc, bool use_tc) {
  unsigned char* ws = h->ws;
  const bool f64 = es == 8;
  CK(cudaMemcpyAsync(h->d_params, &P, sizeof(DevParams), cudaMemcpyHostToDevice, h->stream));
  if (smem_sweep > 48 * 1024)
    CK(cudaFuncSetAttribute(coop ? k.sweep_coop : k.sweep,
                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(smem_sweep)));
  if (!h->cublas) {
    if (cublasCreate(&h->cublas) != CUBLAS_STATUS_SUCCESS)
      return fail(h, PMCMC_ERR_CUDA, "cublasCreate failed");
    cublasSetMathMode(h->cublas, CUBLAS_PEDANTIC_MATH);
  }
  cublasSetStream(h->cublas, h->stream);
  void* init_args[] = {&h->d_params, &h->d_state};
  CK(cudaLaunchKernel(k.init, dim3(init_grid), dim3(256), init_args, 0, h->stream));
  cudaGraphConditionalHandle none = 0;
  int zero = 0;
  void* sweep_args[] = {&h->d_params, &h->d_state, &none, &zero};
  void *Bb = ws + L.Bb, *Lb = ws + L.Lb, *Gb = ws + L.Gb;
  int* tc_err = use_tc ? lg_tc_err_word(ws + L.tcws, tg->lg, P.T) : nullptr;
  if (use_tc) CK(cudaMemsetAsync(tc_err, 0, sizeof(int), h->stream));
  auto pass = [&](int mode, double* lp) -> int {
    if (use_tc) {
      float* G = reinterpret_cast<float*>(ws + L.Gtc);
      if (lg_tc_pass(h->stream, tg->lg, h->d_params, h->d_state, lp, mode, P.T, ws + L.tcws, G))
        return 1;
      if (mode != 2 && lg_mid(h->stream, false, h->d_params, h->d_state, mode + 1, 0,
                              static_cast<int>(P.T), P.Dp, G) != cudaSuccess)
        return 1;
      return 0;
    }
    return lg_plain_pass(h->stream, h->cublas, tg->lg, f64, h->d_params, h->d_state, lp, mode,
                         P.T, P.Dp, Bb, Lb, Gb, Tc);
  };
  for (int it = 0; it < P.maxiter; ++it) {
    if (pass(0, P.lpx))
      return fail(h, PMCMC_ERR_CUDA, "logistic pass 1 failed: %s",
                  cudaGetErrorString(cudaGetLastError()));
    if (pass(1, P.lpy))
      return fail(h, PMCMC_ERR_CUDA, "logistic pass 2 failed: %s",
                  cudaGetErrorString(cudaGetLastError()));
    if (h->profiling) CK(cudaEventRecord(h->ev[0], h->stream));
    CK(launch_sweep(coop ? k.sweep_coop : k.sweep, coop, P.ntiles, smem_sweep, sweep_args,
                    h->stream));
    if (h->profiling) CK(cudaEventRecord(h->ev[1], h->stream));
    CK(cudaMemcpyAsync(h->h_state, h->d_state, sizeof(DevState), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (h->profiling) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
      h->prof.sweep_launches += 1;
      h->prof.sweep_ms += ms;
    }
    if (h->h_state->converged || h->h_state->status) break;
  }
  if (pass(2, P.lpx)) return fail(h, PMCMC_ERR_CUDA, "logistic logp pass failed");
  void* fin_args[] = {&h->d_params, &h->d_state};
  CK(cudaLaunchKernel(k.finalize, dim3(fin_grid), dim3(kThreads), fin_args, 0, h->stream));
  if (use_tc) {
    int e = 0;
    CK(cudaMemcpyAsync(&e, tc_err, sizeof e, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (e) return fail(h, PMCMC_ERR_TIMEOUT, "tensor-core pass: a bounded wait gave up");
  }
  return PMCMC_OK;
}

void fill_info(const DevState& s, pmcmc_info* info) {
  if (!info) return;
  info->iters = s.iter;
  info->converged = s.converged;
  info->metric = s.metric;
  info->n_accept = static_cast<int64_t>(s.n_accept);
  double mm, md;
  std::memcpy(&mm, &s.min_margin_bits, 8);
  std::memcpy(&md, &s.max_defect_bits, 8);
  info->min_margin = mm;
  info->max_defect = md;
  info->status = s.status;
}

int status_error(pmcmc_handle* h, int status) {
  if (status == kStTimeout)
    return fail(h, PMCMC_ERR_TIMEOUT, "device look-back wait exceeded its bound");
  if (status == kStNonfinite)
    return fail(h, PMCMC_ERR_NONFINITE, "non-finite value in the DEER trajectory");
  return PMCMC_OK;
}

// Shared implementation of pmcmc_deer_solve (nblocks = 1, N = T) and
// pmcmc_sample (block loop of interface.jl:584-599).
int solve_blocks(pmcmc_handle* h, const pmcmc_target* tg, const pmcmc_deer_params* p,
                 const void* x0, uint64_t seed, uint64_t block0, int64_t N, void* S_out,
                 void* logp_out, uint8_t* accept_out, int32_t mem, pmcmc_info* info) {
  int rc = validate(h, tg, p);
  if (rc) return rc;
  if (!x0 || !S_out) return fail(h, PMCMC_ERR_ARGUMENT, "x0 and the output must not be NULL");
  if (mem != PMCMC_MEM_HOST && mem != PMCMC_MEM_DEVICE)
    return fail(h, PMCMC_ERR_ARGUMENT, "mem must be PMCMC_MEM_HOST or PMCMC_MEM_DEVICE");
  if (N < 1) return fail(h, PMCMC_ERR_ARGUMENT, "the number of samples must be >= 1");
  if (tg->kind == kLogistic) {
    if (p->jacobian != PMCMC_JAC_STOCH_DIAG)
      return fail(h, PMCMC_ERR_UNSUPPORTED, "logistic target: only :stoch_diag is built");
    if (p->probes != 1)
      return fail(h, PMCMC_ERR_UNSUPPORTED, "logistic target: probes must be 1");
    if (p->window > 0 && p->window < p->T)
      return fail(h, PMCMC_ERR_UNSUPPORTED, "logistic target: no sliding window");
  }
  if (p->jacobian == PMCMC_JAC_FULL)
    return fail(h, PMCMC_ERR_UNSUPPORTED, ":full jacobian is not built into this library yet");
  DeviceGuard guard(h->device);
  const bool f64 = p->dtype == PMCMC_F64;
  const size_t es = f64 ? 8 : 4;
  const int64_t D = tg->D, Dp = tg->Dp, T = p->T;
  const int64_t W = (p->window > 0 && p->window < T) ? p->window : T;
  const bool dense = tg->kind == kDenseGauss;

  const bool plain = p->exec == PMCMC_EXEC_PLAIN;
  if (plain && W < T)
    return fail(h, PMCMC_ERR_UNSUPPORTED, "the plain path has no sliding window");
  const bool logistic = tg->kind == kLogistic;
  const SweepKernels k = logistic ? logistic_sweep_kernels(f64, D)
                                  : gauss_sweep_kernels(f64, tg->kind, p->jacobian, D);
  const TilePlan tp = choose_tile(h, k, f64, Dp, W, dense);
  const int TT = tp.TT;
  const int ntiles = static_cast<int>((W + TT - 1) / TT);
  const SmemPlan sp_sweep = gauss_sweep_smem(f64, Dp, TT, dense);
  const SmemPlan sp_fin = gauss_sweep_smem(f64, Dp, 1, dense);
  if (sp_sweep.total > 200 * 1024)
    return fail(h, PMCMC_ERR_UNSUPPORTED, "dimension %lld too large for the fused sweep",
                (long long)D);
  const bool use_tc = logistic && !plain && !f64 && lg_tc_supported(tg->lg);
  const int64_t Tc = logistic && !use_tc ? std::min<int64_t>(T, lg_chunk_cols(tg->N, T)) : 0;
  const SolveLayout L = layout(D, Dp, T, ntiles, es, plain, logistic ? tg->N : 0, Tc,
                               use_tc ? lg_tc_ws_bytes(tg->lg, T) : 0);
  rc = ensure_ws(h, L.total);
  if (rc) return rc;
  unsigned char* ws = h->ws;

  // x0 -> padded device buffer
  CK(cudaMemsetAsync(ws + L.x0a, 0, es * Dp, h->stream));
  CK(cudaMemsetAsync(ws + L.x0b, 0, es * Dp, h->stream));
  CK(cudaMemcpyAsync(ws + L.x0a, x0, es * D,
                     mem == PMCMC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     h->stream));

  DevParams P{};
  P.D = D;
  P.Dp = Dp;
  P.T = T;
  P.W = W;
  P.eps = p->epsilon;
  P.sqrt2eps = std::sqrt(2 * p->epsilon);
  P.inv4eps = 1.0 / (4 * p->epsilon);
  P.inv2eps = 1.0 / (2 * p->epsilon);
  P.damping = p->damping;
  P.tol_abs = p->tol_abs;
  P.tol_rel = p->tol_rel;
  P.seed = seed;
  P.jac = p->jacobian;
  P.probes = p->probes;
  P.maxiter = p->maxiter;
  P.tile_cols = TT;
  P.ntiles = ntiles;
  P.tkind = tg->kind;
  P.out_device = mem == PMCMC_MEM_DEVICE;
  P.mean_d = tg->mean_d;
  P.prec_d = tg->prec_d;
  P.mean_f = tg->mean_f;
  P.prec_f = tg->prec_f;
  P.S[0] = ws + L.S0;
  P.S[1] = ws + L.S1;
  P.flags = reinterpret_cast<uint32_t*>(ws + L.flags);
  P.agg_a = ws + L.agg_a;
  P.agg_b = ws + L.agg_b;
  P.incl = ws + L.incl;
  P.colmax = reinterpret_cast<float*>(ws + L.colmax);
  P.xi = reinterpret_cast<float*>(ws + L.xi);
  P.logu = reinterpret_cast<double*>(ws + L.logu);
  if (logistic) {
    for (int i = 0; i < 5; ++i) P.lg[i] = ws + L.lg[i];
    P.lpx = reinterpret_cast<double*>(ws + L.lpx);
    P.lpy = reinterpret_cast<double*>(ws + L.lpy);
    P.acc_col = ws + L.acc_col;
    P.la_col = reinterpret_cast<double*>(ws + L.la_col);
    P.tau = tg->lg.tau;
  }

  const int fin_grid = static_cast<int>(std::min<int64_t>((T + kWarps - 1) / kWarps,
                                                          int64_t(h->num_sms) * 8));
  const int init_grid = static_cast<int>(
      std::min<int64_t>((T * (Dp / 4) + 255) / 256, int64_t(h->num_sms) * 8));
  const int64_t nblocks = (N + T - 1) / T;
  std::vector<DevState> states(static_cast<size_t>(nblocks));
  int64_t nsteps = 0;
  for (int64_t b = 0; b < nblocks; ++b) {
    const int64_t nkeep = std::min<int64_t>(T, N - nsteps);
    P.block = block0 + static_cast<uint64_t>(b);
    P.x0 = ws + ((b & 1) ? L.x0b : L.x0a);
    P.x_next = ws + ((b & 1) ? L.x0a : L.x0b);
    P.ncols_out = nkeep;
    if (mem == PMCMC_MEM_DEVICE) {
      P.S_out = static_cast<unsigned char*>(S_out) + es * nsteps * D;
      P.logp_out = logp_out ? static_cast<unsigned char*>(logp_out) + es * nsteps : nullptr;
      P.accept_out = accept_out ? accept_out + nsteps : nullptr;
    } else {
      P.S_out = ws + L.out_S;
      P.logp_out = logp_out ? ws + L.out_lp : nullptr;
      P.accept_out = accept_out ? ws + L.out_acc : nullptr;
    }
    rc = logistic ? run_logistic(h, tg, k, tp.coop, P, L, es, sp_sweep.total, fin_grid,
                                 init_grid, Tc, use_tc)
         : plain  ? run_plain(h, k, P, L, es, sp_fin.total, fin_grid, init_grid)
                  : run_fused(h, k, tp.coop, P, sp_sweep.total, sp_fin.total, fin_grid,
                              init_grid);
    if (rc) return rc;
    if (mem == PMCMC_MEM_HOST) {
      CK(cudaMemcpyAsync(static_cast<unsigned char*>(S_out) + es * nsteps * D, ws + L.out_S,
                         es * nkeep * D, cudaMemcpyDeviceToHost, h->stream));
      if (logp_out)
        CK(cudaMemcpyAsync(static_cast<unsigned char*>(logp_out) + es * nsteps, ws + L.out_lp,
                           es * nkeep, cudaMemcpyDeviceToHost, h->stream));
      if (accept_out)
        CK(cudaMemcpyAsync(accept_out + nsteps, ws + L.out_acc, nkeep, cudaMemcpyDeviceToHost,
                           h->stream));
    }
    CK(cudaMemcpyAsync(h->h_state, h->d_state, sizeof(DevState), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    states[static_cast<size_t>(b)] = *h->h_state;
    nsteps += nkeep;
    if (h->h_state->status) break;
  }
  // aggregate
  pmcmc_info agg{};
  agg.converged = 1;
  agg.min_margin = INFINITY;
  int status = 0;
  for (const DevState& s : states) {
    pmcmc_info bi{};
    fill_info(s, &bi);
    agg.iters += bi.iters;
    agg.converged &= bi.converged;
    agg.metric = std::isnan(bi.metric) ? bi.metric : std::max(agg.metric, bi.metric);
    agg.n_accept += bi.n_accept;
    agg.min_margin = std::min(agg.min_margin, bi.min_margin);
    agg.max_defect = std::max(agg.max_defect, bi.max_defect);
    if (bi.status && !status) status = bi.status;
  }
  agg.status = status;
  if (nblocks == 1) fill_info(states[0], &agg);
  agg.path = (plain ? 0 : PMCMC_PATH_FUSED_SWEEP) | (tp.coop && !plain ? PMCMC_PATH_COOPERATIVE : 0) |
             (!plain && !logistic && !h->force_eager && !h->profiling ? PMCMC_PATH_GRAPH : 0) |
             (use_tc ? PMCMC_PATH_TENSOR_CORE : 0);
  if (info) *info = agg;
  return status_error(h, status);
}

int make_target(pmcmc_handle* h, int kind, int64_t D, const double* mean, const double* prec,
                pmcmc_target** out) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  if (!out) return fail(h, PMCMC_ERR_ARGUMENT, "out must not be NULL");
  if (D < 1) return fail(h, PMCMC_ERR_ARGUMENT, "dimension must be >= 1");
  if (!prec) return fail(h, PMCMC_ERR_ARGUMENT, "precision must not be NULL");
  DeviceGuard guard(h->device);
  auto* t = new pmcmc_target();
  t->h = h;
  t->kind = kind;
  t->D = D;
  t->Dp = round4(D);
  const int64_t Dp = t->Dp;
  const int64_t np = kind == kDenseGauss ? Dp * Dp : Dp;
  std::vector<double> md(static_cast<size_t>(Dp), 0.0), pd(static_cast<size_t>(np), 0.0);
  if (mean)
    for (int64_t i = 0; i < D; ++i) md[i] = mean[i];
  if (kind == kDenseGauss) {
    for (int64_t j = 0; j < D; ++j)
      for (int64_t i = 0; i < D; ++i) pd[j * Dp + i] = prec[j * D + i];
  } else {
    for (int64_t i = 0; i < D; ++i) pd[i] = prec[i];
  }
  std::vector<float> mf(md.begin(), md.end()), pf(pd.begin(), pd.end());
  auto cleanup = [&]() {
    cudaFree(t->mean_d);
    cudaFree(t->prec_d);
    cudaFree(t->mean_f);
    cudaFree(t->prec_f);
    delete t;
  };
  if (cudaMalloc(&t->mean_d, 8 * Dp) != cudaSuccess || cudaMalloc(&t->prec_d, 8 * np) != cudaSuccess ||
      cudaMalloc(&t->mean_f, 4 * Dp) != cudaSuccess || cudaMalloc(&t->prec_f, 4 * np) != cudaSuccess) {
    cudaGetLastError();
    cleanup();
    return fail(h, PMCMC_ERR_NOMEM, "target allocation failed");
  }
  cudaError_t e = cudaMemcpy(t->mean_d, md.data(), 8 * Dp, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->prec_d, pd.data(), 8 * np, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->mean_f, mf.data(), 4 * Dp, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->prec_f, pf.data(), 4 * np, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cleanup();
    return fail(h, PMCMC_ERR_CUDA, "target upload failed: %s", cudaGetErrorString(e));
  }
  *out = t;
  return PMCMC_OK;
}

}  // namespace

extern "C" {

int pmcmc_abi_version(void) { return PMCMC_ABI_VERSION; }

int pmcmc_create(int device, void* stream, pmcmc_handle** out) {
  if (!out) return PMCMC_ERR_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return PMCMC_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return PMCMC_ERR_ARGUMENT;
  auto* h = new pmcmc_handle();
  h->device = device;
  DeviceGuard guard(device);
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (stream) {
    h->stream = static_cast<cudaStream_t>(stream);
  } else {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete h;
      return PMCMC_ERR_CUDA;
    }
    h->own_stream = true;
  }
  if (cudaMalloc(&h->d_params, sizeof(DevParams)) != cudaSuccess ||
      cudaMalloc(&h->d_state, sizeof(DevState)) != cudaSuccess ||
      cudaMallocHost(&h->h_state, sizeof(DevState)) != cudaSuccess ||
      cudaMallocHost(&h->h_red, 4 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    pmcmc_destroy(h);
    return PMCMC_ERR_NOMEM;
  }
  cudaMemset(h->d_state, 0, sizeof(DevState));
  cudaMemset(h->d_params, 0, sizeof(DevParams));
  const char* ev = std::getenv("PMCMC_EAGER");
  h->force_eager = ev && ev[0] == '1';
  const char* cv = std::getenv("PMCMC_NO_COOP");
  h->no_coop = cv && cv[0] == '1';
  const char* tv = std::getenv("PMCMC_TILE_COLS");
  h->tile_override = tv ? std::atoi(tv) : 0;
  if (cudaDeviceSynchronize() != cudaSuccess) {
    cudaGetLastError();
    pmcmc_destroy(h);
    return PMCMC_ERR_CUDA;
  }
  *out = h;
  return PMCMC_OK;
}

int pmcmc_destroy(pmcmc_handle* h) {
  if (!h) return PMCMC_OK;
  DeviceGuard guard(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->cublas) cublasDestroy(h->cublas);
  cudaFree(h->ws);
  cudaFree(h->scan_ws);
  cudaFree(h->d_params);
  cudaFree(h->d_state);
  if (h->h_state) cudaFreeHost(h->h_state);
  if (h->h_red) cudaFreeHost(h->h_red);
  for (cudaEvent_t e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return PMCMC_OK;
}

const char* pmcmc_last_error(const pmcmc_handle* h) { return h ? h->err.c_str() : "null handle"; }

int pmcmc_set_profiling(pmcmc_handle* h, int32_t on) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  DeviceGuard guard(h->device);
  if (on && !h->ev[0]) {
    CK(cudaEventCreate(&h->ev[0]));
    CK(cudaEventCreate(&h->ev[1]));
  }
  h->profiling = on != 0;
  return PMCMC_OK;
}

int pmcmc_get_profile(pmcmc_handle* h, pmcmc_profile* out, int32_t reset) {
  if (!h || !out) return PMCMC_ERR_ARGUMENT;
  *out = h->prof;
  if (reset) h->prof = pmcmc_profile{};
  return PMCMC_OK;
}

int pmcmc_target_diag_gauss(pmcmc_handle* h, int64_t D, const double* mean, const double* prec,
                            pmcmc_target** out) {
  return make_target(h, kDiagGauss, D, mean, prec, out);
}

int pmcmc_target_dense_gauss(pmcmc_handle* h, int64_t D, const double* mean, const double* prec,
                             pmcmc_target** out) {
  return make_target(h, kDenseGauss, D, mean, prec, out);
}

int pmcmc_target_logistic(pmcmc_handle* h, int64_t N, int64_t D, const double* X,
                          const double* y, double prior_prec, pmcmc_target** out) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  if (!out || !X || !y) return fail(h, PMCMC_ERR_ARGUMENT, "null argument");
  if (N < 1 || D < 1) return fail(h, PMCMC_ERR_ARGUMENT, "N and D must be >= 1");
  if (!(prior_prec > 0)) return fail(h, PMCMC_ERR_ARGUMENT, "prior_prec must be > 0");
  for (int64_t n = 0; n < N; ++n)
    if (!(y[n] == 0.0 || y[n] == 1.0)) return fail(h, PMCMC_ERR_ARGUMENT, "labels must be 0 or 1");
  DeviceGuard guard(h->device);
  auto* t = new pmcmc_target();
  t->h = h;
  t->kind = kLogistic;
  t->D = D;
  t->N = N;
  t->Dp = round4(D);
  const int64_t Dp = t->Dp;
  t->lg.N = N;
  t->lg.D = D;
  t->lg.Dp = Dp;
  t->lg.tau = prior_prec;
  std::vector<double> x64(static_cast<size_t>(N * Dp), 0.0);
  for (int64_t i = 0; i < D; ++i)
    for (int64_t n = 0; n < N; ++n) x64[n * Dp + i] = X[i * N + n];
  std::vector<float> x32(x64.begin(), x64.end());
  std::vector<float> y32(y, y + N);
  cudaError_t e = cudaMalloc(&t->lg.X64, 8 * N * Dp);
  if (e == cudaSuccess) e = cudaMalloc(&t->lg.X32, 4 * N * Dp);
  if (e == cudaSuccess) e = cudaMalloc(&t->lg.y64, 8 * N);
  if (e == cudaSuccess) e = cudaMalloc(&t->lg.y32, 4 * N);
  if (e == cudaSuccess) e = cudaMemcpy(t->lg.X64, x64.data(), 8 * N * Dp, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->lg.X32, x32.data(), 4 * N * Dp, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->lg.y64, y, 8 * N, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->lg.y32, y32.data(), 4 * N, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && D <= 256) {
    // FP16 hi + lo operands for the tensor-core pass
    const int64_t Dk = D <= 128 ? 128 : 256;
    const int64_t Np = (N + 127) / 128 * 128;
    std::vector<__half> xh(static_cast<size_t>(Np * Dk), __float2half(0.f)), xl(xh);
    for (int64_t n = 0; n < N; ++n)
      for (int64_t i = 0; i < D; ++i) {
        const float v = static_cast<float>(X[i * N + n]);
        const __half hi = __float2half_rn(v);
        xh[n * Dk + i] = hi;
        xl[n * Dk + i] = __float2half_rn(v - __half2float(hi));
      }
    t->lg.Np = Np;
    t->lg.Dk = Dk;
    e = cudaMalloc(&t->lg.Xh, 2 * Np * Dk);
    if (e == cudaSuccess) e = cudaMalloc(&t->lg.Xl, 2 * Np * Dk);
    if (e == cudaSuccess) e = cudaMemcpy(t->lg.Xh, xh.data(), 2 * Np * Dk, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t->lg.Xl, xl.data(), 2 * Np * Dk, cudaMemcpyHostToDevice);
    // labels padded to Np for the tensor-core epilogue
    if (e == cudaSuccess) {
      float* y32p = nullptr;
      e = cudaMalloc(&y32p, 4 * Np);
      if (e == cudaSuccess) e = cudaMemset(y32p, 0, 4 * Np);
      if (e == cudaSuccess) e = cudaMemcpy(y32p, y32.data(), 4 * N, cudaMemcpyHostToDevice);
      if (e == cudaSuccess) {
        cudaFree(t->lg.y32);
        t->lg.y32 = y32p;
      }
    }
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    pmcmc_target_destroy(t);
    return fail(h, PMCMC_ERR_NOMEM, "logistic target upload failed: %s", cudaGetErrorString(e));
  }
  *out = t;
  return PMCMC_OK;
}

int pmcmc_target_destroy(pmcmc_target* t) {
  if (!t) return PMCMC_OK;
  DeviceGuard guard(t->h->device);
  cudaFree(t->mean_d);
  cudaFree(t->prec_d);
  cudaFree(t->mean_f);
  cudaFree(t->prec_f);
  cudaFree(t->lg.X32);
  cudaFree(t->lg.X64);
  cudaFree(t->lg.y32);
  cudaFree(t->lg.y64);
  cudaFree(t->lg.Xh);
  cudaFree(t->lg.Xl);
  delete t;
  return PMCMC_OK;
}

int pmcmc_tape(pmcmc_handle* h, int64_t D, int64_t T, uint64_t seed, uint64_t block, float* Xi,
               float* u, int32_t mem) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  if (D < 1 || T < 0) return fail(h, PMCMC_ERR_ARGUMENT, "D must be >= 1 and T >= 0");
  if (!Xi) return fail(h, PMCMC_ERR_ARGUMENT, "Xi must not be NULL");
  if (T == 0) return PMCMC_OK;
  DeviceGuard guard(h->device);
  if (mem == PMCMC_MEM_DEVICE) {
    CK(launch_tape(h->stream, D, T, seed, block, Xi, u));
    CK(cudaStreamSynchronize(h->stream));
    return PMCMC_OK;
  }
  const size_t bytes = 4 * static_cast<size_t>(D * T + T);
  int rc = ensure_ws(h, bytes + 256);
  if (rc) return rc;
  float* dXi = reinterpret_cast<float*>(h->ws);
  float* du = dXi + D * T;
  CK(launch_tape(h->stream, D, T, seed, block, dXi, du));
  CK(cudaMemcpyAsync(Xi, dXi, 4 * D * T, cudaMemcpyDeviceToHost, h->stream));
  if (u) CK(cudaMemcpyAsync(u, du, 4 * T, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PMCMC_OK;
}

int pmcmc_deer_solve(pmcmc_handle* h, const pmcmc_target* t, const pmcmc_deer_params* p,
                     const void* x0, uint64_t seed, uint64_t block, void* S_out, void* logp_out,
                     uint8_t* accept_out, int32_t mem, pmcmc_info* info) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  if (!p) return fail(h, PMCMC_ERR_ARGUMENT, "params must not be NULL");
  return solve_blocks(h, t, p, x0, seed, block, p->T, S_out, logp_out, accept_out, mem, info);
}

int pmcmc_sample(pmcmc_handle* h, const pmcmc_target* t, const pmcmc_deer_params* p,
                 const void* x0, uint64_t seed, int64_t N, void* vals_out, void* logp_out,
                 uint8_t* accept_out, int32_t mem, pmcmc_info* info) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  return solve_blocks(h, t, p, x0, seed, 0, N, vals_out, logp_out, accept_out, mem, info);
}

int pmcmc_affine_scan_diag(pmcmc_handle* h, int32_t dtype, int64_t D, int64_t T, const void* A,
                           const void* B, const void* s0, void* S, int32_t mem) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  if (dtype != PMCMC_F32 && dtype != PMCMC_F64)
    return fail(h, PMCMC_ERR_ARGUMENT, "dtype must be PMCMC_F32 or PMCMC_F64");
  if (D < 0 || T < 0) return fail(h, PMCMC_ERR_DIMENSION, "negative dimension");
  if (T == 0 || D == 0) return PMCMC_OK;
  if (!A || !B || !s0 || !S) return fail(h, PMCMC_ERR_ARGUMENT, "null buffer");
  if (S == A) return fail(h, PMCMC_ERR_ARGUMENT, "S must not alias A");
  if (S == B) return fail(h, PMCMC_ERR_ARGUMENT, "S must not alias B");
  const bool f64 = dtype == PMCMC_F64;
  const size_t es = f64 ? 8 : 4;
  if (3 * es * static_cast<size_t>(D) > 200 * 1024)
    return fail(h, PMCMC_ERR_UNSUPPORTED, "dimension %lld too large for the scan kernel",
                (long long)D);
  DeviceGuard guard(h->device);
  const int TT = scan_tile_cols(D, T);
  const int64_t nt = (T + TT - 1) / TT;
  // scratch: counter[2] | flags[nt] | agg_a | agg_b | incl | (host I/O staging)
  const size_t o_flags = 64;
  const size_t o_agg_a = (o_flags + 4 * static_cast<size_t>(nt) + 255) & ~size_t(255);
  const size_t o_agg_b = o_agg_a + ((es * nt * D + 255) & ~size_t(255));
  const size_t o_incl = o_agg_b + ((es * nt * D + 255) & ~size_t(255));
  const size_t o_io = o_incl + ((es * nt * D + 255) & ~size_t(255));
  const size_t need = o_io + (mem == PMCMC_MEM_HOST ? 3 * es * D * T + es * D + 256 : 0);
  if (need > h->scan_ws_bytes) {
    CK(cudaStreamSynchronize(h->stream));
    cudaFree(h->scan_ws);
    h->scan_ws = nullptr;
    h->scan_ws_bytes = 0;
    if (cudaMalloc(&h->scan_ws, need) != cudaSuccess) {
      cudaGetLastError();
      return fail(h, PMCMC_ERR_NOMEM, "scan scratch allocation failed");
    }
    CK(cudaMemsetAsync(h->scan_ws, 0, need, h->stream));
    h->scan_ws_bytes = need;
  }
  unsigned char* base = h->scan_ws;
  ScanScratch scr;
  scr.counter = reinterpret_cast<uint32_t*>(base);
  scr.flags = reinterpret_cast<uint32_t*>(base + o_flags);
  scr.agg_a = base + o_agg_a;
  scr.agg_b = base + o_agg_b;
  scr.incl = base + o_incl;
  const void *dA = A, *dB = B, *ds0 = s0;
  void* dS = S;
  if (mem == PMCMC_MEM_HOST) {
    unsigned char* io = base + o_io;
    dA = io;
    dB = io + es * D * T;
    dS = io + 2 * es * D * T;
    ds0 = io + 3 * es * D * T;
    CK(cudaMemcpyAsync(const_cast<void*>(dA), A, es * D * T, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(const_cast<void*>(dB), B, es * D * T, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(const_cast<void*>(ds0), s0, es * D, cudaMemcpyHostToDevice, h->stream));
  }
  h->scan_epoch = (h->scan_epoch + 1) & 0x3fffffffu;
  if (h->scan_epoch == 0) h->scan_epoch = 1;
  CK(launch_affine_scan(h->stream, f64, D, T, dA, dB, ds0, dS, scr, h->scan_epoch));
  if (mem == PMCMC_MEM_HOST)
    CK(cudaMemcpyAsync(S, dS, es * D * T, cudaMemcpyDeviceToHost, h->stream));
  uint32_t flags[2] = {0, 0};
  CK(cudaMemcpyAsync(flags, scr.counter, sizeof flags, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flags[1]) return fail(h, PMCMC_ERR_TIMEOUT, "scan look-back wait exceeded its bound");
  return PMCMC_OK;
}

}  // extern "C"
