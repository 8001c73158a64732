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
#include <atomic>
#include <map>
#include <tuple>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pmcmc_deer.h"
#include "deer_device.cuh"
#include "deer_launch.h"
#include "full.h"
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

// One slice [t0, t0 + W) of a block, solved by the T-split Newton iteration
// (pmcmc_slice_*): the handle keeps the slice's iterate, tape and A/B.
struct SliceState {
  bool active = false;
  const pmcmc_target* tg = nullptr;
  pmcmc_deer_params p{};
  DevParams P{};
  int cur = 0, iter = 0;
  size_t es = 4;
  size_t S[2], x0, xbar, carry, ones, A, B, Sloc, Zb, xi, logu, red, scr, out_S, out_lp,
      out_acc, x_next, total;
};

constexpr size_t kCublasWsBytes = size_t(32) << 20;

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
  bool no_persist = false;  // solves of Gaussian targets through the per-sweep graph instead
  int tile_override = 0;
  unsigned long long* h_red = nullptr;  // pinned, plain-path metric readback
  cublasHandle_t cublas = nullptr;
  bool profiling = false;
  pmcmc_profile prof{};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  // :full mode
  FullArgs* d_full = nullptr;
  DevParams* d_params_e = nullptr;  // eigenbasis view of the :full solve
  cudaGraphExec_t gexec_full = nullptr;
  cudaGraphConditionalHandle cond_full = 0;
  unsigned char gkey_full[192] = {};
  int full_chunks_override = 0;
  // candidate shapes while pmcmc_autotune times them (0: none)
  int tune_per_sm = 0;
  int tune_full_chunks = 0;
  SliceState slice;
  void* cublas_ws = nullptr;  // cuBLAS workspace of its own (no allocation inside its calls)
  std::vector<pmcmc_handle*> fleet;  // worker handles of pmcmc_fleet_solve (own streams)
  // host-output pipeline of multi-block solves: block b's device-to-host copy
  // runs on copy_stream while block b + 1 solves on stream
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_fin[2] = {nullptr, nullptr};   // block output ready (slot b & 1)
  cudaEvent_t ev_copy[2] = {nullptr, nullptr};  // slot b & 1 copied out, reusable
  DevState* h_states = nullptr;                 // pinned, one per block
  int64_t h_states_cap = 0;
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
  // Gaussian targets: host copy of the precision and, once the :full mode or
  // the adjoint first needs it, its eigendecomposition P = Q diag(lam) Q^T
  std::vector<double> prec_host;  // D x D column-major (dense) or D (diagonal)
  bool eig_ready = false;
  std::vector<double> eig_lam, eig_Q;  // D, D x D column-major
  float* lam_f = nullptr;              // Dp
  float* qrm_f = nullptr;              // Dp x Dp, Q row-major
  float* qcm_f = nullptr;              // Dp x Dp, Q column-major
  // the same, padded to the :full sweep stride Dq (zero when D > 128)
  int dq = 0;
  float* lamq_f = nullptr;   // Dq
  double* lamq_d = nullptr;  // Dq
  float* zq_f = nullptr;     // Dq zeros (eigenbasis mean)
  double* zq_d = nullptr;    // Dq zeros
  float* qrmq = nullptr;     // Dq x Dq, Q row-major
  float* qcmq = nullptr;     // Dq x Dq, Q column-major
  std::vector<double> mean_host;  // D (Gaussian targets)
  // Mass-matrix targets (pmcmc_target_mass): this target is the whitened one,
  // and L (D x D column-major, lower triangular) maps its chains back.
  std::vector<double> mass_L;
  double* mass_Ld = nullptr;
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

// Copy stream, slot events and a pinned per-block state ring for a host-output
// solve of nblocks blocks.
int ensure_pipeline(pmcmc_handle* h, int64_t nblocks) {
  if (!h->copy_stream) {
    int lo = 0, hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CK(cudaStreamCreateWithPriority(&h->copy_stream, cudaStreamNonBlocking, lo));
    for (int i = 0; i < 2; ++i) {
      CK(cudaEventCreateWithFlags(&h->ev_fin[i], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&h->ev_copy[i], cudaEventDisableTiming));
    }
  }
  if (nblocks > h->h_states_cap) {
    if (h->h_states) {
      CK(cudaStreamSynchronize(h->stream));
      CK(cudaFreeHost(h->h_states));
      h->h_states = nullptr;
      h->h_states_cap = 0;
    }
    const int64_t cap = std::max<int64_t>(nblocks, 64);
    CK(cudaMallocHost(&h->h_states, sizeof(DevState) * static_cast<size_t>(cap)));
    h->h_states_cap = cap;
  }
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
  // targets are read-only device data: any handle on the target's device may use them
  if (t->h != h && t->h->device != h->device)
    return fail(h, PMCMC_ERR_ARGUMENT, "target lives on another device");
  return PMCMC_OK;
}

// Resident CTAs per SM of a kernel at kThreads threads and `smem` bytes of
// dynamic shared memory, cached per (kernel, bytes): the query costs
// microseconds of host time and a solve asks for several sizes.
int max_active_blocks(const void* fn, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<const void*, size_t>, int> cache;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find({fn, smem});
    if (it != cache.end()) return it->second;
  }
  if (raise_smem_limit(fn, smem) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kThreads, smem) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  std::lock_guard<std::mutex> lk(mu);
  cache[{fn, smem}] = nb;
  return nb;
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
      const int nb = max_active_blocks(k.sweep_coop, smem);
      if (nb < 0) break;
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

// Shapes chosen by pmcmc_autotune, process-wide, keyed by problem shape:
// what = 0: CTAs a SM of the persistent solve; what = 1: :full chunk count.
struct TuneKey {
  int what, kind, jac, f64;
  int64_t D, T;
  bool operator<(const TuneKey& o) const {
    return std::tie(what, kind, jac, f64, D, T) < std::tie(o.what, o.kind, o.jac, o.f64, o.D, o.T);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, int> g_tune;

int tune_get(const TuneKey& k) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(k);
  return it == g_tune.end() ? 0 : it->second;
}
void tune_put(const TuneKey& k, int v) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[k] = v;
}

// TT for `per_sm` co-resident CTAs a SM of the persistent solve, 0 if they do not fit.
int persist_tile_for(const void* fn, bool f64, int64_t Dp, int64_t T, bool dense, int per_sm,
                     int num_sms) {
  const int64_t TT = (T + int64_t(per_sm) * num_sms - 1) / (int64_t(per_sm) * num_sms);
  if (TT > 256) return 0;
  const size_t smem = persist_smem(f64, Dp, static_cast<int>(TT), dense).total;
  if (smem > 200 * 1024) return 0;
  const int nb = max_active_blocks(fn, smem);
  return nb >= per_sm ? static_cast<int>(TT) : 0;
}

// Columns per CTA of the persistent solve: the autotuned CTAs a SM for this
// shape when there is one, else the most CTAs a SM whose tiles all fit
// co-resident (one cooperative launch), TT = ceil(T / (CTAs a SM x SMs)); 0
// when none fits.
int choose_persist_tile(pmcmc_handle* h, const void* fn, bool f64, int64_t Dp, int64_t T,
                        bool dense, const TuneKey& key) {
  if (!fn || h->no_coop || h->tile_override > 0) return 0;
  if (h->tune_per_sm > 0) return persist_tile_for(fn, f64, Dp, T, dense, h->tune_per_sm, h->num_sms);
  if (const int tuned = tune_get(key)) {
    const int TT = persist_tile_for(fn, f64, Dp, T, dense, tuned, h->num_sms);
    if (TT > 0) return TT;
  }
  for (int per_sm = 8; per_sm >= 1; --per_sm) {
    const int64_t TT = (T + int64_t(per_sm) * h->num_sms - 1) / (int64_t(per_sm) * h->num_sms);
    if (TT > 256) break;
    const size_t smem = persist_smem(f64, Dp, static_cast<int>(TT), dense).total;
    if (smem > 200 * 1024) continue;
    const int nb = max_active_blocks(fn, smem);
    if (nb < 0) return 0;
    if (nb >= per_sm) return static_cast<int>(TT);
  }
  return 0;
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
  size_t la_ref, tie, lg_acc;                           // logistic: log alpha, near-tie scratch, probe sum
  size_t xi, logu;
  size_t tcws, Gtc;  // tensor-core logistic path
  size_t fU, fV, fR, facc, fPhi, fbeta, fdin, fpart, eS0, eS1, exi, ex0;  // :full mode
  size_t alam, acterm, aarev, adirect, ascr, aout;                 // adjoint
  size_t out2_S, out2_lp, out2_acc;  // second output slot of the host-output pipeline
  size_t part;                       // per-CTA partial reductions of the persistent solve
  size_t total;
};

SolveLayout layout(int64_t D, int64_t Dp, int64_t T, int ntiles, size_t es, bool plain,
                   int64_t N = 0, int64_t Tc = 0, size_t tc_bytes = 0,
                   const FullPlan* fp = nullptr, bool adjoint = false,
                   bool dual_out = false, size_t tie_bytes = 0) {
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
  L.incl = take(es * (ntiles + 1) * Dp);  // + the persistent solve's S_0
  L.colmax = take(4 * static_cast<size_t>(T));
  L.part = take(8 * 8 * static_cast<size_t>(ntiles));
  L.out_S = take(es * T * D);
  L.out_lp = take(es * T);
  L.out_acc = take(static_cast<size_t>(T));
  if (dual_out) {
    L.out2_S = take(es * T * D);
    L.out2_lp = take(es * T);
    L.out2_acc = take(static_cast<size_t>(T));
  }
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
    L.la_ref = take(8 * static_cast<size_t>(T));
    L.tie = take(tie_bytes);
    L.lg_acc = take(es * T * Dp);
  }
  if (tc_bytes) {
    L.tcws = take(tc_bytes);
    L.Gtc = take(4 * Dp * 2 * static_cast<size_t>(T));
  }
  if (fp || adjoint) L.facc = take(static_cast<size_t>(T));
  if (fp) {
    const int64_t Dq = fp->Dq;
    L.eS0 = take(4 * T * Dq);
    L.eS1 = take(4 * T * Dq);
    L.exi = take(4 * T * Dq);
    L.ex0 = take(4 * Dq);
    L.fU = take(4 * T * Dq);
    L.fV = take(4 * T * Dq);
    L.fR = take(4 * T * Dq);
    L.fPhi = take(4 * static_cast<size_t>(fp->nchunks) * Dq * Dq);
    L.fbeta = take(4 * static_cast<size_t>(fp->nchunks) * Dq);
    L.fdin = take(4 * static_cast<size_t>(fp->nchunks) * Dq);
    L.fpart = take(16 * static_cast<size_t>(fp->nchunks));
  }
  if (adjoint) {
    L.alam = take(4 * T * Dp);
    L.acterm = take(4 * T * Dp);
    L.aarev = take(4 * T * Dp);
    L.adirect = take(8);
    L.ascr = take(full_adjoint_scratch_bytes(Dp, T));
    L.aout = take(8 * static_cast<size_t>(D + 1));
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
  if (smem_sweep > 0)
    CK(raise_smem_limit(reinterpret_cast<const void*>(sweep_fn), smem_sweep));
  if (smem_fin > 0)
    CK(raise_smem_limit(reinterpret_cast<const void*>(k.finalize), smem_fin));
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

// One DEER block as one cooperative launch of the persistent solve kernel
// (tape, every sweep and the verification pass; deer_persist.cu).
int run_persist(pmcmc_handle* h, const SweepKernels& k, const DevParams& P, size_t smem,
                int64_t nblk) {
  CK(raise_smem_limit(k.persist, smem));
  DevParams Pv = P;  // by value in the launch
  void* args[] = {&Pv, &h->d_state};
  if (h->profiling) CK(cudaEventRecord(h->ev[0], h->stream));
  CK(cudaLaunchCooperativeKernel(k.persist, dim3(P.ntiles), dim3(kThreads), args, smem,
                                 h->stream));
  if (h->profiling) {
    CK(cudaEventRecord(h->ev[1], h->stream));
    CK(cudaMemcpyAsync(h->h_state, h->d_state, sizeof(DevState), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
    h->prof.solve_launches += 1;
    h->prof.solve_ms += ms;
    if (nblk > 1) {  // the blocks' states are in the pinned ring
      for (int64_t b = 0; b < nblk; ++b) h->prof.solve_sweeps += P.st_host[b].iter;
    } else {
      h->prof.solve_sweeps += h->h_state->iter;
    }
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
  if (smem_fin > 0) {
    CK(raise_smem_limit(reinterpret_cast<const void*>(k.finalize), smem_fin));
    CK(raise_smem_limit(reinterpret_cast<const void*>(k.eval), smem_fin));
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

// Near-tie band of the FP64 decisions of the logistic target and the most
// columns one refinement recomputes (logistic_tie.cu).  The tensor-core
// log alpha is off by up to ~1e-4; columns inside 1e-3 (about 60 of 65536 at
// N = 10000, D = 256) are decided in FP64.
constexpr float kTieBand = 1e-3f;
constexpr int kTieMax = 256;
int tie_kmax(int64_t T) { return static_cast<int>(std::min<int64_t>(kTieMax, T)); }

// One DEER block for the logistic target: per Newton iteration two GEMM
// passes (pass 1 at [x_bar | z], pass 2 at [y | w]) feed the fused
// finish + scan sweep kernel.  On the fused FP32 path the columns near a tie
// are decided in FP64 before the sweep (`refine`).  Then, on the fused path, a
// verification pass at the returned trajectory (its passes at x_bar_t =
// S_{t-1}: accept flags, margins, defect) and a logp pass over it.
// The handle's cuBLAS (pedantic math, a workspace of its own so that cuBLAS
// allocates nothing during a solve), on the handle's stream.
int ensure_cublas(pmcmc_handle* h) {
  if (!h->cublas) {
    if (cublasCreate(&h->cublas) != CUBLAS_STATUS_SUCCESS)
      return fail(h, PMCMC_ERR_CUDA, "cublasCreate failed");
    cublasSetMathMode(h->cublas, CUBLAS_PEDANTIC_MATH);
    CK(cudaMalloc(&h->cublas_ws, kCublasWsBytes));
    if (cublasSetWorkspace(h->cublas, h->cublas_ws, kCublasWsBytes) != CUBLAS_STATUS_SUCCESS)
      return fail(h, PMCMC_ERR_CUDA, "cublasSetWorkspace failed");
  }
  cublasSetStream(h->cublas, h->stream);
  return PMCMC_OK;
}

int run_logistic(pmcmc_handle* h, const pmcmc_target* tg, const SweepKernels& k, bool coop,
                 DevParams P, const SolveLayout& L, size_t es, size_t smem_sweep,
                 int fin_grid, int init_grid, int64_t Tc, bool use_tc, bool plain) {
  unsigned char* ws = h->ws;
  const bool f64 = es == 8;
  const bool refine = !plain && !f64;
  double* la_ref = reinterpret_cast<double*>(ws + L.la_ref);
  const TieBufs tb = lg_tie_carve(ws + L.tie, tg->lg, P.T, tie_kmax(P.T));
  P.la_ref = refine ? la_ref : nullptr;
  P.lg_acc = ws + L.lg_acc;
  P.tc_err = use_tc ? lg_tc_err_word(ws + L.tcws, tg->lg, P.T) : nullptr;
  const void* k_acc = k.eval;  // the probe accumulation kernel of the logistic target
  CK(cudaMemcpyAsync(h->d_params, &P, sizeof(DevParams), cudaMemcpyHostToDevice, h->stream));
  if (smem_sweep > 0)
    CK(raise_smem_limit(reinterpret_cast<const void*>(coop ? k.sweep_coop : k.sweep), smem_sweep));
  int rc = ensure_cublas(h);
  if (rc) return rc;
  void* init_args[] = {&h->d_params, &h->d_state};
  CK(cudaLaunchKernel(k.init, dim3(init_grid), dim3(256), init_args, 0, h->stream));
  cudaGraphConditionalHandle none = 0;
  int zero = 0;
  void* sweep_args[] = {&h->d_params, &h->d_state, &none, &zero};
  void *Bb = ws + L.Bb, *Lb = ws + L.Lb, *Gb = ws + L.Gb;
  int* tc_err = use_tc ? lg_tc_err_word(ws + L.tcws, tg->lg, P.T) : nullptr;
  if (use_tc) CK(cudaMemsetAsync(tc_err, 0, sizeof(int), h->stream));
  auto pass_impl = [&](int mode, double* lp, int probe) -> int {
    if (use_tc) {
      float* G = reinterpret_cast<float*>(ws + L.Gtc);
      if (lg_tc_pass(h->stream, tg->lg, h->d_params, h->d_state, lp, mode, P.T, ws + L.tcws, G,
                     probe))
        return 1;
      if (mode != 2 && lg_mid(h->stream, false, h->d_params, h->d_state, mode + 1, 0,
                              static_cast<int>(P.T), probe, P.Dp, G) != cudaSuccess)
        return 1;
      return 0;
    }
    return lg_plain_pass(h->stream, h->cublas, tg->lg, f64, h->d_params, h->d_state, lp, mode,
                         P.T, P.Dp, Bb, Lb, Gb, Tc, probe);
  };
  auto pass = [&](int mode, double* lp, int probe = 0) -> int {
    if (h->profiling && mode != 2) {
      // one contraction pass timed on its own (events around it, synchronised)
      if (cudaEventRecord(h->ev[0], h->stream) != cudaSuccess) return 1;
      const int rc = pass_impl(mode, lp, probe);
      float ms = 0;
      if (rc || cudaEventRecord(h->ev[1], h->stream) != cudaSuccess ||
          cudaEventSynchronize(h->ev[1]) != cudaSuccess ||
          cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]) != cudaSuccess)
        return 1;
      h->prof.pass_launches += 1;
      h->prof.pass_ms += ms;
      return 0;
    }
    return pass_impl(mode, lp, probe);
  };
  auto tie = [&]() -> int {
    if (lg_tie_refine(h->stream, h->cublas, tg->lg, f64, h->d_params, h->d_state, P.T, la_ref,
                      tb, kTieBand))
      return fail(h, PMCMC_ERR_CUDA, "near-tie refinement failed: %s",
                  cudaGetErrorString(cudaGetLastError()));
    return PMCMC_OK;
  };
  // the tensor-core error word travels with the state in every per-sweep copy
  int* h_err = reinterpret_cast<int*>(h->h_red + 3);
  *h_err = 0;
  // probes > 1 (DEER.jl:412-418): the passes run once per probe; the probes before the
  // last add z_k .* J z_k into lg_acc, the sweep adds the last and divides
  const int grid_acc = static_cast<int>(std::min<int64_t>((P.T + kWarps - 1) / kWarps,
                                                          int64_t(h->num_sms) * 8));
  const bool lg_diag = P.jac == PMCMC_JAC_DIAG;
  // The launches of one Newton sweep, ending with the finish-and-scan kernel.
  auto issue_sweep = [&]() -> int {
    // exact diagonal: g_x, y, diag H_x | g_y | H_y r | H_x u (logistic.cu, modes 3-6)
    for (int m = 3; lg_diag && m <= 6; ++m) {
      if (pass(m, m == 4 || m == 5 ? P.lpy : P.lpx))
        return fail(h, PMCMC_ERR_CUDA, "logistic :diag pass failed: %s",
                    cudaGetErrorString(cudaGetLastError()));
      if (refine && m == 4) {
        const int rc = tie();
        if (rc) return rc;
      }
    }
    for (int pr = 0; !lg_diag && pr < P.probes; ++pr) {
      if (pass(0, P.lpx, pr))
        return fail(h, PMCMC_ERR_CUDA, "logistic pass 1 failed: %s",
                    cudaGetErrorString(cudaGetLastError()));
      if (pass(1, P.lpy, pr))
        return fail(h, PMCMC_ERR_CUDA, "logistic pass 2 failed: %s",
                    cudaGetErrorString(cudaGetLastError()));
      if (refine && pr == 0) {  // the value columns, and so log alpha, are the same for every probe
        const int rc = tie();
        if (rc) return rc;
      }
      if (pr + 1 < P.probes) {
        int probe = pr;
        void* acc_args[] = {&h->d_params, &h->d_state, &probe};
        CK(cudaLaunchKernel(k_acc, dim3(grid_acc), dim3(kThreads), acc_args, 0, h->stream));
      }
    }
    if (h->profiling) CK(cudaEventRecord(h->ev[0], h->stream));
    CK(launch_sweep(coop ? k.sweep_coop : k.sweep, coop, P.ntiles, smem_sweep, sweep_args,
                    h->stream));
    if (h->profiling) CK(cudaEventRecord(h->ev[1], h->stream));
    return PMCMC_OK;
  };
  // The Newton loop: one sweep after another, with a host check of the state after
  // each (the convergence test, maxiter, a non-finite state, a tensor-core wait error).
  auto eager_sweep = [&]() -> int {  // one sweep with the host check of its state
    const int rc = issue_sweep();
    if (rc) return rc;
    CK(cudaMemcpyAsync(h->h_state, h->d_state, sizeof(DevState), cudaMemcpyDeviceToHost,
                       h->stream));
    if (use_tc)
      CK(cudaMemcpyAsync(h_err, tc_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (h->profiling) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
      h->prof.sweep_launches += 1;
      h->prof.sweep_ms += ms;
    }
    if (*h_err) return fail(h, PMCMC_ERR_TIMEOUT, "tensor-core pass: a bounded wait gave up");
    return PMCMC_OK;
  };
  for (int it = 0; it < P.maxiter; ++it) {
    const int rc = eager_sweep();
    if (rc) return rc;
    if (h->h_state->converged || h->h_state->status) break;
  }
  if (!plain && !h->h_state->status) {
    // verification at the returned trajectory: the passes at x_bar_t = S_{t-1},
    // the near-tie decisions in FP64, then flags, margins and the defect
    if (pass(0, P.lpx) || pass(1, P.lpy))
      return fail(h, PMCMC_ERR_CUDA, "logistic verification pass failed: %s",
                  cudaGetErrorString(cudaGetLastError()));
    if (refine) {
      const int rc = tie();
      if (rc) return rc;
    } else {
      CK(lg_margin(h->stream, f64, h->d_params, h->d_state, P.T, la_ref, tb.mg));
    }
    CK(lg_verify(h->stream, f64, h->d_params, h->d_state, P.T, la_ref));
  }
  if (pass(2, P.lpx)) return fail(h, PMCMC_ERR_CUDA, "logistic logp pass failed");
  void* fin_args[] = {&h->d_params, &h->d_state};
  CK(cudaLaunchKernel(k.finalize, dim3(fin_grid), dim3(kThreads), fin_args, 0, h->stream));
  if (use_tc) {
    CK(cudaMemcpyAsync(h_err, tc_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (*h_err) return fail(h, PMCMC_ERR_TIMEOUT, "tensor-core pass: a bounded wait gave up");
  }
  return PMCMC_OK;
}

// Symmetric eigendecomposition by cyclic Jacobi rotations (Golub & Van Loan,
// Matrix Computations, sec. 8.5): A (n x n, row-major) is overwritten; on
// return w holds the eigenvalues ascending and V (row-major) the eigenvectors
// as columns.
void jacobi_eigen(int n, std::vector<double>& A, std::vector<double>& w, std::vector<double>& V) {
  V.assign(static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i) V[static_cast<size_t>(i) * n + i] = 1.0;
  auto a = [&](int i, int j) -> double& { return A[static_cast<size_t>(i) * n + j]; };
  auto v = [&](int i, int j) -> double& { return V[static_cast<size_t>(i) * n + j]; };
  double scale = 0.0;
  for (double x : A) scale += x * x;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += a(p, q) * a(p, q);
    if (off <= 1e-30 * scale) break;
    for (int p = 0; p < n; ++p) {
      for (int q = p + 1; q < n; ++q) {
        const double apq = a(p, q);
        if (apq == 0.0) continue;
        const double theta = (a(q, q) - a(p, p)) / (2.0 * apq);
        const double tt =
            (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(tt * tt + 1.0), sn = tt * c;
        for (int k = 0; k < n; ++k) {
          const double kp = a(k, p), kq = a(k, q);
          a(k, p) = c * kp - sn * kq;
          a(k, q) = sn * kp + c * kq;
        }
        for (int k = 0; k < n; ++k) {
          const double pk = a(p, k), qk = a(q, k);
          a(p, k) = c * pk - sn * qk;
          a(q, k) = sn * pk + c * qk;
        }
        for (int k = 0; k < n; ++k) {
          const double kp = v(k, p), kq = v(k, q);
          v(k, p) = c * kp - sn * kq;
          v(k, q) = sn * kp + c * kq;
        }
      }
    }
  }
  std::vector<int> ord(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int x, int y) { return a(x, x) < a(y, y); });
  w.resize(static_cast<size_t>(n));
  std::vector<double> Vs(V.size());
  for (int j = 0; j < n; ++j) {
    w[j] = a(ord[j], ord[j]);
    for (int i = 0; i < n; ++i) Vs[static_cast<size_t>(i) * n + j] = v(i, ord[j]);
  }
  V.swap(Vs);
}

// Eigendecomposition of a Gaussian target's precision, on the host in FP64,
// uploaded once: lam and Q (row-major and column-major) at the target's
// stride Dp and at the :full sweep stride Dq.  A diagonal target keeps its
// order with Q = I.
int ensure_eigen(pmcmc_handle* h, pmcmc_target* t) {
  if (t->eig_ready) return PMCMC_OK;
  if (t->kind != kDiagGauss && t->kind != kDenseGauss)
    return fail(h, PMCMC_ERR_UNSUPPORTED, "eigendecomposition is defined for the Gaussian targets");
  const int64_t D = t->D, Dp = t->Dp;
  std::vector<double> lam, Qrow;
  if (t->kind == kDenseGauss) {
    std::vector<double> A(static_cast<size_t>(D * D));
    for (int64_t j = 0; j < D; ++j)
      for (int64_t i = 0; i < D; ++i)  // symmetrised row-major copy of the column-major input
        A[i * D + j] = 0.5 * (t->prec_host[j * D + i] + t->prec_host[i * D + j]);
    jacobi_eigen(static_cast<int>(D), A, lam, Qrow);
  } else {
    lam = t->prec_host;
    Qrow.assign(static_cast<size_t>(D * D), 0.0);
    for (int64_t i = 0; i < D; ++i) Qrow[i * D + i] = 1.0;
  }
  t->eig_lam = lam;
  t->eig_Q.assign(static_cast<size_t>(D * D), 0.0);
  for (int64_t i = 0; i < D; ++i)
    for (int64_t k = 0; k < D; ++k) t->eig_Q[k * D + i] = Qrow[i * D + k];
  DeviceGuard guard(h->device);
  // layout at stride n: lam (n), Q row-major and column-major (n x n)
  auto upload = [&](int64_t n, float* lf, double* ld, float* qr, float* qc) -> int {
    std::vector<float> lv(static_cast<size_t>(n), 0.f), rv(static_cast<size_t>(n * n), 0.f),
        cv(static_cast<size_t>(n * n), 0.f);
    std::vector<double> ldv(static_cast<size_t>(n), 0.0);
    for (int64_t i = 0; i < D; ++i) {
      lv[i] = static_cast<float>(lam[i]);
      ldv[i] = lam[i];
      for (int64_t k = 0; k < D; ++k) {
        const float q = static_cast<float>(Qrow[i * D + k]);  // component i of eigenvector k
        rv[i * n + k] = q;
        cv[k * n + i] = q;
      }
    }
    CK(cudaMemcpy(lf, lv.data(), 4 * n, cudaMemcpyHostToDevice));
    if (ld) CK(cudaMemcpy(ld, ldv.data(), 8 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(qr, rv.data(), 4 * n * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(qc, cv.data(), 4 * n * n, cudaMemcpyHostToDevice));
    return PMCMC_OK;
  };
  if (!t->lam_f) {
    if (cudaMalloc(&t->lam_f, 4 * Dp) != cudaSuccess ||
        cudaMalloc(&t->qrm_f, 4 * Dp * Dp) != cudaSuccess ||
        cudaMalloc(&t->qcm_f, 4 * Dp * Dp) != cudaSuccess) {
      cudaGetLastError();
      return fail(h, PMCMC_ERR_NOMEM, "eigenbasis allocation failed");
    }
  }
  int rc = upload(Dp, t->lam_f, nullptr, t->qrm_f, t->qcm_f);
  if (rc) return rc;
  const int Dq = full_stride(Dp);
  if (Dq) {
    if (!t->lamq_f &&
        (cudaMalloc(&t->lamq_f, 4 * Dq) != cudaSuccess || cudaMalloc(&t->lamq_d, 8 * Dq) != cudaSuccess ||
         cudaMalloc(&t->zq_f, 4 * Dq) != cudaSuccess || cudaMalloc(&t->zq_d, 8 * Dq) != cudaSuccess ||
         cudaMalloc(&t->qrmq, 4 * Dq * Dq) != cudaSuccess ||
         cudaMalloc(&t->qcmq, 4 * Dq * Dq) != cudaSuccess)) {
      cudaGetLastError();
      return fail(h, PMCMC_ERR_NOMEM, "eigenbasis allocation failed");
    }
    rc = upload(Dq, t->lamq_f, t->lamq_d, t->qrmq, t->qcmq);
    if (rc) return rc;
    CK(cudaMemset(t->zq_f, 0, 4 * Dq));
    CK(cudaMemset(t->zq_d, 0, 8 * Dq));
    t->dq = Dq;
  }
  t->eig_ready = true;
  return PMCMC_OK;
}

// The eigenbasis view of a :full solve: the diagonal Gaussian N(0, diag(1/lam))
// at the sweep stride Dq, with the rotated tape and iterate buffers (Q = I for
// a diagonal target).
DevParams eigen_view(const DevParams& P, const pmcmc_target* tg, unsigned char* ws,
                     const SolveLayout& L) {
  DevParams Pe = P;
  Pe.Dp = tg->dq;
  Pe.prec_f = tg->lamq_f;
  Pe.prec_d = tg->lamq_d;
  Pe.mean_f = tg->zq_f;
  Pe.mean_d = tg->zq_d;
  Pe.xi = reinterpret_cast<float*>(ws + L.exi);
  Pe.x0 = ws + L.ex0;
  Pe.S[0] = ws + L.eS0;
  Pe.S[1] = ws + L.eS1;
  Pe.tkind = kDiagGauss;
  return Pe;
}

struct FullGraphKey {
  FullPlan fp;
  const void* init;
  const void* fin;
  int init_grid, fin_grid;
  size_t smem_fin;
};
static_assert(sizeof(FullGraphKey) <= sizeof(pmcmc_handle::gkey_full), "graph key size");

// init -> rotate -> while(eval, chunk, carry, apply) -> finalize, the loop
// condition set by the last CTA of the apply kernel.
int build_graph_full(pmcmc_handle* h, const FullGraphKey& key) {
  unsigned char kb[sizeof(pmcmc_handle::gkey_full)] = {};
  std::memcpy(kb, &key, sizeof key);
  if (h->gexec_full && std::memcmp(kb, h->gkey_full, sizeof kb) == 0) return PMCMC_OK;
  if (h->gexec_full) {
    cudaGraphExecDestroy(h->gexec_full);
    h->gexec_full = nullptr;
  }
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle cond = 0;
  cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(h, PMCMC_ERR_CUDA, "cudaGraphConditionalHandleCreate: %s", cudaGetErrorString(e));
  }
  h->cond_full = cond;
  int one = 1;
  void* pair_args[] = {&h->d_params, &h->d_state};
  void* sweep_args[] = {&h->d_params, &h->d_full, &h->d_state, &h->cond_full, &one};
  cudaKernelNodeParams kp{};
  kp.func = const_cast<void*>(key.init);
  kp.gridDim = dim3(key.init_grid);
  kp.blockDim = dim3(256);
  kp.kernelParams = pair_args;
  cudaGraphNode_t n_init, n_rot, n_while, n_fin;
  e = cudaGraphAddKernelNode(&n_init, g, nullptr, 0, &kp);
  if (e == cudaSuccess) {
    cudaKernelNodeParams rp{};
    rp.func = const_cast<void*>(key.fp.rotate);
    rp.gridDim = dim3(key.fp.rotate_grid);
    rp.blockDim = dim3(kThreads);
    rp.sharedMemBytes = static_cast<unsigned>(key.fp.smem_rotate);
    rp.kernelParams = sweep_args;
    e = cudaGraphAddKernelNode(&n_rot, g, &n_init, 1, &rp);
  }
  cudaGraphNodeParams cp{};
  if (e == cudaSuccess) {
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&n_while, g, &n_rot, 1, &cp);
  }
  if (e == cudaSuccess) {
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const void* fns[4] = {key.fp.eval, key.fp.chunk, key.fp.carry, key.fp.apply};
    const size_t sm[4] = {key.fp.smem_eval, key.fp.smem_chunk, key.fp.smem_carry,
                          key.fp.smem_apply};
    const int grid[4] = {key.fp.eval_grid, key.fp.nchunks, 1, key.fp.nchunks};
    const int thr[4] = {kThreads, key.fp.threads_chunk, 256, kThreads};
    cudaGraphNode_t prev = nullptr;
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) {
      cudaKernelNodeParams sp{};
      sp.func = const_cast<void*>(fns[i]);
      sp.gridDim = dim3(grid[i]);
      sp.blockDim = dim3(thr[i]);
      sp.sharedMemBytes = static_cast<unsigned>(sm[i]);
      sp.kernelParams = sweep_args;
      cudaGraphNode_t n;
      e = cudaGraphAddKernelNode(&n, body, prev ? &prev : nullptr, prev ? 1 : 0, &sp);
      prev = n;
    }
  }
  if (e == cudaSuccess) {
    cudaKernelNodeParams fp{};
    fp.func = const_cast<void*>(key.fin);
    fp.gridDim = dim3(key.fin_grid);
    fp.blockDim = dim3(kThreads);
    fp.sharedMemBytes = static_cast<unsigned>(key.smem_fin);
    fp.kernelParams = pair_args;
    e = cudaGraphAddKernelNode(&n_fin, g, &n_while, 1, &fp);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&h->gexec_full, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->gexec_full = nullptr;
    return fail(h, PMCMC_ERR_CUDA, "CUDA graph construction failed: %s", cudaGetErrorString(e));
  }
  std::memcpy(h->gkey_full, kb, sizeof kb);
  return PMCMC_OK;
}

// One DEER block in :full mode (FP32 Gaussian targets).
int run_full(pmcmc_handle* h, const SweepKernels& k, const FullPlan& fp, const DevParams& P,
             const DevParams& Pe, const FullArgs& F, size_t smem_fin, int fin_grid,
             int init_grid) {
  CK(cudaMemcpyAsync(h->d_params, &P, sizeof(DevParams), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_params_e, &Pe, sizeof(DevParams), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_full, &F, sizeof(FullArgs), cudaMemcpyHostToDevice, h->stream));
  {
    const void* fns[6] = {fp.eval, fp.chunk, fp.carry, fp.apply, k.finalize, fp.rotate};
    const size_t sm[6] = {fp.smem_eval, fp.smem_chunk, fp.smem_carry, fp.smem_apply, smem_fin,
                          fp.smem_rotate};
    for (int i = 0; i < 6; ++i)
      if (sm[i] > 0)
        CK(raise_smem_limit(reinterpret_cast<const void*>(fns[i]), sm[i]));
  }
  if (!h->force_eager && !h->profiling) {
    FullGraphKey key{};
    key.fp = fp;
    key.init = k.init;
    key.fin = k.finalize;
    key.init_grid = init_grid;
    key.fin_grid = fin_grid;
    key.smem_fin = smem_fin;
    const int rc = build_graph_full(h, key);
    if (rc == PMCMC_OK) {
      CK(cudaGraphLaunch(h->gexec_full, h->stream));
      return PMCMC_OK;
    }
    h->force_eager = true;
  }
  void* pair_args[] = {&h->d_params, &h->d_state};
  CK(cudaLaunchKernel(k.init, dim3(init_grid), dim3(256), pair_args, 0, h->stream));
  {
    cudaGraphConditionalHandle none = 0;
    int zero = 0;
    void* rargs[] = {&h->d_params, &h->d_full, &h->d_state, &none, &zero};
    CK(cudaLaunchKernel(fp.rotate, dim3(fp.rotate_grid), dim3(kThreads), rargs, fp.smem_rotate,
                        h->stream));
  }
  for (int it = 0; it < P.maxiter; ++it) {
    if (h->profiling) CK(cudaEventRecord(h->ev[0], h->stream));
    CK(full_sweep(h->stream, fp, h->d_params, h->d_full, h->d_state, 0, 0));
    if (h->profiling) {
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
  if (h->profiling) CK(cudaEventRecord(h->ev[0], h->stream));
  CK(cudaLaunchKernel(k.finalize, dim3(fin_grid), dim3(kThreads), pair_args, smem_fin,
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
int solve_core(pmcmc_handle* h, const pmcmc_target* tg, const pmcmc_deer_params* p,
               const void* x0, uint64_t seed, uint64_t block0, int64_t N, void* S_out,
               void* logp_out, uint8_t* accept_out, int32_t mem, pmcmc_info* info,
               int64_t t_off = 0) {
  int rc = validate(h, tg, p);
  if (rc) return rc;
  if (!x0 || !S_out) return fail(h, PMCMC_ERR_ARGUMENT, "x0 and the output must not be NULL");
  if (mem != PMCMC_MEM_HOST && mem != PMCMC_MEM_DEVICE)
    return fail(h, PMCMC_ERR_ARGUMENT, "mem must be PMCMC_MEM_HOST or PMCMC_MEM_DEVICE");
  if (N < 1) return fail(h, PMCMC_ERR_ARGUMENT, "the number of samples must be >= 1");
  if (tg->kind == kLogistic) {
    if (p->jacobian == PMCMC_JAC_FULL)
      return fail(h, PMCMC_ERR_UNSUPPORTED, "logistic target: :full is not built");
    if (p->window > 0 && p->window < p->T)  // solve_blocks runs such blocks in chunks
      return fail(h, PMCMC_ERR_UNSUPPORTED, "logistic target: no sliding window");
  }
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
  const bool full = p->jacobian == PMCMC_JAC_FULL;
  FullPlan fplan;
  if (full) {
    if (f64) return fail(h, PMCMC_ERR_UNSUPPORTED, ":full is built for FP32 state");
    if (plain) return fail(h, PMCMC_ERR_UNSUPPORTED, ":full has no plain path");
    if (W < T) return fail(h, PMCMC_ERR_UNSUPPORTED, ":full has no sliding window");
    const int nch = h->full_chunks_override > 0 ? h->full_chunks_override
                    : h->tune_full_chunks > 0   ? h->tune_full_chunks
                                                : tune_get(TuneKey{1, tg->kind, p->jacobian, 0, D, T});
    if (!full_plan(Dp, T, tg->kind, h->num_sms, nch, &fplan))
      return fail(h, PMCMC_ERR_UNSUPPORTED, ":full is built for D <= 128, got %lld",
                  (long long)D);
    rc = ensure_eigen(h, const_cast<pmcmc_target*>(tg));
    if (rc) return rc;
  }
  const SweepKernels k = logistic ? logistic_sweep_kernels(f64, D, p->jacobian)
                                  : gauss_sweep_kernels(f64, tg->kind, p->jacobian, D);
  // whole solve in one cooperative launch when every tile is co-resident
  const int TTp = (!plain && !logistic && !full && W == T && !h->force_eager && !h->no_persist)
                      ? choose_persist_tile(h, k.persist, f64, Dp, T, dense,
                                            TuneKey{0, tg->kind, p->jacobian, f64, D, T})
                      : 0;
  const bool persist = TTp > 0;
  const TilePlan tp = full      ? TilePlan{}
                      : persist ? TilePlan{TTp, true}
                                : choose_tile(h, k, f64, Dp, W, dense);
  const int TT = tp.TT;
  const int ntiles = static_cast<int>((W + TT - 1) / TT);
  const SmemPlan sp_sweep = gauss_sweep_smem(f64, Dp, TT, dense);
  const SmemPlan sp_fin = gauss_sweep_smem(f64, Dp, 1, dense);
  if (sp_sweep.total > 200 * 1024)
    return fail(h, PMCMC_ERR_UNSUPPORTED, "dimension %lld too large for the fused sweep",
                (long long)D);
  // the exact diagonal contracts X .* X, which the tensor-core pass has no operand for
  const bool lg_diag = logistic && p->jacobian == PMCMC_JAC_DIAG;
  const bool use_tc = logistic && !plain && !f64 && !lg_diag && lg_tc_supported(tg->lg);
  if (lg_diag) {
    static std::mutex square_mu;  // targets are shared by the fleet's worker threads
    std::lock_guard<std::mutex> lk(square_mu);
    auto& lgd = const_cast<pmcmc_target*>(tg)->lg;
    CK(lg_make_square(h->stream, lgd, f64));
    CK(cudaStreamSynchronize(h->stream));
  }
  const int64_t Tc = logistic && !use_tc ? std::min<int64_t>(T, lg_chunk_cols(tg->N, T)) : 0;
  const int64_t nblocks = (N + T - 1) / T;
  // Host outputs of several blocks: block b's copy-out overlaps block b + 1's solve.
  const bool pipe = mem == PMCMC_MEM_HOST && nblocks > 1;
  // Several blocks: each block's state goes to a pinned ring, read after the last
  // block, so the blocks run back to back with no host round trip between them.
  const bool defer = nblocks > 1;
  // Device outputs of several blocks on the persistent path: one launch solves
  // them all, the kernel looping over the blocks (a grid barrier between blocks
  // instead of a kernel boundary).
  const bool batch = persist && mem == PMCMC_MEM_DEVICE && nblocks > 1;
  const SolveLayout L = layout(D, Dp, T, ntiles, es, plain, logistic ? tg->N : 0, Tc,
                               use_tc ? lg_tc_ws_bytes(tg->lg, T) : 0, full ? &fplan : nullptr,
                               false, pipe,
                               logistic ? lg_tie_ws_bytes(tg->lg, T, tie_kmax(T)) : 0);
  rc = ensure_ws(h, L.total);
  if (rc) return rc;
  if (defer) {
    rc = ensure_pipeline(h, nblocks);
    if (rc) return rc;
  }
  // copies still in flight into the caller's buffers end before any return
  struct CopyDrain {
    cudaStream_t s;
    ~CopyDrain() {
      if (s) cudaStreamSynchronize(s);
    }
  } drain{pipe ? h->copy_stream : nullptr};
  unsigned char* ws = h->ws;

  // x0 -> padded device buffer (x0a and x0b are adjacent: one memset clears both).
  // The persistent kernel pads x0 itself and reads a device x0 where it lies.
  if (!persist) CK(cudaMemsetAsync(ws + L.x0a, 0, L.x0b - L.x0a + es * Dp, h->stream));
  if (!persist || mem == PMCMC_MEM_HOST)
    CK(cudaMemcpyAsync(ws + L.x0a, x0, es * D,
                       mem == PMCMC_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                               : cudaMemcpyHostToDevice,
                       h->stream));

  DevParams P{};
  P.D = D;
  P.Dp = Dp;
  P.T = T;
  P.W = W;
  P.t_off = static_cast<int32_t>(t_off);  // tape column of local column 0 (a chunk of the block)
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
  P.part = reinterpret_cast<double*>(ws + L.part);
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
  FullArgs F{};
  if (full) {
    F.Pe = h->d_params_e;
    F.lam = tg->lam_f;
    F.Qrm = tg->qrm_f;
    F.Qcm = tg->qcm_f;
    F.lamQ = tg->lamq_f;
    F.QrmQ = tg->qrmq;
    F.QcmQ = tg->qcmq;
    F.U = reinterpret_cast<float*>(ws + L.fU);
    F.V = reinterpret_cast<float*>(ws + L.fV);
    F.R = reinterpret_cast<float*>(ws + L.fR);
    F.acc = ws + L.facc;
    F.Phi = reinterpret_cast<float*>(ws + L.fPhi);
    F.beta = reinterpret_cast<float*>(ws + L.fbeta);
    F.din = reinterpret_cast<float*>(ws + L.fdin);
    F.part = reinterpret_cast<double*>(ws + L.fpart);
    F.L = fplan.L;
    F.nchunks = fplan.nchunks;
    F.rot = dense ? 1 : 0;
    F.Dq = fplan.Dq;
  }

  const int fin_grid = static_cast<int>(std::min<int64_t>((T + kWarps - 1) / kWarps,
                                                          int64_t(h->num_sms) * 8));
  const int init_grid = static_cast<int>(
      std::min<int64_t>((T * (Dp / 4) + 255) / 256, int64_t(h->num_sms) * 8));
  std::vector<DevState> states(static_cast<size_t>(nblocks));
  int64_t nsteps = 0;
  for (int64_t b = 0; b < nblocks; ++b) {
    const int64_t nkeep = std::min<int64_t>(T, N - nsteps);
    const bool slot = pipe && (b & 1);
    const size_t oS = slot ? L.out2_S : L.out_S, olp = slot ? L.out2_lp : L.out_lp,
                 oacc = slot ? L.out2_acc : L.out_acc;
    P.block = block0 + static_cast<uint64_t>(b);
    P.x0 = ws + ((b & 1) ? L.x0b : L.x0a);
    P.x_next = ws + ((b & 1) ? L.x0a : L.x0b);
    P.ncols_out = nkeep;
    if (batch) {  // every block of the call in this launch; ncols_out: the last block's
      P.nblk = nblocks;
      P.ncols_out = N - (nblocks - 1) * T;
    }
    if (persist) {
      P.x0_src = (b == 0 && mem == PMCMC_MEM_DEVICE) ? x0 : P.x0;
      P.st_host = defer ? h->h_states + b : h->h_state;  // written by the kernel
    }
    if (mem == PMCMC_MEM_DEVICE) {
      P.S_out = static_cast<unsigned char*>(S_out) + es * nsteps * D;
      P.logp_out = logp_out ? static_cast<unsigned char*>(logp_out) + es * nsteps : nullptr;
      P.accept_out = accept_out ? accept_out + nsteps : nullptr;
    } else {
      P.S_out = ws + oS;
      P.logp_out = logp_out ? ws + olp : nullptr;
      P.accept_out = accept_out ? ws + oacc : nullptr;
    }
    // the slot's previous contents (block b - 2) must be copied out first
    if (pipe && b >= 2) CK(cudaStreamWaitEvent(h->stream, h->ev_copy[slot], 0));
    rc = logistic ? run_logistic(h, tg, k, tp.coop, P, L, es, sp_sweep.total, fin_grid,
                                 init_grid, Tc, use_tc, plain)
         : full   ? run_full(h, k, fplan, P, eigen_view(P, tg, ws, L), F, sp_fin.total,
                             fin_grid, init_grid)
         : plain   ? run_plain(h, k, P, L, es, sp_fin.total, fin_grid, init_grid)
         : persist ? run_persist(h, k, P, persist_smem(f64, Dp, TT, dense).total,
                                 batch ? nblocks : 1)
                   : run_fused(h, k, tp.coop, P, sp_sweep.total, sp_fin.total, fin_grid,
                               init_grid);
    if (rc) return rc;
    if (mem == PMCMC_MEM_HOST) {
      cudaStream_t cs = h->stream;
      if (pipe) {
        CK(cudaEventRecord(h->ev_fin[slot], h->stream));
        CK(cudaStreamWaitEvent(h->copy_stream, h->ev_fin[slot], 0));
        cs = h->copy_stream;
      }
      CK(cudaMemcpyAsync(static_cast<unsigned char*>(S_out) + es * nsteps * D, ws + oS,
                         es * nkeep * D, cudaMemcpyDeviceToHost, cs));
      if (logp_out)
        CK(cudaMemcpyAsync(static_cast<unsigned char*>(logp_out) + es * nsteps, ws + olp,
                           es * nkeep, cudaMemcpyDeviceToHost, cs));
      if (accept_out)
        CK(cudaMemcpyAsync(accept_out + nsteps, ws + oacc, nkeep, cudaMemcpyDeviceToHost, cs));
      if (pipe) CK(cudaEventRecord(h->ev_copy[slot], cs));
    }
    nsteps += nkeep;
    if (batch) {  // the launch solved every block
      nsteps = N;
      break;
    }
    if (defer) {  // block states are read after the last block
      if (!persist)
        CK(cudaMemcpyAsync(h->h_states + b, h->d_state, sizeof(DevState),
                           cudaMemcpyDeviceToHost, h->stream));
      continue;
    }
    if (!persist)
      CK(cudaMemcpyAsync(h->h_state, h->d_state, sizeof(DevState), cudaMemcpyDeviceToHost,
                         h->stream));
    CK(cudaStreamSynchronize(h->stream));
    states[static_cast<size_t>(b)] = *h->h_state;
    if (h->h_state->status) break;
  }
  if (defer) {
    CK(cudaStreamSynchronize(h->stream));
    if (pipe) CK(cudaStreamSynchronize(h->copy_stream));
    for (int64_t b = 0; b < nblocks; ++b) {
      states[static_cast<size_t>(b)] = h->h_states[b];
      if (h->h_states[b].status) {  // the blocks after a failed one do not count
        states.resize(static_cast<size_t>(b + 1));
        break;
      }
    }
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
  // the plain logistic path keeps the last sweep's flags and verifies nothing
  if (logistic && plain) agg.max_defect = NAN;
  agg.path = (plain || full ? 0 : PMCMC_PATH_FUSED_SWEEP) |
             (tp.coop && !plain && !full ? PMCMC_PATH_COOPERATIVE : 0) |
             (!plain && !logistic && !persist && !h->force_eager && !h->profiling
                  ? PMCMC_PATH_GRAPH
                  : 0) |
             (persist ? PMCMC_PATH_PERSISTENT : 0) |
             (use_tc ? PMCMC_PATH_TENSOR_CORE : 0) | (full ? PMCMC_PATH_FULL_JACOBIAN : 0) |
             (logistic && !plain && !f64 ? PMCMC_PATH_TIE_FP64 : 0);
  if (info) *info = agg;
  return status_error(h, status);
}

// A mass-matrix target (M = L L^T, the reference's cholM) is stored as the
// whitened Gaussian x' = L^-1 x.  MALA with mass M is plain MALA on the
// whitened target with the same tape and the same log alpha (src/MALA/MALA.jl:
// 29-47 applies L, L^T and L \ inside every step), so the Newton solve runs in
// whitened coordinates: x0 is whitened once on the device, the solve writes to
// device memory, every column maps back as S = L S' in place, and host outputs
// are copied out last.  log p and the accept flags are coordinate-free; the
// defects in `info` are in whitened coordinates.
int solve_mass(pmcmc_handle* h, const pmcmc_target* tg, const pmcmc_deer_params* p,
               const void* x0, uint64_t seed, uint64_t block0, int64_t N, void* S_out,
               void* logp_out, uint8_t* accept_out, int32_t mem, pmcmc_info* info) {
  int rc = validate(h, tg, p);
  if (rc) return rc;
  if (!x0 || !S_out) return fail(h, PMCMC_ERR_ARGUMENT, "x0 and the output must not be NULL");
  if (mem != PMCMC_MEM_HOST && mem != PMCMC_MEM_DEVICE)
    return fail(h, PMCMC_ERR_ARGUMENT, "mem must be PMCMC_MEM_HOST or PMCMC_MEM_DEVICE");
  if (N < 1) return fail(h, PMCMC_ERR_ARGUMENT, "the number of samples must be >= 1");
  DeviceGuard guard(h->device);
  const bool f64 = p->dtype == PMCMC_F64;
  const size_t es = f64 ? 8 : 4;
  const int64_t D = tg->D;
  const bool host = mem == PMCMC_MEM_HOST;
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t bx = up(es * D), bS = host ? up(es * N * D) : 0,
               blp = host && logp_out ? up(es * N) : 0, bac = host && accept_out ? up(N) : 0;
  // stream-ordered scratch: freeing it does not wait for the device (fleet workers
  // on other streams keep running)
  struct Scratch {
    void* buf = nullptr;
    cudaStream_t s = nullptr;
    ~Scratch() {
      if (buf) cudaFreeAsync(buf, s);
    }
  } sc;
  sc.s = h->stream;
  CK(cudaMallocAsync(&sc.buf, 2 * bx + bS + blp + bac, h->stream));
  unsigned char* b = static_cast<unsigned char*>(sc.buf);
  CK(cudaMemcpyAsync(b, x0, es * D, host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                     h->stream));
  CK(mass_whiten(h->stream, tg->mass_Ld, D, 1, b, b + bx, f64));
  void* S = host ? b + 2 * bx : S_out;
  void* lp = host ? (logp_out ? b + 2 * bx + bS : nullptr) : logp_out;
  uint8_t* ac = host ? (accept_out ? b + 2 * bx + bS + blp : nullptr) : accept_out;
  rc = solve_core(h, tg, p, b + bx, seed, block0, N, S, lp, ac, PMCMC_MEM_DEVICE, info);
  if (rc) return rc;
  CK(mass_map(h->stream, tg->mass_Ld, D, N, S, f64, h->num_sms));
  if (host) {
    CK(cudaMemcpyAsync(S_out, S, es * N * D, cudaMemcpyDeviceToHost, h->stream));
    if (logp_out) CK(cudaMemcpyAsync(logp_out, lp, es * N, cudaMemcpyDeviceToHost, h->stream));
    if (accept_out)
      CK(cudaMemcpyAsync(accept_out, ac, N, cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return PMCMC_OK;
}

// Logistic target with a window W < T: every block is solved as consecutive
// chunks of W columns, chunk k a DEER solve of its own from the last state of
// chunk k - 1 on tape columns [k W, k W + W) of the block (the tape, the
// uniforms and the probes are drawn at the block's column index).  The chain is
// Markov, so the chunks' fixed points together are the block's: the same
// sequential chain.  Each chunk's Newton solve sees only W columns, and the
// number of sweeps a DEER solve needs grows with its length.  The info adds the
// chunks' sweeps and accepts and keeps the worst metric, margin and defect.
int solve_chunks(pmcmc_handle* h, const pmcmc_target* tg, const pmcmc_deer_params* p,
                 const void* x0, uint64_t seed, uint64_t block0, int64_t N, void* S_out,
                 void* logp_out, uint8_t* accept_out, int32_t mem, pmcmc_info* info) {
  int rc = validate(h, tg, p);
  if (rc) return rc;
  if (!x0 || !S_out) return fail(h, PMCMC_ERR_ARGUMENT, "x0 and the output must not be NULL");
  if (N < 1) return fail(h, PMCMC_ERR_ARGUMENT, "the number of samples must be >= 1");
  const size_t es = p->dtype == PMCMC_F64 ? 8 : 4;
  const int64_t T = p->T, W = p->window, D = tg->D;
  const int64_t nblocks = (N + T - 1) / T;
  pmcmc_info agg{};
  agg.converged = 1;
  agg.min_margin = INFINITY;
  const unsigned char* xprev = static_cast<const unsigned char*>(x0);
  unsigned char* S = static_cast<unsigned char*>(S_out);
  unsigned char* lp = static_cast<unsigned char*>(logp_out);
  rc = PMCMC_OK;
  for (int64_t b = 0; b < nblocks && rc == PMCMC_OK; ++b) {
    const int64_t nkeep = std::min(T, N - b * T);
    for (int64_t t0 = 0; t0 < nkeep && rc == PMCMC_OK; t0 += W) {
      pmcmc_deer_params pc = *p;
      pc.T = std::min(W, T - t0);
      pc.window = 0;
      const int64_t keep = std::min(pc.T, nkeep - t0), col = b * T + t0;
      pmcmc_info ci{};
      rc = solve_core(h, tg, &pc, xprev, seed, block0 + static_cast<uint64_t>(b), keep,
                      S + es * col * D, lp ? lp + es * col : nullptr,
                      accept_out ? accept_out + col : nullptr, mem, &ci, t0);
      agg.iters += ci.iters;
      agg.converged &= ci.converged;
      agg.metric = std::isnan(ci.metric) ? ci.metric : std::max(agg.metric, ci.metric);
      agg.n_accept += ci.n_accept;
      agg.min_margin = std::min(agg.min_margin, ci.min_margin);
      agg.max_defect = std::isnan(ci.max_defect) ? ci.max_defect
                                                 : std::max(agg.max_defect, ci.max_defect);
      if (ci.status && !agg.status) agg.status = ci.status;
      agg.path |= ci.path;
      xprev = S + es * (col + keep - 1) * D;  // the next chunk starts from this one's end
    }
  }
  if (info) *info = agg;
  return rc;
}

int solve_blocks(pmcmc_handle* h, const pmcmc_target* tg, const pmcmc_deer_params* p,
                 const void* x0, uint64_t seed, uint64_t block0, int64_t N, void* S_out,
                 void* logp_out, uint8_t* accept_out, int32_t mem, pmcmc_info* info) {
  if (tg && tg->mass_Ld)
    return solve_mass(h, tg, p, x0, seed, block0, N, S_out, logp_out, accept_out, mem, info);
  if (tg && p && tg->kind == kLogistic && p->window > 0 && p->window < p->T)
    return solve_chunks(h, tg, p, x0, seed, block0, N, S_out, logp_out, accept_out, mem, info);
  return solve_core(h, tg, p, x0, seed, block0, N, S_out, logp_out, accept_out, mem, info);
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
  t->prec_host.assign(prec, prec + (kind == kDenseGauss ? D * D : D));
  t->mean_host.assign(md.begin(), md.begin() + D);
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
      cudaMallocHost(&h->h_red, 4 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&h->d_full, sizeof(FullArgs)) != cudaSuccess ||
      cudaMalloc(&h->d_params_e, sizeof(DevParams)) != cudaSuccess) {
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
  const char* nv = std::getenv("PMCMC_NO_PERSIST");
  h->no_persist = nv && nv[0] == '1';
  const char* tv = std::getenv("PMCMC_TILE_COLS");
  h->tile_override = tv ? std::atoi(tv) : 0;
  const char* fv = std::getenv("PMCMC_FULL_CHUNKS");
  h->full_chunks_override = fv ? std::atoi(fv) : 0;
  // profiler runs: every Newton loop eager, one launch per real sweep
  const char* pv = std::getenv("PMCMC_PROFILE");
  if (pv && pv[0] == '1' &&
      (cudaEventCreate(&h->ev[0]) != cudaSuccess || cudaEventCreate(&h->ev[1]) != cudaSuccess)) {
    cudaGetLastError();
    pmcmc_destroy(h);
    return PMCMC_ERR_CUDA;
  }
  h->profiling = pv && pv[0] == '1';
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
  if (h->gexec_full) cudaGraphExecDestroy(h->gexec_full);
  for (pmcmc_handle* w : h->fleet) pmcmc_destroy(w);
  if (h->copy_stream) {
    cudaStreamSynchronize(h->copy_stream);
    cudaStreamDestroy(h->copy_stream);
  }
  for (int i = 0; i < 2; ++i) {
    if (h->ev_fin[i]) cudaEventDestroy(h->ev_fin[i]);
    if (h->ev_copy[i]) cudaEventDestroy(h->ev_copy[i]);
  }
  if (h->h_states) cudaFreeHost(h->h_states);
  if (h->cublas) cublasDestroy(h->cublas);
  cudaFree(h->cublas_ws);
  cudaFree(h->d_full);
  cudaFree(h->d_params_e);
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

int pmcmc_check_wait_bound(pmcmc_handle* h, int32_t kind, double* wait_ms) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  if (kind != PMCMC_WAIT_LOOKBACK && kind != PMCMC_WAIT_MBARRIER)
    return fail(h, PMCMC_ERR_ARGUMENT, "kind must be PMCMC_WAIT_LOOKBACK or PMCMC_WAIT_MBARRIER");
  DeviceGuard guard(h->device);
  struct Scratch {
    void* buf = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~Scratch() {
      cudaFree(buf);  // synchronises the device first
      for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    }
  } sc;
  CK(cudaMalloc(&sc.buf, 256));
  CK(cudaEventCreate(&sc.ev[0]));
  CK(cudaEventCreate(&sc.ev[1]));
  uint32_t* flags = static_cast<uint32_t*>(sc.buf);                    // 32 zero words
  int* err = reinterpret_cast<int*>(static_cast<char*>(sc.buf) + 128);  // out
  CK(cudaMemsetAsync(sc.buf, 0, 256, h->stream));
  CK(cudaEventRecord(sc.ev[0], h->stream));
  if (kind == PMCMC_WAIT_LOOKBACK)
    CK(launch_lookback_bound(h->stream, flags, err));
  else
    CK(lg_tc_mbar_bound(h->stream, err));
  CK(cudaEventRecord(sc.ev[1], h->stream));
  int gave_up = 0;
  CK(cudaMemcpyAsync(&gave_up, err, sizeof gave_up, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, sc.ev[0], sc.ev[1]));
  if (wait_ms) *wait_ms = ms;
  if (!gave_up) return PMCMC_OK;
  return fail(h, PMCMC_ERR_TIMEOUT, "%s wait reached its bound after %.1f ms",
              kind == PMCMC_WAIT_LOOKBACK ? "look-back" : "mbarrier", ms);
}

int pmcmc_target_diag_gauss(pmcmc_handle* h, int64_t D, const double* mean, const double* prec,
                            pmcmc_target** out) {
  return make_target(h, kDiagGauss, D, mean, prec, out);
}

int pmcmc_target_dense_gauss(pmcmc_handle* h, int64_t D, const double* mean, const double* prec,
                             pmcmc_target** out) {
  return make_target(h, kDenseGauss, D, mean, prec, out);
}

// The reference's cholM = cholesky(M) on MALASampler / ParallelMALASampler /
// AdaptiveMALASampler (src/interface.jl:84-100, 241-287, 899-930), applied by
// MALA.jl's _apply_M!, _apply_L!, _quad_Minv! and _logdet_M (src/MALA/MALA.jl:
// 29-47).  The new target is the base Gaussian in whitened coordinates
// x' = L^-1 x: precision L^T P L, mean L^-1 mu; it keeps L to map chains back.
int pmcmc_target_mass(pmcmc_handle* h, const pmcmc_target* base, const double* L,
                      pmcmc_target** out) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  if (!out) return fail(h, PMCMC_ERR_ARGUMENT, "out must not be NULL");
  if (!base || !L) return fail(h, PMCMC_ERR_ARGUMENT, "base target and L must not be NULL");
  if (base->kind == kLogistic)
    return fail(h, PMCMC_ERR_UNSUPPORTED, "mass matrix: built for Gaussian targets");
  if (base->mass_Ld)
    return fail(h, PMCMC_ERR_ARGUMENT, "base target already carries a mass matrix");
  const int64_t D = base->D;
  if (D > mass_max_dim())
    return fail(h, PMCMC_ERR_UNSUPPORTED, "mass matrix: built for D <= %lld",
                (long long)mass_max_dim());
  const size_t DD = static_cast<size_t>(D) * D;
  std::vector<double> Lc(DD, 0.0);  // lower triangle only
  for (int64_t j = 0; j < D; ++j) {
    if (!(L[j * D + j] > 0) || !std::isfinite(L[j * D + j]))
      return fail(h, PMCMC_ERR_ARGUMENT, "L must have a positive diagonal (L[%lld,%lld] = %g)",
                  (long long)j, (long long)j, L[j * D + j]);
    for (int64_t i = j; i < D; ++i) {
      if (!std::isfinite(L[j * D + i]))
        return fail(h, PMCMC_ERR_ARGUMENT, "L has a non-finite entry");
      Lc[j * D + i] = L[j * D + i];
    }
  }
  // P L (column j of L is zero above row j), then L^T (P L), symmetrised
  const bool dense = base->kind == kDenseGauss;
  const std::vector<double>& P = base->prec_host;
  std::vector<double> PL(DD, 0.0), Pw(DD, 0.0);
  for (int64_t j = 0; j < D; ++j)
    for (int64_t k = j; k < D; ++k) {
      const double l = Lc[j * D + k];
      if (dense)
        for (int64_t i = 0; i < D; ++i) PL[j * D + i] += P[k * D + i] * l;
      else
        PL[j * D + k] += P[k] * l;
    }
  for (int64_t j = 0; j < D; ++j)
    for (int64_t i = 0; i <= j; ++i) {
      double acc = 0.0;
      for (int64_t k = i; k < D; ++k) acc += Lc[i * D + k] * PL[j * D + k];
      Pw[j * D + i] = acc;
    }
  for (int64_t j = 0; j < D; ++j)
    for (int64_t i = j + 1; i < D; ++i) Pw[j * D + i] = Pw[i * D + j];
  // mu' = L^-1 mu (forward substitution)
  std::vector<double> mw(static_cast<size_t>(D));
  for (int64_t i = 0; i < D; ++i) {
    double r = base->mean_host[i];
    for (int64_t k = 0; k < i; ++k) r -= Lc[k * D + i] * mw[k];
    mw[i] = r / Lc[i * D + i];
  }
  pmcmc_target* t = nullptr;
  int rc = make_target(h, kDenseGauss, D, mw.data(), Pw.data(), &t);
  if (rc) return rc;
  DeviceGuard guard(h->device);
  t->mass_L = std::move(Lc);
  cudaError_t e = cudaMalloc(&t->mass_Ld, 8 * DD);
  if (e == cudaSuccess)
    e = cudaMemcpy(t->mass_Ld, t->mass_L.data(), 8 * DD, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaGetLastError();
    pmcmc_target_destroy(t);
    return fail(h, e == cudaErrorMemoryAllocation ? PMCMC_ERR_NOMEM : PMCMC_ERR_CUDA,
                "mass matrix upload failed: %s", cudaGetErrorString(e));
  }
  *out = t;
  return PMCMC_OK;
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
  if (e == cudaSuccess && D <= 512) {
    // FP16 hi + lo operands for the tensor-core pass (Dk = 512: its wide variant)
    const int64_t Dk = D <= 128 ? 128 : D <= 256 ? 256 : 512;
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
  cudaFree(t->lg.X2_32);
  cudaFree(t->lg.X2_64);
  cudaFree(t->mass_Ld);
  for (void* q : {static_cast<void*>(t->lam_f), static_cast<void*>(t->qrm_f),
                  static_cast<void*>(t->qcm_f), static_cast<void*>(t->lamq_f),
                  static_cast<void*>(t->lamq_d), static_cast<void*>(t->zq_f),
                  static_cast<void*>(t->zq_d), static_cast<void*>(t->qrmq),
                  static_cast<void*>(t->qcmq)})
    cudaFree(q);
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

int pmcmc_autotune(pmcmc_handle* h, const pmcmc_target* tg, const pmcmc_deer_params* p,
                   const void* x0, uint64_t seed, int32_t mem, int32_t* choice,
                   double* best_ms) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  int rc = validate(h, tg, p);
  if (rc) return rc;
  if (!x0) return fail(h, PMCMC_ERR_ARGUMENT, "x0 must not be NULL");
  if (mem != PMCMC_MEM_HOST && mem != PMCMC_MEM_DEVICE)
    return fail(h, PMCMC_ERR_ARGUMENT, "mem must be PMCMC_MEM_HOST or PMCMC_MEM_DEVICE");
  DeviceGuard guard(h->device);
  const bool f64 = p->dtype == PMCMC_F64;
  const size_t es = f64 ? 8 : 4;
  const int64_t D = tg->D, T = p->T;
  const bool full = p->jacobian == PMCMC_JAC_FULL;
  const bool windowed = p->window > 0 && p->window < T;
  std::vector<int> cands;
  TuneKey key{};
  if (full) {
    key = TuneKey{1, tg->kind, p->jacobian, 0, D, T};
    for (double f : {0.5, 1.0, 2.0, 4.0}) {
      const int n = std::max(1, std::min(h->num_sms, static_cast<int>(std::sqrt(f * T) + 0.5)));
      if (std::find(cands.begin(), cands.end(), n) == cands.end()) cands.push_back(n);
    }
  } else if (p->exec != PMCMC_EXEC_PLAIN && tg->kind != kLogistic && !windowed &&
             !h->force_eager && !h->no_persist && !h->no_coop && h->tile_override == 0) {
    key = TuneKey{0, tg->kind, p->jacobian, f64, D, T};
    const SweepKernels k = gauss_sweep_kernels(f64, tg->kind, p->jacobian, D);
    for (int per_sm = 1; per_sm <= 4; ++per_sm)
      if (persist_tile_for(k.persist, f64, tg->Dp, T, tg->kind == kDenseGauss, per_sm,
                           h->num_sms) > 0)
        cands.push_back(per_sm);
  }
  if (choice) *choice = cands.empty() ? 0 : cands.front();
  if (best_ms) *best_ms = 0.0;
  if (cands.size() < 2) return PMCMC_OK;  // nothing to choose between

  struct Scratch {
    void* buf = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    pmcmc_handle* h = nullptr;
    ~Scratch() {
      if (h) h->tune_per_sm = h->tune_full_chunks = 0;
      cudaFree(buf);
      for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    }
  } sc;
  sc.h = h;
  const size_t bx = (es * D + 255) & ~size_t(255), bS = (es * T * D + 255) & ~size_t(255),
               blp = (es * T + 255) & ~size_t(255);
  CK(cudaMalloc(&sc.buf, bx + bS + blp + static_cast<size_t>(T)));
  CK(cudaEventCreate(&sc.ev[0]));
  CK(cudaEventCreate(&sc.ev[1]));
  unsigned char* b = static_cast<unsigned char*>(sc.buf);
  CK(cudaMemcpyAsync(b, x0, es * D,
                     mem == PMCMC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     h->stream));
  int best = cands.front();
  double best_t = INFINITY;
  for (const int c : cands) {
    if (full) h->tune_full_chunks = c;
    else h->tune_per_sm = c;
    double t_min = INFINITY;
    for (int rep = 0; rep < 3; ++rep) {  // the first run builds graphs and warms caches
      pmcmc_info info{};
      CK(cudaEventRecord(sc.ev[0], h->stream));
      rc = solve_blocks(h, tg, p, b, seed, 0, T, b + bx, b + bx + bS, b + bx + bS + blp,
                        PMCMC_MEM_DEVICE, &info);
      if (rc) return rc;
      CK(cudaEventRecord(sc.ev[1], h->stream));
      CK(cudaEventSynchronize(sc.ev[1]));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, sc.ev[0], sc.ev[1]));
      if (rep > 0) t_min = std::min(t_min, static_cast<double>(ms));
    }
    if (t_min < best_t) {
      best_t = t_min;
      best = c;
    }
  }
  tune_put(key, best);
  if (choice) *choice = best;
  if (best_ms) *best_ms = best_t;
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

// Fleet: many independent chains of uneven size on one GPU.  Worker handles
// (each with its own stream and workspace) take chains from a queue ordered by
// estimated cost, largest first, so that small chains fill the device while
// the large ones run; every chain keeps its own Newton loop and convergence
// test.  The reference runs independent chains through AbstractMCMC's
// MCMCThreads, one chain per Julia thread (test/test-DEER-Interface.jl:300-318).
int pmcmc_fleet_solve(pmcmc_handle* h, pmcmc_fleet_chain* chains, int64_t n, int32_t workers,
                      int32_t mem) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  if (n < 0 || (n > 0 && !chains)) return fail(h, PMCMC_ERR_ARGUMENT, "null chain array");
  if (workers < 1 || workers > 64) return fail(h, PMCMC_ERR_ARGUMENT, "workers must be in [1, 64]");
  if (n == 0) return PMCMC_OK;
  DeviceGuard guard(h->device);
  CK(cudaStreamSynchronize(h->stream));
  while (static_cast<int>(h->fleet.size()) < workers) {
    pmcmc_handle* w = nullptr;
    const int rc = pmcmc_create(h->device, nullptr, &w);
    if (rc) return fail(h, rc, "fleet worker handle creation failed");
    h->fleet.push_back(w);
  }
  std::vector<int64_t> order(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) order[i] = i;
  auto cost = [&](int64_t i) {
    const pmcmc_fleet_chain& c = chains[i];
    const double D = c.target ? static_cast<double>(c.target->D) : 0.0;
    const double N = c.target && c.target->kind == kLogistic ? static_cast<double>(c.target->N) : 1.0;
    return D * N * static_cast<double>(c.params.T);
  };
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cost(a) > cost(b); });
  std::atomic<int64_t> next{0};
  std::vector<std::string> msg(static_cast<size_t>(n));
  auto work = [&](pmcmc_handle* w) {
    DeviceGuard g(w->device);
    for (int64_t k = next.fetch_add(1); k < n; k = next.fetch_add(1)) {
      pmcmc_fleet_chain& c = chains[order[k]];
      c.info = pmcmc_info{};
      c.status = c.target ? solve_blocks(w, c.target, &c.params, c.x0, c.seed, c.block,
                                         c.params.T, c.S_out, c.logp_out, c.accept_out, mem,
                                         &c.info)
                          : PMCMC_ERR_ARGUMENT;
      if (c.status) msg[static_cast<size_t>(order[k])] = c.target ? w->err : "null target";
    }
  };
  std::vector<std::thread> pool;
  for (int i = 0; i < workers; ++i) pool.emplace_back(work, h->fleet[static_cast<size_t>(i)]);
  for (std::thread& t : pool) t.join();
  for (int64_t i = 0; i < n; ++i)
    if (chains[i].status)
      return fail(h, chains[i].status, "fleet chain %lld: %s", (long long)i,
                  msg[static_cast<size_t>(i)].c_str());
  return PMCMC_OK;
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

namespace {

// Sequential chains, fixed or adaptive step size (ad == nullptr: fixed).
int chains_impl(pmcmc_handle* h, const pmcmc_target* tg, const pmcmc_deer_params* p, int64_t n,
                const void* x0, const uint64_t* seeds, uint64_t block, const pmcmc_adapt* ad,
                void* S_out, void* logp_out, uint8_t* accept_out, double* eps_out,
                double* state_out, int32_t mem) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  int rc = validate(h, tg, p);
  if (rc) return rc;
  if (!x0 || !seeds || !S_out)
    return fail(h, PMCMC_ERR_ARGUMENT, "x0, seeds and S_out must not be NULL");
  if (n < 1) return fail(h, PMCMC_ERR_ARGUMENT, "the number of chains must be >= 1");
  if (mem != PMCMC_MEM_HOST && mem != PMCMC_MEM_DEVICE)
    return fail(h, PMCMC_ERR_ARGUMENT, "mem must be PMCMC_MEM_HOST or PMCMC_MEM_DEVICE");
  if (tg->kind == kLogistic)
    return fail(h, PMCMC_ERR_UNSUPPORTED, "sequential chains are built for Gaussian targets");
  DeviceGuard guard(h->device);
  const bool f64 = p->dtype == PMCMC_F64;
  const size_t es = f64 ? 8 : 4;
  const int64_t D = tg->D, T = p->T;
  if (mala_chains_smem(f64, tg->Dp, tg->kind == kDenseGauss) > 200 * 1024)
    return fail(h, PMCMC_ERR_UNSUPPORTED, "dimension %lld too large for the chain kernel",
                (long long)D);
  DevParams P{};
  P.D = D;
  P.Dp = tg->Dp;
  P.T = T;
  P.W = T;
  P.eps = p->epsilon;
  P.sqrt2eps = std::sqrt(2 * p->epsilon);
  P.inv4eps = 1.0 / (4 * p->epsilon);
  P.inv2eps = 1.0 / (2 * p->epsilon);
  P.block = block;
  P.tkind = tg->kind;
  P.mean_d = tg->mean_d;
  P.prec_d = tg->prec_d;
  P.mean_f = tg->mean_f;
  P.prec_f = tg->prec_f;
  ChainAdapt cad{};
  if (ad) {
    // AdaptiveMALASampler's checks (src/interface.jl:919-923)
    if (!(ad->target_accept > 0 && ad->target_accept < 1))
      return fail(h, PMCMC_ERR_ARGUMENT, "target_accept must be in (0,1), got %g",
                  ad->target_accept);
    if (!(ad->gamma > 0)) return fail(h, PMCMC_ERR_ARGUMENT, "gamma must be > 0, got %g", ad->gamma);
    if (!(ad->t0 > 0)) return fail(h, PMCMC_ERR_ARGUMENT, "t0 must be > 0, got %g", ad->t0);
    if (!(ad->kappa > 0.5 && ad->kappa <= 1.0))
      return fail(h, PMCMC_ERR_ARGUMENT, "kappa must be in (0.5, 1], got %g", ad->kappa);
    if (ad->n_warmup < 0) return fail(h, PMCMC_ERR_ARGUMENT, "n_warmup must be >= 0");
    cad = ChainAdapt{1, ad->n_warmup, ad->target_accept, ad->gamma, ad->t0, ad->kappa};
  }
  const void* dx0 = x0;
  const uint64_t* dseeds = seeds;
  void *dS = S_out, *dlp = logp_out;
  uint8_t* dacc = accept_out;
  double *deps = eps_out, *dst = state_out;
  const size_t bx = es * n * D, bs = 8 * static_cast<size_t>(n), bS = es * n * T * D,
               blp = logp_out ? es * n * T : 0, bacc = accept_out ? n * T : 0,
               beps = eps_out ? 8 * n * T : 0, bst = state_out ? 24 * static_cast<size_t>(n) : 0;
  // mass-matrix targets: the chains run whitened from x0' = L^-1 x0 (the
  // solve's whitening, solve_mass), and map back in place after the launch
  const bool mass = tg->mass_Ld != nullptr;
  auto a = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t bw = mass ? a(bx) : 0;
  if (mem == PMCMC_MEM_HOST) {
    rc = ensure_ws(h, bw + a(bx) + a(bs) + a(bS) + a(blp) + a(bacc) + a(beps) + a(bst));
    if (rc) return rc;
    unsigned char* w = h->ws + bw;
    dx0 = w;
    dseeds = reinterpret_cast<const uint64_t*>(w + a(bx));
    dS = w + a(bx) + a(bs);
    dlp = logp_out ? w + a(bx) + a(bs) + a(bS) : nullptr;
    dacc = accept_out ? w + a(bx) + a(bs) + a(bS) + a(blp) : nullptr;
    unsigned char* w2 = w + a(bx) + a(bs) + a(bS) + a(blp) + a(bacc);
    deps = eps_out ? reinterpret_cast<double*>(w2) : nullptr;
    dst = state_out ? reinterpret_cast<double*>(w2 + a(beps)) : nullptr;
    CK(cudaMemcpyAsync(const_cast<void*>(dx0), x0, bx, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(const_cast<uint64_t*>(dseeds), seeds, bs, cudaMemcpyHostToDevice,
                       h->stream));
  } else if (mass) {
    rc = ensure_ws(h, bw);
    if (rc) return rc;
  }
  if (mass) {
    CK(mass_whiten(h->stream, tg->mass_Ld, D, n, dx0, h->ws, f64));
    dx0 = h->ws;
  }
  CK(launch_mala_chains(h->stream, f64, tg->kind, P, cad, n, dx0, dseeds, dS, dlp, dacc, deps,
                        dst));
  if (mass) CK(mass_map(h->stream, tg->mass_Ld, D, n * T, dS, f64, h->num_sms));
  if (mem == PMCMC_MEM_HOST) {
    CK(cudaMemcpyAsync(S_out, dS, bS, cudaMemcpyDeviceToHost, h->stream));
    if (logp_out) CK(cudaMemcpyAsync(logp_out, dlp, blp, cudaMemcpyDeviceToHost, h->stream));
    if (accept_out)
      CK(cudaMemcpyAsync(accept_out, dacc, bacc, cudaMemcpyDeviceToHost, h->stream));
    if (eps_out) CK(cudaMemcpyAsync(eps_out, deps, beps, cudaMemcpyDeviceToHost, h->stream));
    if (state_out) CK(cudaMemcpyAsync(state_out, dst, bst, cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return PMCMC_OK;
}

}  // namespace

extern "C" {

int pmcmc_mala_chains(pmcmc_handle* h, const pmcmc_target* tg, const pmcmc_deer_params* p,
                      int64_t n, const void* x0, const uint64_t* seeds, uint64_t block,
                      void* S_out, void* logp_out, uint8_t* accept_out, int32_t mem) {
  return chains_impl(h, tg, p, n, x0, seeds, block, nullptr, S_out, logp_out, accept_out, nullptr,
                     nullptr, mem);
}

int pmcmc_mala_chains_adaptive(pmcmc_handle* h, const pmcmc_target* tg,
                               const pmcmc_deer_params* p, int64_t n, const void* x0,
                               const uint64_t* seeds, uint64_t block, const pmcmc_adapt* ad,
                               void* S_out, void* logp_out, uint8_t* accept_out,
                               double* eps_out, double* state_out, int32_t mem) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  if (!ad) return fail(h, PMCMC_ERR_ARGUMENT, "adaptation settings must not be NULL");
  return chains_impl(h, tg, p, n, x0, seeds, block, ad, S_out, logp_out, accept_out, eps_out,
                     state_out, mem);
}

int pmcmc_target_eigen(pmcmc_target* t, double* lam, double* Q) {
  if (!t || !lam) return PMCMC_ERR_ARGUMENT;
  const int rc = ensure_eigen(t->h, t);
  if (rc) return rc;
  std::memcpy(lam, t->eig_lam.data(), sizeof(double) * t->D);
  if (Q) std::memcpy(Q, t->eig_Q.data(), sizeof(double) * t->D * t->D);
  return PMCMC_OK;
}

}  // extern "C"

namespace {

int scan_device(void* ctx, int64_t D, int64_t T, const double* A, const double* B,
                const double* s0, double* S) {
  return pmcmc_affine_scan_diag(static_cast<pmcmc_handle*>(ctx), PMCMC_F64, D, T, A, B, s0, S,
                                PMCMC_MEM_DEVICE);
}

// The logistic adjoint (logistic_adjoint.cu): x0 and S staged on the device,
// X .* X made on first use, the Jacobi iterations capped at p->maxiter.
int adjoint_logistic(pmcmc_handle* h, const pmcmc_target* tg, const pmcmc_deer_params* p,
                     const void* x0, uint64_t seed, uint64_t block, const void* S, int32_t mem,
                     int32_t objective, double* grad) {
  DeviceGuard guard(h->device);
  const bool f64 = p->dtype == PMCMC_F64;
  const size_t es = f64 ? 8 : 4;
  const int64_t D = tg->D, T = p->T;
  int rc = ensure_cublas(h);
  if (rc) return rc;
  {
    static std::mutex square_mu;  // targets are shared across handles
    std::lock_guard<std::mutex> lk(square_mu);
    CK(lg_make_square(h->stream, const_cast<pmcmc_target*>(tg)->lg, true));
    CK(cudaStreamSynchronize(h->stream));
  }
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t bx = up(es * D), bS = up(es * T * D);
  rc = ensure_ws(h, bx + bS + lg_adjoint_ws_bytes(tg->lg, T));
  if (rc) return rc;
  unsigned char* ws = h->ws;
  const cudaMemcpyKind kin =
      mem == PMCMC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CK(cudaMemcpyAsync(ws, x0, es * D, kin, h->stream));
  CK(cudaMemcpyAsync(ws + bx, S, es * T * D, kin, h->stream));
  double g = 0.0;
  int iters = 0;
  rc = lg_adjoint(h->stream, h->cublas, tg->lg, f64, ws, ws + bx, seed, block, T, p->epsilon,
                  objective == PMCMC_OBJ_ESJD, ws + bx + bS, p->maxiter, &g, &iters, scan_device,
                  h);
  if (rc == 3) return fail(h, PMCMC_ERR_CUDA, "logistic adjoint: a CUDA or cuBLAS call failed");
  if (rc == 4) return fail(h, PMCMC_ERR_NONFINITE, "logistic adjoint: non-finite lambda");
  if (rc == 5)
    return fail(h, PMCMC_ERR_TIMEOUT,
                "logistic adjoint: the Jacobi iterations did not converge in %d", iters);
  if (rc) return rc;  // a status of the scan
  grad[0] = g;
  for (int64_t d = 0; d < D; ++d) grad[1 + d] = NAN;  // no density-parameter gradient
  return PMCMC_OK;
}

}  // namespace

extern "C" {

int pmcmc_deer_adjoint(pmcmc_handle* h, const pmcmc_target* tg, const pmcmc_deer_params* p,
                       const void* x0, uint64_t seed, uint64_t block, const void* S, int32_t mem,
                       int32_t objective, double* grad) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  int rc = validate(h, tg, p);
  if (rc) return rc;
  if (!x0 || !S || !grad) return fail(h, PMCMC_ERR_ARGUMENT, "x0, S and grad must not be NULL");
  if (mem != PMCMC_MEM_HOST && mem != PMCMC_MEM_DEVICE)
    return fail(h, PMCMC_ERR_ARGUMENT, "mem must be PMCMC_MEM_HOST or PMCMC_MEM_DEVICE");
  if (objective != PMCMC_OBJ_ESJD && objective != PMCMC_OBJ_MEAN_SQ)
    return fail(h, PMCMC_ERR_ARGUMENT, "objective must be PMCMC_OBJ_ESJD or PMCMC_OBJ_MEAN_SQ");
  if (tg->mass_Ld) return fail(h, PMCMC_ERR_UNSUPPORTED, "the adjoint takes no mass matrix");
  if (tg->kind == kLogistic)
    return adjoint_logistic(h, tg, p, x0, seed, block, S, mem, objective, grad);
  if (p->dtype != PMCMC_F32) return fail(h, PMCMC_ERR_UNSUPPORTED, "the adjoint is built for FP32");
  const int64_t D = tg->D, Dp = tg->Dp, T = p->T;
  if (Dp > 128) return fail(h, PMCMC_ERR_UNSUPPORTED, "the adjoint is built for D <= 128");
  rc = ensure_eigen(h, const_cast<pmcmc_target*>(tg));
  if (rc) return rc;
  DeviceGuard guard(h->device);
  const bool dense = tg->kind == kDenseGauss;
  const SolveLayout L = layout(D, Dp, T, 1, 4, false, 0, 0, 0, nullptr, true);
  rc = ensure_ws(h, L.total);
  if (rc) return rc;
  unsigned char* ws = h->ws;
  const cudaMemcpyKind kin =
      mem == PMCMC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CK(cudaMemsetAsync(ws + L.x0a, 0, 4 * Dp, h->stream));
  CK(cudaMemcpyAsync(ws + L.x0a, x0, 4 * D, kin, h->stream));
  CK(cudaMemsetAsync(ws + L.S0, 0, 4 * T * Dp, h->stream));
  CK(cudaMemcpy2DAsync(ws + L.S0, 4 * Dp, S, 4 * D, 4 * D, T, kin, h->stream));
  DevParams P{};
  P.D = D;
  P.Dp = Dp;
  P.T = T;
  P.W = T;
  P.eps = p->epsilon;
  P.sqrt2eps = std::sqrt(2 * p->epsilon);
  P.inv4eps = 1.0 / (4 * p->epsilon);
  P.inv2eps = 1.0 / (2 * p->epsilon);
  P.damping = p->damping;
  P.tol_abs = p->tol_abs;
  P.tol_rel = p->tol_rel;
  P.seed = seed;
  P.block = block;
  P.jac = p->jacobian;
  P.probes = p->probes;
  P.maxiter = p->maxiter;
  P.tkind = tg->kind;
  P.mean_d = tg->mean_d;
  P.prec_d = tg->prec_d;
  P.mean_f = tg->mean_f;
  P.prec_f = tg->prec_f;
  P.S[0] = ws + L.S0;
  P.S[1] = ws + L.S1;
  P.x0 = ws + L.x0a;
  P.xi = reinterpret_cast<float*>(ws + L.xi);
  P.logu = reinterpret_cast<double*>(ws + L.logu);
  FullArgs F{};
  F.lam = tg->lam_f;
  F.Qrm = tg->qrm_f;
  F.Qcm = tg->qcm_f;
  F.acc = ws + L.facc;
  F.rot = dense ? 1 : 0;
  F.lam_adj = reinterpret_cast<float*>(ws + L.alam);
  F.cterm = reinterpret_cast<float*>(ws + L.acterm);
  F.arev = reinterpret_cast<float*>(ws + L.aarev);
  F.direct = reinterpret_cast<double*>(ws + L.adirect);
  CK(cudaMemcpyAsync(h->d_params, &P, sizeof(DevParams), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_full, &F, sizeof(FullArgs), cudaMemcpyHostToDevice, h->stream));
  const SweepKernels k = gauss_sweep_kernels(false, tg->kind, PMCMC_JAC_DIAG, D);
  const int init_grid = static_cast<int>(
      std::min<int64_t>((T * (Dp / 4) + 255) / 256, int64_t(h->num_sms) * 8));
  void* init_args[] = {&h->d_params, &h->d_state};
  CK(cudaLaunchKernel(k.init, dim3(init_grid), dim3(256), init_args, 0, h->stream));
  h->scan_epoch = (h->scan_epoch + 1) & 0x3fffffffu;
  if (h->scan_epoch == 0) h->scan_epoch = 1;
  double* out = reinterpret_cast<double*>(ws + L.aout);
  CK(full_adjoint(h->stream, h->d_params, h->d_full, F, D, Dp, T, tg->kind, h->num_sms,
                  objective, reinterpret_cast<const float*>(ws + L.S0), out, ws + L.ascr,
                  h->scan_epoch));
  uint32_t flags[2] = {0, 0};
  CK(cudaMemcpyAsync(grad, out, sizeof(double) * (1 + D), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(flags, ws + L.ascr, sizeof flags, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flags[1])
    return fail(h, PMCMC_ERR_TIMEOUT, "adjoint scan look-back wait exceeded its bound");
  return PMCMC_OK;
}

// ---- T-split slices ---------------------------------------------------------
// A long chain split across ranks: each rank owns columns [t0, t0 + W) of the
// block and per Newton sweep (1) evaluates A, B from its iterate and its left
// boundary, (2) scans them locally into the slice's affine map (prod A, b),
// (3) after the ranks have exchanged maps, rescans from the carried state and
// damps (DEER.jl:398-475 applied to a slice; the composition of slice maps is
// the associativity the scan relies on, DEERScan.jl:102-173).
namespace {

int slice_copy_in(pmcmc_handle* h, void* dst, const void* src, size_t bytes, int32_t mem) {
  CK(cudaMemcpyAsync(dst, src, bytes,
                     mem == PMCMC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     h->stream));
  return PMCMC_OK;
}
int slice_copy_out(pmcmc_handle* h, void* dst, const void* src, size_t bytes, int32_t mem) {
  CK(cudaMemcpyAsync(dst, src, bytes,
                     mem == PMCMC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     h->stream));
  return PMCMC_OK;
}

ScanScratch slice_scratch(pmcmc_handle* h) {
  SliceState& sl = h->slice;
  unsigned char* w = h->ws + sl.scr;
  const int64_t Dp = sl.P.Dp, W = sl.P.T;
  const int TT = scan_tile_cols(Dp, W);
  const int64_t nt = (W + TT - 1) / TT;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  ScanScratch scr;
  scr.counter = reinterpret_cast<uint32_t*>(w);
  size_t off = 256;
  scr.flags = reinterpret_cast<uint32_t*>(w + off);
  off += al(4 * static_cast<size_t>(nt));
  scr.agg_a = w + off;
  off += al(sl.es * nt * Dp);
  scr.agg_b = w + off;
  off += al(sl.es * nt * Dp);
  scr.incl = w + off;
  return scr;
}

int slice_scan(pmcmc_handle* h, const void* B, const void* s0, void* out) {
  SliceState& sl = h->slice;
  ScanScratch scr = slice_scratch(h);
  h->scan_epoch = (h->scan_epoch + 1) & 0x3fffffffu;
  if (h->scan_epoch == 0) h->scan_epoch = 1;
  CK(launch_affine_scan(h->stream, sl.es == 8, sl.P.Dp, sl.P.T, h->ws + sl.A, B, s0, out, scr,
                        h->scan_epoch));
  return PMCMC_OK;
}

}  // namespace

int pmcmc_slice_begin(pmcmc_handle* h, const pmcmc_target* tg, const pmcmc_deer_params* p,
                      const void* x0, uint64_t seed, uint64_t block, int64_t t0, int64_t W,
                      int32_t mem) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  int rc = validate(h, tg, p);
  if (rc) return rc;
  if (!x0) return fail(h, PMCMC_ERR_ARGUMENT, "x0 must not be NULL");
  if (tg->kind == kLogistic)
    return fail(h, PMCMC_ERR_UNSUPPORTED, "slices are built for the Gaussian targets");
  if (tg->mass_Ld) return fail(h, PMCMC_ERR_UNSUPPORTED, "slices take no mass matrix");
  if (p->jacobian == PMCMC_JAC_FULL)
    return fail(h, PMCMC_ERR_UNSUPPORTED, "slices take the diagonal Jacobians");
  if (t0 < 0 || W < 1 || t0 + W > p->T)
    return fail(h, PMCMC_ERR_DIMENSION, "slice [t0, t0 + W) must lie inside [0, T)");
  DeviceGuard guard(h->device);
  SliceState& sl = h->slice;
  sl = SliceState{};
  sl.tg = tg;
  sl.p = *p;
  sl.es = p->dtype == PMCMC_F64 ? 8 : 4;
  const int64_t D = tg->D, Dp = tg->Dp;
  const size_t es = sl.es;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = (off + bytes + 255) & ~size_t(255);
    return o;
  };
  sl.S[0] = take(es * W * Dp);
  sl.S[1] = take(es * W * Dp);
  sl.x0 = take(es * Dp);
  sl.xbar = take(es * Dp);
  sl.carry = take(es * Dp);
  sl.ones = take(es * Dp);
  sl.A = take(es * W * Dp);
  sl.B = take(es * W * Dp);
  sl.Sloc = take(es * W * Dp);
  sl.Zb = take(es * W * Dp);
  sl.xi = take(4 * W * Dp);
  sl.logu = take(8 * static_cast<size_t>(W));
  sl.red = take(4 * sizeof(unsigned long long));
  sl.scr = take(scan_scratch_bytes(es == 8, Dp, W) + 1024);
  sl.out_S = take(es * W * D);
  sl.out_lp = take(es * W);
  sl.out_acc = take(static_cast<size_t>(W));
  sl.x_next = take(es * Dp);
  sl.total = off;
  rc = ensure_ws(h, sl.total);
  if (rc) return rc;
  unsigned char* ws = h->ws;
  CK(cudaMemsetAsync(ws, 0, sl.total, h->stream));
  rc = slice_copy_in(h, ws + sl.x0, x0, es * D, mem);
  if (rc) return rc;
  std::vector<double> one64(static_cast<size_t>(Dp), 1.0);
  std::vector<float> one32(static_cast<size_t>(Dp), 1.f);
  CK(cudaMemcpyAsync(ws + sl.ones, es == 8 ? static_cast<const void*>(one64.data()) : one32.data(),
                     es * Dp, cudaMemcpyHostToDevice, h->stream));
  DevParams& P = sl.P;
  P.D = D;
  P.Dp = Dp;
  P.T = W;
  P.W = W;
  P.eps = p->epsilon;
  P.sqrt2eps = std::sqrt(2 * p->epsilon);
  P.inv4eps = 1.0 / (4 * p->epsilon);
  P.inv2eps = 1.0 / (2 * p->epsilon);
  P.damping = p->damping;
  P.tol_abs = p->tol_abs;
  P.tol_rel = p->tol_rel;
  P.seed = seed;
  P.block = block;
  P.jac = p->jacobian;
  P.probes = p->probes;
  P.maxiter = p->maxiter;
  P.tkind = tg->kind;
  P.t_off = static_cast<int32_t>(t0);
  P.mean_d = tg->mean_d;
  P.prec_d = tg->prec_d;
  P.mean_f = tg->mean_f;
  P.prec_f = tg->prec_f;
  P.S[0] = ws + sl.S[0];
  P.S[1] = ws + sl.S[1];
  P.x0 = ws + sl.xbar;
  P.xi = reinterpret_cast<float*>(ws + sl.xi);
  P.logu = reinterpret_cast<double*>(ws + sl.logu);
  P.ncols_out = W;
  P.S_out = ws + sl.out_S;
  P.logp_out = ws + sl.out_lp;
  P.accept_out = ws + sl.out_acc;
  P.x_next = ws + sl.x_next;
  CK(cudaMemcpyAsync(h->d_params, &P, sizeof(DevParams), cudaMemcpyHostToDevice, h->stream));
  const SweepKernels k = gauss_sweep_kernels(es == 8, tg->kind, p->jacobian, D);
  const int init_grid = static_cast<int>(
      std::min<int64_t>((W * (Dp / 4) + 255) / 256, int64_t(h->num_sms) * 8));
  void* init_args[] = {&h->d_params, &h->d_state};
  CK(cudaLaunchKernel(k.init, dim3(init_grid), dim3(256), init_args, 0, h->stream));
  // the iterate starts as x0 broadcast over the slice (DEER.jl:538-542)
  CK(launch_broadcast(h->stream, es == 8, Dp, W, ws + sl.x0, ws + sl.S[0]));
  CK(cudaStreamSynchronize(h->stream));
  sl.active = true;
  return PMCMC_OK;
}

int pmcmc_slice_local(pmcmc_handle* h, const void* xbar0, void* agg, int32_t mem) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  SliceState& sl = h->slice;
  if (!sl.active) return fail(h, PMCMC_ERR_ARGUMENT, "no slice: call pmcmc_slice_begin first");
  if (!xbar0 || !agg) return fail(h, PMCMC_ERR_ARGUMENT, "null buffer");
  DeviceGuard guard(h->device);
  unsigned char* ws = h->ws;
  const int64_t D = sl.P.D, Dp = sl.P.Dp, W = sl.P.T;
  const size_t es = sl.es;
  int rc = slice_copy_in(h, ws + sl.xbar, xbar0, es * D, mem);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h->d_params, &sl.P, sizeof(DevParams), cudaMemcpyHostToDevice, h->stream));
  const SweepKernels k = gauss_sweep_kernels(es == 8, sl.tg->kind, sl.p.jacobian, D);
  const size_t smem = gauss_sweep_smem(es == 8, Dp, 1, sl.tg->kind == kDenseGauss).total;
  if (smem > 0)
    CK(raise_smem_limit(reinterpret_cast<const void*>(k.eval), smem));
  const int grid = static_cast<int>(std::min<int64_t>((W + kWarps - 1) / kWarps,
                                                      int64_t(h->num_sms) * 8));
  const void* Sold = ws + sl.S[sl.cur];
  int it = sl.iter, from_x0 = 0;
  void* A = ws + sl.A;
  void* B = ws + sl.B;
  void* eval_args[] = {&h->d_params, const_cast<void**>(&Sold), &it, &from_x0, &A, &B};
  CK(cudaLaunchKernel(k.eval, dim3(grid), dim3(kThreads), eval_args, smem, h->stream));
  // slice map: b = scan(A, B) from 0, prod A = scan(A, 0) from 1 (last columns)
  rc = slice_scan(h, ws + sl.B, ws + sl.Zb, ws + sl.Sloc);
  if (rc) return rc;
  unsigned char* out = static_cast<unsigned char*>(agg);
  rc = slice_copy_out(h, out + es * D, ws + sl.Sloc + es * (W - 1) * Dp, es * D, mem);
  if (rc) return rc;
  rc = slice_scan(h, ws + sl.Zb, ws + sl.ones, ws + sl.Sloc);
  if (rc) return rc;
  rc = slice_copy_out(h, out, ws + sl.Sloc + es * (W - 1) * Dp, es * D, mem);
  if (rc) return rc;
  uint32_t flags[2] = {0, 0};
  CK(cudaMemcpyAsync(flags, ws + sl.scr, sizeof flags, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flags[1]) return fail(h, PMCMC_ERR_TIMEOUT, "slice scan look-back wait exceeded its bound");
  return PMCMC_OK;
}

int pmcmc_slice_finish(pmcmc_handle* h, const void* carry_in, void* last_out, double* red,
                       int32_t mem) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  SliceState& sl = h->slice;
  if (!sl.active) return fail(h, PMCMC_ERR_ARGUMENT, "no slice: call pmcmc_slice_begin first");
  if (!carry_in || !red) return fail(h, PMCMC_ERR_ARGUMENT, "null buffer");
  DeviceGuard guard(h->device);
  unsigned char* ws = h->ws;
  const int64_t D = sl.P.D, Dp = sl.P.Dp, W = sl.P.T;
  const size_t es = sl.es;
  int rc = slice_copy_in(h, ws + sl.carry, carry_in, es * D, mem);
  if (rc) return rc;
  void* Snew = ws + sl.S[sl.cur ^ 1];
  rc = slice_scan(h, ws + sl.B, ws + sl.carry, Snew);
  if (rc) return rc;
  auto* r = reinterpret_cast<unsigned long long*>(ws + sl.red);
  CK(launch_damp_metric(h->stream, es == 8, D, Dp, W, ws + sl.S[sl.cur], Snew, sl.P.damping, r));
  if (last_out) {
    rc = slice_copy_out(h, last_out, static_cast<unsigned char*>(Snew) + es * (W - 1) * Dp,
                        es * D, mem);
    if (rc) return rc;
  }
  unsigned long long hr[3] = {0, 0, 0};
  uint32_t flags[2] = {0, 0};
  CK(cudaMemcpyAsync(hr, r, sizeof hr, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(flags, ws + sl.scr, sizeof flags, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flags[1]) return fail(h, PMCMC_ERR_TIMEOUT, "slice scan look-back wait exceeded its bound");
  std::memcpy(&red[0], &hr[0], 8);
  std::memcpy(&red[1], &hr[1], 8);
  sl.cur ^= 1;
  sl.iter += 1;
  if (hr[2]) return fail(h, PMCMC_ERR_NONFINITE, "non-finite value in the slice iterate");
  return PMCMC_OK;
}

int pmcmc_slice_result(pmcmc_handle* h, const void* xbar0, void* S_out, void* logp_out,
                       uint8_t* accept_out, pmcmc_info* info, int32_t mem) {
  if (!h) return PMCMC_ERR_ARGUMENT;
  SliceState& sl = h->slice;
  if (!sl.active) return fail(h, PMCMC_ERR_ARGUMENT, "no slice: call pmcmc_slice_begin first");
  if (!xbar0 || !S_out) return fail(h, PMCMC_ERR_ARGUMENT, "null buffer");
  DeviceGuard guard(h->device);
  unsigned char* ws = h->ws;
  const int64_t D = sl.P.D, Dp = sl.P.Dp, W = sl.P.T;
  const size_t es = sl.es;
  int rc = slice_copy_in(h, ws + sl.xbar, xbar0, es * D, mem);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h->d_params, &sl.P, sizeof(DevParams), cudaMemcpyHostToDevice, h->stream));
  DevState st{};
  st.cur = sl.cur;
  st.iter = sl.iter;
  st.min_margin_bits = 0x7ff0000000000000ull;
  *h->h_state = st;
  CK(cudaMemcpyAsync(h->d_state, h->h_state, sizeof(DevState), cudaMemcpyHostToDevice,
                     h->stream));
  const SweepKernels k = gauss_sweep_kernels(es == 8, sl.tg->kind, sl.p.jacobian, D);
  const size_t smem = gauss_sweep_smem(es == 8, Dp, 1, sl.tg->kind == kDenseGauss).total;
  if (smem > 0)
    CK(raise_smem_limit(reinterpret_cast<const void*>(k.finalize), smem));
  const int grid = static_cast<int>(std::min<int64_t>((W + kWarps - 1) / kWarps,
                                                      int64_t(h->num_sms) * 8));
  void* fin_args[] = {&h->d_params, &h->d_state};
  CK(cudaLaunchKernel(k.finalize, dim3(grid), dim3(kThreads), fin_args, smem, h->stream));
  rc = slice_copy_out(h, S_out, ws + sl.out_S, es * W * D, mem);
  if (!rc && logp_out) rc = slice_copy_out(h, logp_out, ws + sl.out_lp, es * W, mem);
  if (!rc && accept_out) rc = slice_copy_out(h, accept_out, ws + sl.out_acc, W, mem);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h->h_state, h->d_state, sizeof(DevState), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (info) {
    fill_info(*h->h_state, info);
    info->path = 0;
  }
  return PMCMC_OK;
}

}  // extern "C"
