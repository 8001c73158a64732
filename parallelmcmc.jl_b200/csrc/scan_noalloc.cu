// scan_noalloc.cu -- the diagonal affine scan for callers that cannot allocate
// device memory.
//
// Some callers may not call cudaMalloc once they are running: a process that
// reserved its whole device memory budget up front in its own pool (a Julia
// session whose CUDA.jl pool owns the device, a serving process with a fixed
// memory budget), or a latency-critical loop that cannot afford the implicit
// device synchronisation of an allocation.  pmcmc_affine_scan_diag_noalloc
// serves them: the caller passes device inputs and outputs, and the scan's
// look-back scratch (tile flags and per-tile aggregates) lives in the
// file-scope array below instead of a handle's workspace.  No cudaMalloc,
// cudaFree or allocating library routine is called.
//
// The array is kPmcmcNoallocScratchBytes (4 MiB) on every GPU that loads the
// library, held until the process exits.  It is shared by all calls on a
// device and keeps the last call's contents, so each call clears its tile
// counter and advances a per-device epoch that invalidates stale tile flags;
// calls that overlap on the GPU (different streams, or several host threads)
// race on the array and must be serialised by the caller.  The array's memory
// is taken when the module is loaded on a device, which under lazy loading is
// the first call there: callers that give every free byte to their own pool
// make one small call first.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>

#include "../../include/pmcmc_deer.h"
#include "deer_launch.h"

namespace {

constexpr size_t kPmcmcNoallocScratchBytes = size_t(4) << 20;
static_assert(kPmcmcNoallocScratchBytes == PMCMC_NOALLOC_SCRATCH_BYTES, "keep in step");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kPmcmcNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};
std::atomic<uint32_t> g_epoch[kMaxDevices];

// Device address of the scratch array for the current device, looked up once
// per device (the host-side symbol is not a device address).
int scratch_for_current_device(void** out, int* dev_out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return PMCMC_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return PMCMC_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  *dev_out = dev;
  return PMCMC_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" int pmcmc_affine_scan_diag_noalloc(int32_t dtype, int64_t D, int64_t T, const void* A,
                                              const void* B, const void* s0, void* S,
                                              void* stream) {
  if (dtype != PMCMC_F32 && dtype != PMCMC_F64) return PMCMC_ERR_ARGUMENT;
  if (D < 0 || T < 0) return PMCMC_ERR_DIMENSION;
  if (T == 0 || D == 0) return PMCMC_OK;
  if (!A || !B || !s0 || !S || S == A || S == B) return PMCMC_ERR_ARGUMENT;
  const bool f64 = dtype == PMCMC_F64;
  const size_t es = f64 ? 8 : 4;
  if (3 * es * static_cast<size_t>(D) > 200 * 1024) return PMCMC_ERR_UNSUPPORTED;
  const int TT = pmcmc::scan_tile_cols(D, T);
  const int64_t nt = (T + TT - 1) / TT;
  // layout inside the array: counter[2] | flags[nt] | agg_a | agg_b | incl
  const size_t o_flags = 64;
  const size_t o_agg_a = align256(o_flags + 4 * static_cast<size_t>(nt));
  const size_t o_agg_b = o_agg_a + align256(es * nt * D);
  const size_t o_incl = o_agg_b + align256(es * nt * D);
  const size_t need = o_incl + align256(es * nt * D);
  if (need > kPmcmcNoallocScratchBytes) return PMCMC_ERR_NOMEM;  // beyond the fixed maximum

  void* base = nullptr;
  int dev = 0;
  const int rc = scratch_for_current_device(&base, &dev);
  if (rc) return rc;
  unsigned char* b = static_cast<unsigned char*>(base);
  pmcmc::ScanScratch scr;
  scr.counter = reinterpret_cast<uint32_t*>(b);
  scr.flags = reinterpret_cast<uint32_t*>(b + o_flags);
  scr.agg_a = b + o_agg_a;
  scr.agg_b = b + o_agg_b;
  scr.incl = b + o_incl;
  uint32_t epoch = (g_epoch[dev].fetch_add(1) + 1) & 0x3fffffffu;
  if (epoch == 0) epoch = (g_epoch[dev].fetch_add(1) + 1) & 0x3fffffffu;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // launch_affine_scan clears the tile counter and the timeout flag on `s`
  if (pmcmc::launch_affine_scan(s, f64, D, T, A, B, s0, S, scr, epoch) != cudaSuccess) {
    cudaGetLastError();
    return PMCMC_ERR_CUDA;
  }
  uint32_t flag = 0;
  if (cudaMemcpyAsync(&flag, scr.counter + 1, sizeof flag, cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return PMCMC_ERR_CUDA;
  }
  return flag ? PMCMC_ERR_TIMEOUT : PMCMC_OK;
}
