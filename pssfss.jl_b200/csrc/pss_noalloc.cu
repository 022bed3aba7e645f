// pss_lu_factor_noalloc: the FP64 blocked LU factorisation (pss_lu.cu) on caller-owned
// device memory, with no device allocation of any kind.
//
// Who needs it: a caller whose device memory is owned by its own allocator or pool (for
// example a Julia CUDA.jl or PyTorch caching pool that has reserved most of the device), or
// one that factors many matrices from a latency-sensitive loop, cannot have this library
// call cudaMalloc/cudaFree per call: cudaMalloc can fail against the pool's reservation,
// and cudaFree synchronises the whole device, stalling every other stream.  The regular
// entry points (pss_lu_solve and the context workers) own their workspaces; this one keeps
// its only scratch, the panels' interchange list, in a fixed file-scope device array.
//
// Limits and rules (also stated in include/pssfss_b200.h):
//   * order n <= kNoAllocMaxOrder (8192, the cluster panel's own limit of 16 CTAs x 512
//     rows); larger n is rejected with an error message before anything is launched;
//   * the scratch is kScratchBytes (1 KB): one panel's interchange list (count, 64
//     destination rows, 64 source rows), rewritten by every panel;
//   * the scratch array is one per device and is shared by every call on that device:
//     calls that overlap in time on one device (different streams or host threads) race
//     on it and produce wrong factors - serialise them (one stream, or synchronise);
//   * nothing in the scratch has to start at zero (each panel writes the list before the
//     interchange kernel reads it); *info must be zero when the factorisation starts,
//     and this function writes that zero itself, on the caller's stream, before the first
//     kernel;
//   * the first call on each device resolves the scratch array's address with
//     cudaGetSymbolAddress (a one-time set-up, done with that device current); make that
//     first call before any stream capture on the device.  The address belongs to the
//     device's current CUDA context: it is cached together with that context's handle and
//     resolved again when a call finds another context current (after cudaDeviceReset, or
//     a context the caller created itself), so a stale address is never used.
#include <cuda.h>

#include <mutex>

#include "pss_internal.cuh"
#include "pssfss_b200.h"

namespace {

constexpr int kNoAllocMaxOrder = 8192;
// One panel's interchange list (129 ints) rounded up: pss_lu_ws_bytes(n, PSS_FP64) for every n.
constexpr size_t kScratchBytes = 1024;

static __device__ __align__(256) unsigned char g_lu_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
void *g_scratch_ptr[kMaxDevices] = {};
CUcontext g_scratch_ctx[kMaxDevices] = {};  // the context each cached address belongs to
std::mutex g_setup_mu;

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
CtxGetCurrentFn g_ctx_get_current = nullptr;  // cuCtxGetCurrent, resolved once under g_setup_mu

// Set-up per device (the caller's current device) and context: the array's device address.
int scratch_for_current_device(void **out) {
  int dev = -1;
  PSS_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    pss_set_error("device %d out of range for the no-allocation scratch table", dev);
    return -3;
  }
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_ctx_get_current) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      pss_set_error("cuCtxGetCurrent unavailable");
      return -3;
    }
    g_ctx_get_current = (CtxGetCurrentFn)fn;
  }
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) {
    pss_set_error("no current CUDA context on device %d", dev);
    return -3;
  }
  if (!g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_lu_scratch);
    if (e != cudaSuccess || !p) {
      pss_set_error("cudaGetSymbolAddress(no-allocation LU scratch) failed on device %d: %s", dev,
                    cudaGetErrorString(e));
      return -3;
    }
    g_scratch_ptr[dev] = p;
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_ptr[dev];
  return 0;
}

}  // namespace

extern "C" int pss_lu_factor_noalloc(int n, double *A, int64_t ld, int *ipiv, int *info, void *stream) {
  if (n <= 0 || !A || !ipiv || !info || ld < n) {
    pss_set_error("invalid argument");
    return -1;
  }
  if (n > kNoAllocMaxOrder) {
    pss_set_error("order %d exceeds the no-allocation LU limit of %d (scratch is a fixed %zu-byte device array)",
                  n, kNoAllocMaxOrder, kScratchBytes);
    return -1;
  }
  if (pss_lu_ws_bytes(n, PSS_FP64) > kScratchBytes) {
    pss_set_error("no-allocation LU scratch (%zu bytes) smaller than the %zu bytes order %d needs", kScratchBytes,
                  pss_lu_ws_bytes(n, PSS_FP64), n);
    return -1;
  }
  cudaStream_t st = (cudaStream_t)stream;
  // first runtime call on the caller's memory: it also makes the device's context current on
  // this host thread, which the scratch look-up below reads
  PSS_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int), st));
  void *scratch = nullptr;
  if (int rc = scratch_for_current_device(&scratch)) return rc;
  return pss_lu64(n, (cd *)A, (long long)ld, ipiv, info, scratch, kScratchBytes, st);
}
