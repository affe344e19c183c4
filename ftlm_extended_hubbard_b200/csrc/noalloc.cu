// Allocation-free variant of the tridiagonal quadrature (ftlm_gpu_tridiag_quadrature_noalloc).
//
// Who needs it: callers that must not call cudaMalloc/cudaFree on this path — code whose device
// memory is owned by another allocator (for example a framework's caching pool that has already
// reserved most of HBM, where a direct cudaMalloc can fail or fragment that pool), and
// latency-critical loops where cudaMalloc/cudaFree would implicitly synchronise the whole device.
// Such callers own the inputs and outputs; the only extra device memory this quadrature needs
// (the Ritz values and first-row weights passed from the Jacobi kernel to the evaluation kernel,
// and one status word) lives in the file-scope array below instead of a cudaMalloc'd buffer.
//
// Limits and sharing:
//   * n_chains * ld <= kNoAllocMaxEntries (65,536) — the array holds 2 x 65,536 doubles (1 MiB)
//     plus a status word, and every GPU that loads this library keeps it until the process exits.
//     Larger requests are rejected with FTLM_ERR_UNSUPPORTED before any GPU work.
//   * The chain lengths live in device memory, so the host cannot check them: the kernels skip a
//     chain whose length is outside [0, ld] (its outputs become NaN) and raise the status word,
//     which the call clears first and reads back at the end (a wait on the caller's stream only)
//     to return FTLM_ERR_INVALID.
//   * Every call on a device uses the same array and it keeps the last call's contents.  Only the
//     status word needs to start at zero (cleared by each call); every other entry a call reads was
//     written earlier in that call.  Calls whose kernels overlap on the GPU (different streams, or
//     different host threads on the same device) race on the array; serialise them on one stream.
//   * The first call on each device (and again after that device's context was destroyed and
//     recreated, e.g. by cudaDeviceReset) looks up the array's device address with
//     cudaGetSymbolAddress, with that device current, and caches it keyed by the context; make
//     that first call before any stream capture on that device.
#include <cuda.h>

#include <mutex>

#include "../../include/ftlm_gpu.h"
#include "hv.cuh"

namespace {

constexpr int kNoAllocMaxEntries = 65536;
constexpr int kNoAllocMaxDevices = 64;
constexpr int kStatusSlot = 2 * kNoAllocMaxEntries;  // one int in the first of 32 trailing doubles

// Ritz values [0, max) and first-row weights [max, 2*max), indexed chain * ld + k; then the status word.
static __device__ __align__(256) double g_quad_scratch[2 * kNoAllocMaxEntries + 32];

// Host-side cache of the array's device address per device, valid for the context it was looked
// up in.  In host code the symbol g_quad_scratch is only a stand-in, never a device address:
// kernels get the looked-up pointer.
struct ScratchEntry {
  CUcontext ctx = nullptr;
  double* ptr = nullptr;
};
ScratchEntry g_scratch[kNoAllocMaxDevices];
std::mutex g_scratch_mu;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);

CUcontext current_context() {
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  CUcontext c = nullptr;
  if (fn) fn(&c);
  return c;
}

int scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return ftlm_b200::set_error(FTLM_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return ftlm_b200::set_error(FTLM_ERR_UNSUPPORTED, "device index >= 64");
  // make sure the device's primary context exists before keying the cache on it
  e = cudaFree(nullptr);
  if (e != cudaSuccess) return ftlm_b200::set_error(FTLM_ERR_CUDA, cudaGetErrorString(e));
  const CUcontext ctx = current_context();
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  ScratchEntry& ent = g_scratch[dev];
  if (ent.ptr == nullptr || ent.ctx != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_quad_scratch);
    if (e != cudaSuccess || p == nullptr)
      return ftlm_b200::set_error(FTLM_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed");
    ent.ptr = static_cast<double*>(p);
    ent.ctx = ctx;
  }
  *out = ent.ptr;
  return FTLM_OK;
}

}  // namespace

extern "C" int ftlm_gpu_tridiag_quadrature_noalloc(const double* alpha_dev, const double* beta_dev, const int* n_dev,
                                                   int n_chains, int ld, const double* bts_dev, int n_bt,
                                                   double* logq_dev, double* energy_dev, void* stream) {
  if (n_chains < 0 || ld <= 0 || n_bt < 0)
    return ftlm_b200::set_error(FTLM_ERR_INVALID, "n_chains >= 0, ld > 0 and n_bt >= 0 required");
  if (n_chains == 0 || n_bt == 0) return FTLM_OK;
  if (!alpha_dev || !beta_dev || !n_dev || !bts_dev || !logq_dev || !energy_dev)
    return ftlm_b200::set_error(FTLM_ERR_INVALID, "null device buffer");
  if (ld > 160)
    return ftlm_b200::set_error(FTLM_ERR_UNSUPPORTED, "tridiagonal size > 160 is not supported by the on-chip Jacobi");
  if (static_cast<long long>(n_chains) * ld > kNoAllocMaxEntries)
    return ftlm_b200::set_error(FTLM_ERR_UNSUPPORTED,
                                "no-alloc quadrature: n_chains * ld exceeds its 65536-entry scratch; split the batch "
                                "or use ftlm_gpu_tridiag_quadrature");
  if (static_cast<long long>(n_chains) * n_bt > 0x7fffffffLL)
    return ftlm_b200::set_error(FTLM_ERR_INVALID, "n_chains * n_bt exceeds 2^31 - 1");
  double* scratch = nullptr;
  const int rc = scratch_for_current_device(&scratch);
  if (rc != FTLM_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* lam = scratch;
  double* w0 = scratch + kNoAllocMaxEntries;
  int* status = reinterpret_cast<int*>(scratch + kStatusSlot);
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), st);
  if (e == cudaSuccess) e = ftlm_b200::quad_jacobi(alpha_dev, beta_dev, n_dev, n_chains, ld, 0, 1e-14, lam, w0, st, status);
  if (e == cudaSuccess)
    e = ftlm_b200::quad_eval(lam, w0, n_dev, n_chains, ld, bts_dev, n_bt, logq_dev, energy_dev, st, status);
  int h_status = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return ftlm_b200::set_error(FTLM_ERR_CUDA, cudaGetErrorString(e));
  if (h_status != 0)
    return ftlm_b200::set_error(FTLM_ERR_INVALID,
                                "no-alloc quadrature: a chain length n_dev[c] lies outside [0, ld]; those chains were "
                                "skipped and their outputs set to NaN");
  return FTLM_OK;
}
