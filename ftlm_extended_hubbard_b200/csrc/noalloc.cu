// Allocation-free variant of the tridiagonal quadrature (ftlm_gpu_tridiag_quadrature_noalloc).
//
// Who needs it: callers that must not call cudaMalloc/cudaFree on this path — code whose device
// memory is owned by another allocator (for example a framework's caching pool that has already
// reserved most of HBM, where a direct cudaMalloc can fail or fragment that pool), and
// latency-critical loops where cudaMalloc/cudaFree would implicitly synchronise the device.
// Such callers own the inputs and outputs; the only extra device memory this quadrature needs
// (the Ritz values and first-row weights passed from the Jacobi kernel to the evaluation kernel)
// lives in the file-scope array below instead of a cudaMalloc'd buffer.
//
// Limits and sharing:
//   * n_chains * ld <= kNoAllocMaxEntries (65,536) — the array holds 2 x 65,536 doubles (1 MiB)
//     and every GPU that loads this library keeps it until the process exits.  Larger requests
//     are rejected with FTLM_ERR_UNSUPPORTED before any GPU work.
//   * Every call on a device uses the same array and it keeps the last call's contents.  Nothing
//     in it needs to start at zero: each entry a call reads was written earlier in that call.
//     Calls whose kernels overlap on the GPU (different streams, or different host threads on
//     the same device) race on the array; serialise them on one stream.
//   * The first call on each device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it; make that first call
//     before any stream capture on that device.
#include <mutex>

#include "../../include/ftlm_gpu.h"
#include "hv.cuh"

namespace {

constexpr int kNoAllocMaxEntries = 65536;
constexpr int kNoAllocMaxDevices = 64;

// Ritz values [0, max) and first-row weights [max, 2*max), indexed chain * ld + k.
static __device__ __align__(256) double g_quad_scratch[2 * kNoAllocMaxEntries];

// Host-side cache of the array's device address per device.  In host code the symbol
// g_quad_scratch is only a stand-in, never a device address: kernels get the looked-up pointer.
double* g_scratch_dev[kNoAllocMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

int scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return ftlm_b200::set_error(FTLM_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return ftlm_b200::set_error(FTLM_ERR_UNSUPPORTED, "device index >= 64");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_dev[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_quad_scratch);
    if (e != cudaSuccess || p == nullptr)
      return ftlm_b200::set_error(FTLM_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed");
    g_scratch_dev[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_dev[dev];
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
  double* scratch = nullptr;
  const int rc = scratch_for_current_device(&scratch);
  if (rc != FTLM_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* lam = scratch;
  double* w0 = scratch + kNoAllocMaxEntries;
  cudaError_t e = ftlm_b200::quad_jacobi(alpha_dev, beta_dev, n_dev, n_chains, ld, 0, 1e-14, lam, w0, st);
  if (e == cudaSuccess) e = ftlm_b200::quad_eval(lam, w0, n_dev, n_chains, ld, bts_dev, n_bt, logq_dev, energy_dev, st);
  if (e != cudaSuccess) return ftlm_b200::set_error(FTLM_ERR_CUDA, cudaGetErrorString(e));
  return FTLM_OK;
}
