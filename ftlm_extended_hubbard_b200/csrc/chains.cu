// Fused small-sector Lanczos; contract in chains.cuh.  Per step: w = H q (hv_element over the
// CTA's rows), z = <q, w>, w -= z q + beta_{k-1} q_prev, ||w||^2, breakdown test (||w||^2 < 1e-24),
// q_prev <- q, q <- w / beta_k.  Reductions: per-thread partial sums in a fixed order, then a
// fixed shared-memory tree.
#include "chains.cuh"

namespace ftlm_b200 {

namespace {

// Deterministic block sum of NV doubles; every thread receives the totals.
template <int kChainThreads, int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < NV; ++i) sh[i * kChainThreads + t] = v[i];
  __syncthreads();
  for (int s = kChainThreads / 2; s > 0; s >>= 1) {
    if (t < s)
#pragma unroll
      for (int i = 0; i < NV; ++i) sh[i * kChainThreads + t] += sh[i * kChainThreads + t + s];
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = sh[i * kChainThreads];
  __syncthreads();
}

template <int kChainThreads>
__global__ void __launch_bounds__(kChainThreads) chains_kernel(const DevSector* __restrict__ sectors,
                                                               const ChainDesc* __restrict__ chains, int M,
                                                               double2* __restrict__ scratch, double* __restrict__ alpha,
                                                               double* __restrict__ beta, int* __restrict__ used) {
  __shared__ double sh[2 * kChainThreads];
  const ChainDesc cd = chains[blockIdx.x];
  const DevSector S = sectors[cd.sector];
  const int64_t dim = S.dim;
  const int t = threadIdx.x;
  double2* q = scratch + cd.off;
  double2* qp = q + dim;
  double2* w = qp + dim;
  double* al = alpha + static_cast<int64_t>(cd.out) * M;
  double* be = beta + static_cast<int64_t>(cd.out) * M;
  double bprev = 0.0;
  int nused = 0;
  for (int k = 0; k < M; ++k) {
    double zz[2] = {0.0, 0.0};
    for (int64_t i = t; i < dim; i += kChainThreads) {
      const double2 y = hv_element(S, q, i);
      w[i] = y;
      const double2 a = q[i];
      zz[0] += a.x * y.x + a.y * y.y;  // conj(q) w
      zz[1] += a.x * y.y - a.y * y.x;
    }
    block_sum<kChainThreads, 2>(zz, sh);
    const double zr = zz[0], zi = zz[1];
    double n2[1] = {0.0};
    for (int64_t i = t; i < dim; i += kChainThreads) {
      const double2 a = q[i];
      double2 v = w[i];
      v.x -= zr * a.x - zi * a.y;
      v.y -= zr * a.y + zi * a.x;
      if (k > 0) {
        const double2 b = qp[i];
        v.x -= bprev * b.x;
        v.y -= bprev * b.y;
      }
      w[i] = v;
      n2[0] += v.x * v.x + v.y * v.y;
    }
    block_sum<kChainThreads, 1>(n2, sh);
    if (t == 0) al[k] = zr;
    nused = k + 1;
    if (n2[0] < 1e-24) break;  // src/lanczos.cpp:187: alpha_k kept, no beta_k
    const double b = sqrt(n2[0]);
    if (t == 0) be[k] = b;
    const double inv = 1.0 / b;
    for (int64_t i = t; i < dim; i += kChainThreads) {
      const double2 v = w[i];
      qp[i] = make_double2(v.x * inv, v.y * inv);  // becomes q_{k+1}
    }
    __syncthreads();
    double2* tmp = qp;
    qp = q;
    q = tmp;
    bprev = b;
  }
  if (t == 0) used[cd.out] = nused;
}

}  // namespace

cudaError_t chains_lanczos(const DevSector* sectors, const ChainDesc* chains, int nc, int M, double2* scratch,
                           double* alpha, double* beta, int* used, bool wide, cudaStream_t st) {
  if (nc <= 0) return cudaSuccess;
  if (wide)
    chains_kernel<1024><<<nc, 1024, 0, st>>>(sectors, chains, M, scratch, alpha, beta, used);
  else
    chains_kernel<256><<<nc, 256, 0, st>>>(sectors, chains, M, scratch, alpha, beta, used);
  return cudaGetLastError();
}

}  // namespace ftlm_b200
