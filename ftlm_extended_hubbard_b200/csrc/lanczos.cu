// Lanczos BLAS-1 kernels (reference src/lanczos.cpp:125-208) with deterministic FP64 reductions:
// a fixed grid of kRedBlocks blocks, a fixed in-block tree, and a single-block final pass, so
// repeated runs give bitwise identical alpha/beta.
#include "hv.cuh"

namespace ftlm_b200 {

namespace {

template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double* sh /* N*kRedThreads */) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < N; ++i) sh[i * kRedThreads + t] = v[i];
  __syncthreads();
  for (int s = kRedThreads / 2; s > 0; s >>= 1) {
    if (t < s) {
#pragma unroll
      for (int i = 0; i < N; ++i) sh[i * kRedThreads + t] += sh[i * kRedThreads + t + s];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = sh[i * kRedThreads];
}

__global__ void __launch_bounds__(kRedThreads) dotc_kernel(const double2* __restrict__ q,
                                                           const double2* __restrict__ w, int64_t n,
                                                           double* __restrict__ partial) {
  __shared__ double sh[2 * kRedThreads];
  double v[2] = {0.0, 0.0};
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kRedThreads;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * kRedThreads + threadIdx.x; i < n; i += stride) {
    const double2 a = q[i], b = w[i];
    v[0] += a.x * b.x + a.y * b.y;  // conj(a) * b
    v[1] += a.x * b.y - a.y * b.x;
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = v[0];
    partial[2 * blockIdx.x + 1] = v[1];
  }
}

// Sums `nb` partial vectors of width W (stride W) into out[0..W).
template <int W>
__global__ void __launch_bounds__(kRedThreads) final_kernel(const double* __restrict__ partial, int nb,
                                                            double* __restrict__ out) {
  __shared__ double sh[W * kRedThreads];
  double v[W];
#pragma unroll
  for (int i = 0; i < W; ++i) v[i] = 0.0;
  for (int b = threadIdx.x; b < nb; b += kRedThreads) {
#pragma unroll
    for (int i = 0; i < W; ++i) v[i] += partial[W * b + i];
  }
  block_sum<W>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < W; ++i) out[i] = v[i];
  }
}

__global__ void __launch_bounds__(kRedThreads) update_kernel(double2* __restrict__ w, const double2* __restrict__ q,
                                                             const double2* __restrict__ qp,
                                                             const double* __restrict__ zp, double bprev,
                                                             int use_prev, int64_t n, double* __restrict__ partial) {
  __shared__ double sh[kRedThreads];
  const double zr = zp[0], zi = zp[1];
  double v[1] = {0.0};
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kRedThreads;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * kRedThreads + threadIdx.x; i < n; i += stride) {
    double2 a = w[i];
    const double2 b = q[i];
    a.x -= zr * b.x - zi * b.y;
    a.y -= zr * b.y + zi * b.x;
    if (use_prev) {
      const double2 c = qp[i];
      a.x -= bprev * c.x;
      a.y -= bprev * c.y;
    }
    w[i] = a;
    v[0] += a.x * a.x + a.y * a.y;
  }
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

// Lanczos update with the scales of the unnormalised vectors applied on the fly.
__global__ void __launch_bounds__(kRedThreads) update_scaled_kernel(double2* __restrict__ w,
                                                                    const double2* __restrict__ Wk, double sk,
                                                                    const double2* __restrict__ Wkm1, double skm1,
                                                                    const double* __restrict__ zp, double bprev,
                                                                    int use_prev, int64_t n,
                                                                    double* __restrict__ partial) {
  __shared__ double sh[kRedThreads];
  const double zr = zp[0], zi = zp[1];
  double v[1] = {0.0};
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kRedThreads;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * kRedThreads + threadIdx.x; i < n; i += stride) {
    double2 a = w[i];
    const double2 b0 = Wk[i];
    const double bx = sk * b0.x, by = sk * b0.y;
    a.x -= zr * bx - zi * by;
    a.y -= zr * by + zi * bx;
    if (use_prev) {
      const double2 c = Wkm1[i];
      a.x -= bprev * (skm1 * c.x);
      a.y -= bprev * (skm1 * c.y);
    }
    w[i] = a;
    v[0] += a.x * a.x + a.y * a.y;
  }
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

// First level of a pair reduction: block b sums pairs [b*per, (b+1)*per) in order.
__global__ void __launch_bounds__(kRedThreads) pairs_kernel(const double* __restrict__ in, int64_t nb, int64_t per,
                                                            double* __restrict__ out) {
  __shared__ double sh[2 * kRedThreads];
  double v[2] = {0.0, 0.0};
  const int64_t b0 = static_cast<int64_t>(blockIdx.x) * per;
  const int64_t b1 = min(nb, b0 + per);
  for (int64_t i = b0 + threadIdx.x; i < b1; i += kRedThreads) {
    v[0] += in[2 * i];
    v[1] += in[2 * i + 1];
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = v[0];
    out[2 * blockIdx.x + 1] = v[1];
  }
}

__global__ void scale_kernel(double2* __restrict__ dst, const double2* __restrict__ src, int64_t n,
                             const double* __restrict__ nw2) {
  const double b = sqrt(*nw2);
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double2 a = src[i];
    dst[i] = make_double2(a.x / b, a.y / b);
  }
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): 10 rounds of the 4x32 S-box with the
// published multipliers and Weyl key increments.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
  constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += W0;
    k.y += W1;
  }
  return c;
}

__global__ void __launch_bounds__(kRedThreads) philox_start_kernel(double2* __restrict__ q, int64_t n, unsigned seed,
                                                                   double* __restrict__ partial) {
  __shared__ double sh[kRedThreads];
  double v[1] = {0.0};
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kRedThreads;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * kRedThreads + threadIdx.x; i < n; i += stride) {
    const uint4 r = philox4x32_10(make_uint4(static_cast<uint32_t>(i), static_cast<uint32_t>(i >> 32), 0u, 0u),
                                  make_uint2(seed, 0x7F4A7C15u));
    const uint64_t a = (static_cast<uint64_t>(r.x) << 21) ^ (r.y >> 11);
    const uint64_t b = (static_cast<uint64_t>(r.z) << 21) ^ (r.w >> 11);
    const double u1 = (static_cast<double>(a & ((1ull << 53) - 1)) + 0.5) * 0x1.0p-53;  // (0,1)
    const double u2 = (static_cast<double>(b & ((1ull << 53) - 1)) + 0.5) * 0x1.0p-53;
    const double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    const double2 z = make_double2(rad * c, rad * s);
    q[i] = z;
    v[0] += z.x * z.x + z.y * z.y;
  }
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

__global__ void normalise_kernel(double2* __restrict__ q, int64_t n, const double* __restrict__ n2) {
  const double n0 = sqrt(*n2);
  const bool degenerate = n0 < 1e-18;
  const double s = 1.0 / n0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (degenerate) {
      q[i] = make_double2(i == 0 ? 1.0 : 0.0, 0.0);
    } else {
      const double2 a = q[i];
      q[i] = make_double2(a.x * s, a.y * s);
    }
  }
}

}  // namespace

cudaError_t lz_dotc(const double2* q, const double2* w, int64_t n, double* scratch, cudaStream_t st) {
  dotc_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(q, w, n, scratch);
  final_kernel<2><<<1, kRedThreads, 0, st>>>(scratch, kRedBlocks, scratch + kResZ);
  return cudaGetLastError();
}

cudaError_t lz_update(double2* w, const double2* q, const double2* qp, double bprev, int use_prev, int64_t n,
                      double* scratch, cudaStream_t st) {
  update_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(w, q, qp, scratch + kResZ, bprev, use_prev, n, scratch);
  final_kernel<1><<<1, kRedThreads, 0, st>>>(scratch, kRedBlocks, scratch + kResNw2);
  return cudaGetLastError();
}

cudaError_t lz_reduce_pairs(const double* partial, int64_t nb, double* scratch, cudaStream_t st) {
  const int64_t per = (nb + kRedBlocks - 1) / kRedBlocks;
  pairs_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(partial, nb, per, scratch);
  final_kernel<2><<<1, kRedThreads, 0, st>>>(scratch, kRedBlocks, scratch + kResZ);
  return cudaGetLastError();
}

cudaError_t lz_update_scaled(double2* w, const double2* Wk, double sk, const double2* Wkm1, double skm1, double bprev,
                             int use_prev, int64_t n, double* scratch, cudaStream_t st) {
  update_scaled_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(w, Wk, sk, Wkm1, skm1, scratch + kResZ, bprev, use_prev, n,
                                                          scratch);
  final_kernel<1><<<1, kRedThreads, 0, st>>>(scratch, kRedBlocks, scratch + kResNw2);
  return cudaGetLastError();
}

cudaError_t lz_scale_by_norm(double2* dst, const double2* src, int64_t n, const double* scratch, cudaStream_t st) {
  scale_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(dst, src, n, scratch + kResNw2);
  return cudaGetLastError();
}

cudaError_t lz_philox_start(double2* q, int64_t n, unsigned seed, double* scratch, cudaStream_t st) {
  philox_start_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(q, n, seed, scratch);
  final_kernel<1><<<1, kRedThreads, 0, st>>>(scratch, kRedBlocks, scratch + kResN0);
  return cudaGetLastError();
}

cudaError_t lz_normalise_start(double2* q, int64_t n, const double* scratch, cudaStream_t st) {
  normalise_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(q, n, scratch + kResN0);
  return cudaGetLastError();
}

}  // namespace ftlm_b200
