// Krylov moments for the FTLM parameter gradient; contract in grad.cuh.
//
// Block = E consecutive elements (state, chain) of the flattened [state][NC] vectors.  The block
// stages its slice of every W_l in shared memory (each thread only reads its own element's
// column, conflict-free), then for rows i in pairs stages K'[i][*][*] and forms
//   X_i = sum_l K'_il W_l   (FP64),
// accumulating Re(conj W_i X_i) (times the diagonal operators) and Re(conj(A W_i) X_i).  Fixed
// grid and fixed per-block order: the sums are bitwise repeatable.
#include <algorithm>

#include "grad.cuh"

namespace ftlm_b200 {

namespace {

constexpr int kIB = 2;  // rows of K' staged per pass

__device__ __forceinline__ double2 ld_c(const float2* p, int64_t i) {
  const float2 v = p[i];
  return make_double2(v.x, v.y);
}
__device__ __forceinline__ double2 ld_c(const double2* p, int64_t i) { return p[i]; }

template <typename T, int NC>
__global__ void __launch_bounds__(256) moments_kernel(DevSector S, const T* __restrict__ W, const T* __restrict__ AW,
                                                      int64_t vstride, const double* __restrict__ Kp, int n, int ld,
                                                      double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int E = blockDim.x;
  T* Ws = reinterpret_cast<T*>(smraw);                                                    // [n][E]
  double* Ks = reinterpret_cast<double*>(smraw + static_cast<size_t>(n) * E * sizeof(T));  // [kIB][n][NC]
  const int t = threadIdx.x;
  const int c = t % NC;  // E and every block start are multiples of NC
  const int64_t nch = (vstride + E - 1) / E;
  double accD = 0.0, accP = 0.0, accA = 0.0;
  for (int64_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
    const int64_t e = ch * E + t;
    const bool valid = e < vstride;
    __syncthreads();
    for (int l = 0; l < n; ++l) {
      T v{};
      if (valid) v = W[static_cast<int64_t>(l) * vstride + e];
      Ws[l * E + t] = v;
    }
    double aD = 0.0, aP = 0.0;
    if (valid) {
      const int64_t s = e / NC;
      const int64_t ru = s / S.Dd, rd = s - ru * S.Dd;
      const uint32_t u = S.umask[ru], d = S.dmask[rd];
      const uint4 w = S.wpl[ru];
      aD = static_cast<double>(__popc(u & d));
      aP = static_cast<double>(S.cnt_uu[ru] + S.cnt_dd[rd] + __popc(d & w.x) + 2 * __popc(d & w.y) +
                               4 * __popc(d & w.z) + 8 * __popc(d & w.w));
    }
    double sW = 0.0, sA = 0.0;
    for (int i0 = 0; i0 < n; i0 += kIB) {
      __syncthreads();
      for (int idx = t; idx < kIB * n * NC; idx += E) {
        const int ib = idx / (n * NC), rem = idx - ib * (n * NC);
        const int i = i0 + ib;
        Ks[idx] = (i < n) ? Kp[(static_cast<int64_t>(i) * ld) * NC + rem] : 0.0;
      }
      __syncthreads();
      if (!valid) continue;
      double xr[kIB], xi[kIB];
#pragma unroll
      for (int ib = 0; ib < kIB; ++ib) xr[ib] = xi[ib] = 0.0;
      for (int l = 0; l < n; ++l) {
        const double2 wl = ld_c(Ws, l * E + t);
#pragma unroll
        for (int ib = 0; ib < kIB; ++ib) {
          const double k = Ks[(ib * n + l) * NC + c];
          xr[ib] = fma(k, wl.x, xr[ib]);
          xi[ib] = fma(k, wl.y, xi[ib]);
        }
      }
#pragma unroll
      for (int ib = 0; ib < kIB; ++ib) {
        const int i = i0 + ib;
        if (i >= n) break;
        const double2 wi = ld_c(Ws, i * E + t);
        sW = fma(wi.x, xr[ib], fma(wi.y, xi[ib], sW));
        const double2 ai = ld_c(AW, static_cast<int64_t>(i) * vstride + e);
        sA = fma(ai.x, xr[ib], fma(ai.y, xi[ib], sA));
      }
    }
    accD = fma(aD, sW, accD);
    accP = fma(aP, sW, accP);
    accA += sA;
  }
  // per-chain block sums (threads t, t + NC, ... hold chain c)
  __syncthreads();
  double* red = reinterpret_cast<double*>(smraw);
  red[t] = accD;
  red[E + t] = accP;
  red[2 * E + t] = accA;
  __syncthreads();
  if (t < NC) {
    for (int q = 0; q < 3; ++q) {
      double sum = 0.0;
      for (int j = t; j < E; j += NC) sum += red[q * E + j];
      partial[(static_cast<int64_t>(blockIdx.x) * NC + t) * 3 + q] = sum;
    }
  }
}

template <typename T, int NC, int kE>
cudaError_t launch(const DevSector& S, const T* W, const T* AW, int64_t vstride, const double* Kp, int n, int ld,
                   double* partial, int* grid, cudaStream_t st) {
  int dev = 0, sms = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const size_t smem = std::max(static_cast<size_t>(n) * kE * sizeof(T) + static_cast<size_t>(kIB) * n * NC * sizeof(double),
                               static_cast<size_t>(3) * kE * sizeof(double));
  if (n <= 0 || smem > static_cast<size_t>(optin)) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(moments_kernel<T, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  const int64_t nch = (vstride + kE - 1) / kE;
  const int per_sm = std::max(1, static_cast<int>(static_cast<size_t>(optin) / smem));
  const int64_t cap = static_cast<int64_t>(sms) * std::min(per_sm, 2);
  *grid = static_cast<int>(nch < cap ? (nch > 0 ? nch : 1) : cap);
  moments_kernel<T, NC><<<*grid, kE, smem, st>>>(S, W, AW, vstride, Kp, n, ld, partial);
  return cudaGetLastError();
}

}  // namespace

// Widest block whose slice of the n vectors fits in shared memory.
cudaError_t grad_moments_c64(const DevSector& S, const float2* W, const float2* AW, int64_t vstride, const double* Kp,
                             int n, int ld, double* partial, int* grid, cudaStream_t st) {
  cudaError_t e = launch<float2, 32, 256>(S, W, AW, vstride, Kp, n, ld, partial, grid, st);
  if (e == cudaErrorInvalidValue) e = launch<float2, 32, 128>(S, W, AW, vstride, Kp, n, ld, partial, grid, st);
  return e;
}

cudaError_t grad_moments_c128(const DevSector& S, const double2* W, const double2* AW, int64_t vstride,
                              const double* Kp, int n, int ld, double* partial, int* grid, cudaStream_t st) {
  cudaError_t e = launch<double2, 1, 128>(S, W, AW, vstride, Kp, n, ld, partial, grid, st);
  if (e == cudaErrorInvalidValue) e = launch<double2, 1, 64>(S, W, AW, vstride, Kp, n, ld, partial, grid, st);
  return e;
}

}  // namespace ftlm_b200
