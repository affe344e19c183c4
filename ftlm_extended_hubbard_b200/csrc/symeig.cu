// Small dense symmetric eigen-problems on the GPU (FP64), one CTA per matrix:
//
//   symeig_kernel   parallel cyclic Jacobi (Brent-Luk round-robin ordering: m/2 disjoint rotations
//                   per round, m-1 rounds per sweep, sweeps until the off-diagonal Frobenius norm is
//                   below 1e-15 of the matrix norm), the matrix in shared memory (m <= 160, row
//                   stride m+1 so that column accesses of a warp fall in distinct bank pairs).  Input
//                   dense or tridiagonal; output eigenvalues in ascending order, optionally the squared
//                   first row of the eigenvector matrix (the quadrature weights) or all eigenvectors
//                   (row j of Vt = eigenvector j).
//   duhamel_kernel  the Duhamel weight matrix of one Lanczos chain from its eigen-decomposition:
//                   K = Z P Z^T, P_jk = Z_0j Z_0k (e^{-b l_j} - e^{-b l_k}) / (l_k - l_j) (the limit
//                   b e^{-b l_j} on the diagonal), with the same shift l_0 and the same expm1 form
//                   as the host restatement (tridiag.cpp), written in the moment kernel's layout.
//
// These replace host eigen-solves on the product paths: the converged quadrature of the
// differentiable forward, the gradient's Duhamel weights and the exact small-block ED of the
// k-resolved path (reference benchmarks/bench_ftlm_nmu_4x4_k.cpp:249-336 restated).
#include <cfloat>

#include "symeig.cuh"

namespace ftlm_b200 {

namespace {

constexpr int kEigThreads = 256;

// Pair k of round r of the circle method for m (even) players: player m-1 is fixed.
__device__ __forceinline__ void rr_pair(int r, int k, int m, int* p, int* q) {
  int a, b;
  if (k == 0) {
    a = r;
    b = m - 1;
  } else {
    a = (r + k) % (m - 1);
    b = (r - k + (m - 1)) % (m - 1);
  }
  *p = min(a, b);
  *q = max(a, b);
}

template <int kV>  // 0: eigenvalues only, 1: + first row of V, 2: + all eigenvectors (Vt rows)
__global__ void __launch_bounds__(kEigThreads) symeig_kernel(const double* __restrict__ dense,
                                                             const double* __restrict__ alpha,
                                                             const double* __restrict__ beta,
                                                             const int* __restrict__ nv, int ld,
                                                             double* __restrict__ lam, double* __restrict__ v0,
                                                             double* __restrict__ vt, int* __restrict__ info) {
  extern __shared__ double sm[];
  __shared__ double rc[kMaxEig / 2], rs[kMaxEig / 2];
  __shared__ int rp[kMaxEig / 2], rq[kMaxEig / 2];
  __shared__ double red[kEigThreads / 32];
  __shared__ int s_done;
  const int ch = blockIdx.x;
  const int tid = threadIdx.x;
  int n = nv[ch];
  if (n < 0 || n > ld || ld > kMaxEig) {  // out of range: report, touch nothing
    if (tid == 0 && info) info[ch] = 2;
    return;
  }
  double* lo = lam + static_cast<int64_t>(ch) * ld;
  if (n == 0) {
    if (tid == 0 && info) info[ch] = 0;
    return;
  }
  const int m = n + (n & 1);  // even order; a padding index stays decoupled (zero row and column)
  const int S = m + 1;        // row stride in shared memory
  double* A = sm;
  double* V0 = sm + static_cast<size_t>(m) * S;  // first row of V (kV == 1)
  double* Vt = vt ? vt + static_cast<int64_t>(ch) * ld * ld : nullptr;  // kV == 2, rows = eigenvectors
  for (int i = tid; i < m * S; i += kEigThreads) {
    const int r = i / S, c = i - r * S;
    double v = 0.0;
    if (r < n && c < n) {
      if (dense) {
        v = dense[static_cast<int64_t>(ch) * ld * ld + static_cast<int64_t>(r) * ld + c];
      } else {
        const double* a = alpha + static_cast<int64_t>(ch) * ld;
        const double* b = beta + static_cast<int64_t>(ch) * ld;
        if (r == c) v = a[r];
        else if (c == r + 1) v = b[r];
        else if (r == c + 1) v = b[c];
      }
    }
    A[i] = v;
  }
  if (kV == 1)
    for (int i = tid; i < m; i += kEigThreads) V0[i] = (i == 0) ? 1.0 : 0.0;
  if (kV == 2)
    for (int i = tid; i < m * m; i += kEigThreads) {
      const int r = i / m, c = i - r * m;
      if (r < n && c < n) Vt[static_cast<int64_t>(r) * ld + c] = (r == c) ? 1.0 : 0.0;
    }
  __syncthreads();
  // Frobenius norm for the stopping rule
  double fro = 0.0;
  for (int i = tid; i < m * S; i += kEigThreads) fro += A[i] * A[i];
  for (int off = 16; off > 0; off >>= 1) fro += __shfl_down_sync(0xffffffffu, fro, off);
  if ((tid & 31) == 0) red[tid >> 5] = fro;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < kEigThreads / 32; ++w) t += red[w];
    red[0] = t;
  }
  __syncthreads();
  const double stop = 1e-30 * red[0];  // off^2 <= (1e-15 ||A||_F)^2
  const int half = m / 2;
  int sweep = 0;
  for (; sweep < 60; ++sweep) {
    // off-diagonal norm
    double off2 = 0.0;
    for (int i = tid; i < m * S; i += kEigThreads) {
      const int r = i / S, c = i - r * S;
      if (c < m && r != c) off2 += A[i] * A[i];
    }
    for (int o = 16; o > 0; o >>= 1) off2 += __shfl_down_sync(0xffffffffu, off2, o);
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = off2;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < kEigThreads / 32; ++w) t += red[w];
      s_done = !(t > stop);
    }
    __syncthreads();
    if (s_done) break;
    for (int r = 0; r < m - 1; ++r) {
      for (int k = tid; k < half; k += kEigThreads) {
        int p, q;
        rr_pair(r, k, m, &p, &q);
        const double apq = A[p * S + q];
        double c = 1.0, s = 0.0;
        if (apq != 0.0) {
          const double theta = (A[q * S + q] - A[p * S + p]) / (2.0 * apq);
          const double t = copysign(1.0, theta) / (fabs(theta) + sqrt(theta * theta + 1.0));
          c = 1.0 / sqrt(t * t + 1.0);
          s = t * c;
        }
        rc[k] = c;
        rs[k] = s;
        rp[k] = p;
        rq[k] = q;
      }
      __syncthreads();
      // rows: A <- J^T A
      for (int i = tid; i < half * m; i += kEigThreads) {
        const int k = i / m, j = i - k * m;
        const int p = rp[k], q = rq[k];
        const double c = rc[k], s = rs[k];
        const double x = A[p * S + j], y = A[q * S + j];
        A[p * S + j] = c * x - s * y;
        A[q * S + j] = s * x + c * y;
      }
      __syncthreads();
      // columns: A <- A J (and V <- V J)
      for (int i = tid; i < half * m; i += kEigThreads) {
        const int k = i / m, j = i - k * m;
        const int p = rp[k], q = rq[k];
        const double c = rc[k], s = rs[k];
        const double x = A[j * S + p], y = A[j * S + q];
        A[j * S + p] = c * x - s * y;
        A[j * S + q] = s * x + c * y;
      }
      if (kV == 1)
        for (int k = tid; k < half; k += kEigThreads) {
          const int p = rp[k], q = rq[k];
          const double c = rc[k], s = rs[k];
          const double x = V0[p], y = V0[q];
          V0[p] = c * x - s * y;
          V0[q] = s * x + c * y;
        }
      if (kV == 2)
        for (int i = tid; i < half * m; i += kEigThreads) {
          const int k = i / m, j = i - k * m;
          const int p = rp[k], q = rq[k];
          if (p >= n || q >= n || j >= n) continue;  // the padding index never mixes (its column is zero)
          const double c = rc[k], s = rs[k];
          double* vp = Vt + static_cast<int64_t>(p) * ld;
          double* vq = Vt + static_cast<int64_t>(q) * ld;
          const double x = vp[j], y = vq[j];
          vp[j] = c * x - s * y;
          vq[j] = s * x + c * y;
        }
      __syncthreads();
      for (int k = tid; k < half; k += kEigThreads) {  // the rotation annihilates a_pq
        const int p = rp[k], q = rq[k];
        if (rs[k] != 0.0) {
          A[p * S + q] = 0.0;
          A[q * S + p] = 0.0;
        }
      }
      __syncthreads();
    }
  }
  if (tid == 0 && info) info[ch] = s_done ? 0 : 1;
  // ascending order (ties by index): rank sort over the n real eigenvalues (the padding index, if
  // any, is index n and excluded)
  __syncthreads();
  for (int j = tid; j < n; j += kEigThreads) {
    const double lj = A[j * S + j];
    int rank = 0;
    for (int k = 0; k < n; ++k) {
      const double lk = A[k * S + k];
      rank += (lk < lj || (lk == lj && k < j)) ? 1 : 0;
    }
    lo[rank] = lj;
    if (kV == 1) v0[static_cast<int64_t>(ch) * ld + rank] = V0[j] * V0[j];  // weight Z_0j^2
    if (kV == 2) reinterpret_cast<int*>(V0)[j] = rank;  // permutation for the row move below
  }
  if (kV == 2) {
    // Vt rows to ascending order: eigenvector j belongs at row rank(j); move through the row-0
    // scratch of shared memory one destination row at a time (rows are n <= 160 doubles).
    __syncthreads();
    const int* rk = reinterpret_cast<const int*>(V0);
    double* tmp = A;  // A's diagonal was consumed above; reuse its storage
    for (int i = tid; i < n * n; i += kEigThreads) {
      const int j = i / n, c = i - j * n;
      tmp[rk[j] * n + c] = Vt[static_cast<int64_t>(j) * ld + c];
    }
    __syncthreads();
    for (int i = tid; i < n * n; i += kEigThreads) {
      const int j = i / n, c = i - j * n;
      Vt[static_cast<int64_t>(j) * ld + c] = tmp[i];
    }
  }
}

// K = Z P Z^T in the moment kernel's layout Kp[(i*ld + l)*nc + c] / (sc_i sc_l), with
// Z[i][j] = Vt[j][i] (ascending l_j); g = sum_j Z_0j^2 e^{-b (l_j - l_0)}, lmin = l_0.
__global__ void __launch_bounds__(kEigThreads) duhamel_kernel(const double* __restrict__ lam,
                                                              const double* __restrict__ vt,
                                                              const int* __restrict__ nv, int ld, int nc, double bT,
                                                              const double* __restrict__ scale,
                                                              double* __restrict__ Y, double* __restrict__ Kp,
                                                              double* __restrict__ g_out,
                                                              double* __restrict__ lmin_out) {
  const int ch = blockIdx.x;
  const int tid = threadIdx.x;
  const int n = nv[ch];
  if (n <= 0 || n > ld) return;
  const double* l = lam + static_cast<int64_t>(ch) * ld;
  const double* V = vt + static_cast<int64_t>(ch) * ld * ld;  // V[j*ld + i] = Z[i][j]
  double* y = Y + static_cast<int64_t>(ch) * ld * ld;
  const double* sc = scale + static_cast<int64_t>(ch) * ld;
  const double shift = l[0];
  __shared__ double ew[kMaxEig];
  for (int j = tid; j < n; j += kEigThreads) ew[j] = exp(-bT * (l[j] - shift));
  __syncthreads();
  // Y[i][k] = sum_j Z_ij Z_0j D_jk, then K_il = sum_k Y_ik Z_0k Z_lk
  for (int e = tid; e < n * n; e += kEigThreads) {
    const int i = e / n, k = e - i * n;
    double acc = 0.0;
    for (int j = 0; j < n; ++j) {
      const int a = min(j, k), b = max(j, k);
      const double ea = ew[a];
      const double delta = l[b] - l[a];
      const double D = (a == b || delta == 0.0) ? bT * ea : ea * (-expm1(-bT * delta)) / delta;
      acc += V[static_cast<int64_t>(j) * ld + i] * V[static_cast<int64_t>(j) * ld] * D;
    }
    y[static_cast<int64_t>(i) * ld + k] = acc;
  }
  __syncthreads();
  for (int e = tid; e < n * n; e += kEigThreads) {
    const int i = e / n, lq = e - i * n;
    double acc = 0.0;
    for (int k = 0; k < n; ++k)
      acc += y[static_cast<int64_t>(i) * ld + k] * V[static_cast<int64_t>(k) * ld] * V[static_cast<int64_t>(k) * ld + lq];
    Kp[(static_cast<int64_t>(i) * ld + lq) * nc + ch] = acc / (sc[i] * sc[lq]);
  }
  if (tid == 0) {
    double gs = 0.0;
    for (int j = 0; j < n; ++j) {
      const double z0 = V[static_cast<int64_t>(j) * ld];
      gs += z0 * z0 * ew[j];
    }
    g_out[ch] = gs;
    lmin_out[ch] = shift;
  }
}

// R = [[Re H, -Im H], [Im H, Re H]] (2dk x 2dk, row-major) from the columns of H (column j at
// cols + j*dk): the real symmetric embedding of a Hermitian matrix (each eigenvalue twice).
__global__ void embed_kernel(const double2* __restrict__ cols, int dk, double* __restrict__ R) {
  const int m = 2 * dk;
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= static_cast<int64_t>(dk) * dk) return;
  const int j = static_cast<int>(e / dk), i = static_cast<int>(e - static_cast<int64_t>(j) * dk);
  const double2 h = cols[static_cast<int64_t>(j) * dk + i];  // H[i][j]
  R[static_cast<int64_t>(i) * m + j] = h.x;
  R[static_cast<int64_t>(i) * m + j + dk] = -h.y;
  R[static_cast<int64_t>(i + dk) * m + j] = h.y;
  R[static_cast<int64_t>(i + dk) * m + j + dk] = h.x;
}

}  // namespace

cudaError_t embed_hermitian(const double2* cols, int dk, double* R, cudaStream_t st) {
  const int64_t tot = static_cast<int64_t>(dk) * dk;
  if (tot <= 0) return cudaSuccess;
  embed_kernel<<<static_cast<unsigned>((tot + 255) / 256), 256, 0, st>>>(cols, dk, R);
  return cudaGetLastError();
}

cudaError_t symeig_tridiag(const double* alpha, const double* beta, const int* n, int nm, int ld, double* lam,
                           double* v0, double* vt, int* info, cudaStream_t st) {
  if (nm <= 0) return cudaSuccess;
  if (ld > kMaxEig || ld <= 0) return cudaErrorInvalidValue;
  const int m = ld + (ld & 1);
  const size_t sm = (static_cast<size_t>(m) * (m + 1) + m) * sizeof(double);
  cudaError_t e;
  if (vt) {
    e = cudaFuncSetAttribute(symeig_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm));
    if (e == cudaSuccess) symeig_kernel<2><<<nm, kEigThreads, sm, st>>>(nullptr, alpha, beta, n, ld, lam, v0, vt, info);
  } else if (v0) {
    e = cudaFuncSetAttribute(symeig_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm));
    if (e == cudaSuccess) symeig_kernel<1><<<nm, kEigThreads, sm, st>>>(nullptr, alpha, beta, n, ld, lam, v0, vt, info);
  } else {
    e = cudaFuncSetAttribute(symeig_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm));
    if (e == cudaSuccess) symeig_kernel<0><<<nm, kEigThreads, sm, st>>>(nullptr, alpha, beta, n, ld, lam, v0, vt, info);
  }
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t symeig_dense(const double* A, const int* n, int nm, int ld, double* lam, int* info, cudaStream_t st) {
  if (nm <= 0) return cudaSuccess;
  if (ld > kMaxEig || ld <= 0) return cudaErrorInvalidValue;
  const int m = ld + (ld & 1);
  const size_t sm = (static_cast<size_t>(m) * (m + 1) + m) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(symeig_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm));
  if (e != cudaSuccess) return e;
  symeig_kernel<0><<<nm, kEigThreads, sm, st>>>(A, nullptr, nullptr, n, ld, lam, nullptr, nullptr, info);
  return cudaGetLastError();
}

cudaError_t duhamel_weights_dev(const double* lam, const double* vt, const int* n, int nc, int ld, double bT,
                                const double* scale, double* Y, double* Kp, double* g, double* lmin, cudaStream_t st) {
  if (nc <= 0) return cudaSuccess;
  duhamel_kernel<<<nc, kEigThreads, 0, st>>>(lam, vt, n, ld, nc, bT, scale, Y, Kp, g, lmin);
  return cudaGetLastError();
}

}  // namespace ftlm_b200
