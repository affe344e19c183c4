// Small dense symmetric eigen-problems on the GPU (symeig.cu): parallel cyclic Jacobi, one CTA per
// matrix, and the Duhamel weights of the parameter gradient.
#pragma once

#include <cuda_runtime.h>

namespace ftlm_b200 {

constexpr int kMaxEig = 160;  // largest order (the matrix sits in shared memory)

// Tridiagonals alpha/beta [nm][ld] of orders n[nm] (0 <= n <= ld <= 160): eigenvalues ascending
// into lam [nm][ld]; v0 (may be null): squared first components [nm][ld] (quadrature weights);
// vt (may be null): eigenvectors as rows, [nm][ld][ld].  info [nm] (may be null): 0 converged,
// 1 not converged after 60 sweeps, 2 order out of range (nothing written).
cudaError_t symeig_tridiag(const double* alpha, const double* beta, const int* n, int nm, int ld, double* lam,
                           double* v0, double* vt, int* info, cudaStream_t st);
// Dense symmetric matrices A [nm][ld*ld] (row-major, orders n[nm]): eigenvalues ascending into lam.
cudaError_t symeig_dense(const double* A, const int* n, int nm, int ld, double* lam, int* info, cudaStream_t st);
// Real symmetric embedding [[Re H, -Im H], [Im H, Re H]] (2dk x 2dk, row-major) of a Hermitian
// matrix given by its columns (column j at cols + j*dk).
cudaError_t embed_hermitian(const double2* cols, int dk, double* R, cudaStream_t st);
// Duhamel weights of nc chains from symeig_tridiag's lam / vt: Kp[(i*ld + l)*nc + c] =
// K_il / (scale[c][i] scale[c][l]) for i, l < n[c] (other entries untouched: clear Kp first);
// g[c] = sum_j Z_0j^2 e^{-bT (lam_j - lam_0)}, lmin[c] = lam_0.  Y: scratch [nc][ld][ld].
cudaError_t duhamel_weights_dev(const double* lam, const double* vt, const int* n, int nc, int ld, double bT,
                                const double* scale, double* Y, double* Kp, double* g, double* lmin, cudaStream_t st);

}  // namespace ftlm_b200
