// Host-side dense algebra on one Lanczos tridiagonal (n <= a few hundred): eigenvectors and the
// Duhamel weight matrix of the FTLM quadrature.  O(n^3) scalar work per chain, next to the
// O(dim) vector work that stays on the GPU.
#pragma once

#include <string>

namespace ftlm_b200 {

// Eigen-decomposition of the symmetric tridiagonal T (diagonal alpha[0..n), off-diagonal
// beta[0..n-1)) by implicit QL with Wilkinson-type shifts (Bowdler, Martin, Reinsch and Wilkinson,
// Numer. Math. 11 (1968), "tql2").  lam[j] ascending, Z row-major n x n with column j the
// eigenvector of lam[j].  Returns "" or an error message.
std::string tridiag_eigvec(int n, const double* alpha, const double* beta, double* lam, double* Z);

// For g(T) = e_1^T exp(-bT (T - lam_min)) e_1 (lam_min = lowest eigenvalue of T) and a symmetric
// perturbation T -> T + eps G, with lam_min held fixed:
//   dg/deps = -sum_il G_il K_il,
//   K = Z P Z^T, P_jk = Z_0j Z_0k (e^{-bT lam_j'} - e^{-bT lam_k'}) / (lam_k - lam_j)
// (divided difference of e^{-bT x}; bT e^{-bT lam_j'} on the diagonal; lam' = lam - lam_min): the
// Duhamel formula d e^{-bT T} = -int_0^bT e^{-(bT-t)T} dT e^{-tT} dt in the eigenbasis.
// Outputs K (row-major n x n), g and the lowest eigenvalue.  Returns "" or an error message.
std::string duhamel_weights(int n, const double* alpha, const double* beta, double bT, double* K, double* g,
                            double* lam_min);

// Eigenvalues (ascending) of a dense real symmetric m x m matrix A (row-major, overwritten) by
// cyclic Jacobi rotations (Rutishauser's formulation) until the off-diagonal norm is below
// 1e-15 of the Frobenius norm.  Returns "" or an error message.
std::string sym_eigvals(int m, double* A, double* lam);

}  // namespace ftlm_b200
