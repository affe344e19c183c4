// Krylov moments for the FTLM parameter gradient (grad.cu).
//
// For one chain c with stored (unnormalised) Lanczos vectors W_0..W_{n-1} and a real symmetric
// weight matrix K'_c (scales 1/(b_i b_l) folded in), the kernel returns per chain
//   m0 = sum_il K'_il <W_i| D |W_l>,  m1 = sum_il K'_il <W_i| P |W_l>,  m2 = sum_il K'_il <A W_i|W_l>
// with D = number of doubly occupied sites, P = sum over neighbour pairs of n_i n_j (both
// diagonal, evaluated from the sector tables) and A W_i supplied by the caller (the t' hopping
// operator applied to each W_i).  Vectors are [state][NC chains]: NC = 32 complex64 (block
// vectors of the batched path) or NC = 1 complex128 (one chain of the plain path).
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

namespace ftlm_b200 {

// Kp: [n][ld][NC] (row i, column l, chain fastest).  partial: [grid][NC][3] doubles, grid returned
// in *grid (at most 2 * SM count blocks).  smem needs n * E * sizeof(element) + 2 * n * NC * 8
// bytes with E = 256 (NC = 32) or 128 (NC = 1) elements per block; fails with
// cudaErrorInvalidValue when that exceeds the device's limit.
cudaError_t grad_moments_c64(const DevSector& S, const float2* W, const float2* AW, int64_t vstride, const double* Kp,
                             int n, int ld, double* partial, int* grid, cudaStream_t st);
cudaError_t grad_moments_c128(const DevSector& S, const double2* W, const double2* AW, int64_t vstride,
                              const double* Kp, int n, int ld, double* partial, int* grid, cudaStream_t st);

}  // namespace ftlm_b200
