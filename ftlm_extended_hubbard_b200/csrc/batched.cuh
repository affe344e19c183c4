// Batched complex64 FTLM kernels (batched.cu): 32 chains of one sector per block vector.
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"
#include "orbit.cuh"

namespace ftlm_b200 {

constexpr int kBtBlocksPerSm = 5;
constexpr int kBtBlocks = kBtBlocksPerSm * 148;  // fixed persistent grid: deterministic reductions
constexpr int kBtChains = 32;   // chains per block vector (one warp lane each)
// Per-chain scalar state, st[field * 32 + chain] (doubles).
constexpr int kBtSin = 0;     // 1 / beta_{k-1}: scale of H W_k
constexpr int kBtC1r = 1;     // z / beta_{k-1} (coefficient of W_k), real and imaginary parts
constexpr int kBtC1i = 2;
constexpr int kBtC2 = 3;      // beta_{k-1} / beta_{k-2} (coefficient of W_{k-1})
constexpr int kBtActive = 4;  // 1 while the chain has not broken down
constexpr int kBtFields = 8;
constexpr int kBtPartialDoubles = kBtBlocks * kBtChains * 2;

// W <- complex64 Philox start vectors (chain r: key seed + r*100003), norms -> scalar state.
// flags: 2 ints (tiny-entry flags of the current and next vector, cleared here).  gauge: the sector
// whose spin-ordered basis the block vectors of bt_step live in (the start vector G r, G the
// diagonal sign matrix of gauge_sign); null for orbit blocks (their own basis).
cudaError_t bt_start(float2* W, int64_t dim, unsigned seed, double* st, double* partial, int* used, int* flags,
                     cudaStream_t s, const DevSector* gauge);
// One Lanczos step k for all chains on block vectors in the sector's gauge basis (bt_start with
// gauge = &S): Y <- H W_k, z, W_{k+1} (into Y), beta_k; alpha/beta [M][32].  G H G has the same
// spectrum and the start vectors are G r, so alpha/beta are those of the original basis.
cudaError_t bt_step(const DevSector& S, const float2* Wk, const float2* Wkm1, float2* Y, int k, double* st,
                    double* partial, double* alpha, double* beta, int* used, int* flags, cudaStream_t s);

// One Lanczos step for 32 chains of an orbit momentum block (block vectors over its dk
// representatives); same contract as bt_step.  Needs the sector's max up-degree <= 120 and at most
// 256 sources per representative.
cudaError_t bt_orbit_step(const OrbitApplyDev& A, const float2* Wk, const float2* Wkm1, float2* Y, int k, double* st,
                          double* partial, double* alpha, double* beta, int* used, int* flags, cudaStream_t s);

// Y = (G H G) X for one block vector in the gauge basis, without Lanczos bookkeeping (st_unit is
// unused), zero_flag points to an int 0 (no small-entry filter), partial receives unused dot sums.
cudaError_t bt_apply(const DevSector& S, const float2* X, float2* Y, const double* st_unit, double* partial,
                     const int* zero_flag, cudaStream_t s);

}  // namespace ftlm_b200
