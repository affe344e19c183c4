// Fused Lanczos for many small sectors (chains.cu): one CTA per chain runs all M steps of the
// src/lanczos.cpp:180-205 recurrence on vectors of its own sector, so a whole sweep of small
// sectors is one launch instead of M host-synchronised steps per chain.
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

namespace ftlm_b200 {

struct ChainDesc {
  int sector;   // index into the DevSector array
  int out;      // row of alpha/beta/used written by this chain
  int64_t off;  // first element of the chain's three vectors (q, q_prev, w) in the scratch
};

// q_0 of every chain (normalised) at scratch[off]; outputs alpha/beta [out][M] (beta of a chain
// that broke down at step k: k entries), used [out].  Deterministic (fixed per-CTA order).
// wide: 1024 threads per chain (for larger sectors) instead of 256.
cudaError_t chains_lanczos(const DevSector* sectors, const ChainDesc* chains, int nc, int M, double2* scratch,
                           double* alpha, double* beta, int* used, bool wide, cudaStream_t st);

}  // namespace ftlm_b200
