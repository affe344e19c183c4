// Translation-orbit k-block kernels (orbit.cu).  Reference: OrbitKBlockBasis::build and
// apply_orbit_k_block (src/orbit_k_block_basis.cpp:70-220), orbit helpers
// (include/ftlm/symmetry/orbit.hpp:93-156), fermionic translation sign
// (include/ftlm/symmetry/fermionic_translation.hpp:32-54), Bloch phase
// (include/ftlm/symmetry/momentum_sector.hpp:57-63).
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

namespace ftlm_b200 {

struct OrbitDev {
  int n, Lx, Ly, G;        // sites, lattice, translation group order
  int64_t Du, Dd, dim;     // full sector
  const uint32_t* umask;   // [Du] (sector tables)
  const uint32_t* dmask;   // [Dd]
  const int32_t* rank_u;   // [65536] mask -> rank of the up string (-1 outside)
  const int32_t* rank_d;   // [65536]
  const uint16_t* tlut;    // [G][2][256]: T_R(m) = tlut[R][0][m & 255] | tlut[R][1][m >> 8]
  const uint8_t* tsite;    // [G][16] translated site of each site
  const uint8_t* rorder;   // [G] translations in the reference's search order (dx outer, dy inner)
};

// Per full state: full index of its canonical representative, and (R | eta<<4) with
// T_R rep = state (first R in the reference's search order), eta = fermionic sign of T_R on rep.
cudaError_t orbit_canon(const OrbitDev& O, int32_t* rep_full, uint8_t* reta, cudaStream_t st);
// Order-preserving device compaction (scratch `counts` of orbit_compact_counts(n) ints): a count
// call (synchronises st to return the number) and a write call into outputs of that size.
int64_t orbit_compact_counts(int64_t n);
// The sector's orbit representatives in ascending packed (up<<16 | dn) order: inv_u / inv_d list the
// up / down ranks by ascending mask value; packed[], full[] receive the representatives and their
// full indices.
cudaError_t orbit_count_reps(const OrbitDev& O, const int32_t* rep_full, const int32_t* inv_u, const int32_t* inv_d,
                             int32_t* counts, int64_t* nreps, cudaStream_t st);
cudaError_t orbit_write_reps(const OrbitDev& O, const int32_t* rep_full, const int32_t* inv_u, const int32_t* inv_d,
                             const int32_t* counts, uint32_t* packed, int64_t* full, cudaStream_t st);

// The representatives of one momentum block: those with |A(K)| > tol, in order.
struct OrbitBlockIn {
  const uint32_t* reps;   // [nreps] packed, ascending
  const int64_t* full;    // [nreps]
  const double* absA;     // [nreps]
  const double2* A;       // [nreps]
  const int* stab;        // [nreps]
};
struct OrbitBlockOut {
  uint32_t* reps;
  int64_t* full;
  double* absA;
  double2* A;
  int* stab;
  int64_t* orbit_idx;     // index among all representatives
  double* sqrtA;
};
cudaError_t orbit_count_survivors(const double* absA, int64_t nreps, double tol, int32_t* counts, int64_t* dk,
                                  cudaStream_t st);
cudaError_t orbit_write_survivors(const OrbitBlockIn& in, int64_t nreps, double tol, const int32_t* counts,
                                  const OrbitBlockOut& out, cudaStream_t st);

// |A(K)| per representative: A = sum over stabiliser S of eta(rep,S) chi*(S) (chi* from chi_tab);
// optionally A itself and the stabiliser size (A, stab may be null).
cudaError_t orbit_absA(const OrbitDev& O, const uint32_t* reps_packed, int64_t nreps, const double2* chi_tab,
                       double* absA, double2* A, int* stab, cudaStream_t st);
// table[state] = beta | R<<24 | eta<<28 (beta = reduced index of its orbit at K) or 0xFFFFFFFF.
cudaError_t orbit_table(const OrbitDev& O, const int32_t* rep_full, const uint8_t* reta, const int32_t* red_of_full,
                        uint32_t* table, cudaStream_t st);

struct OrbitApplyDev {
  OrbitDev O;
  DevSector S;               // hop tables, diagonal tables of the sector
  int64_t dk;                // reduced dimension
  const uint32_t* reps;      // [dk] packed up<<16 | dn
  const double* sqrtA;       // [dk] sqrt(|A|)
  const uint32_t* table;     // [dim]
  const double2* chi_tab;    // [G] translation_bloch_phase(K, R)
  const int32_t* uhop_from;  // merged up hops: from, to, coefficient, JW masks
  const int32_t* uhop_to;
  const double2* uhop_c;
  const uint32_t* uhop_own;
  const uint32_t* uhop_oth;
  int n_uhops;
  const int32_t* dhop_from;
  const int32_t* dhop_to;
  const double2* dhop_c;
  const uint32_t* dhop_own;
  const uint32_t* dhop_oth;
  int n_dhops;
  double2* xs;               // [dk] workspace: sqrt(|A_b|) x_b, zero where |x_b|^2 < 1e-28
  int path;                  // 0: hop list per representative; 1: sector gather tables (default)
};

// red[full[b]] = b for b < n.
cudaError_t orbit_scatter_index(const int64_t* full, int64_t n, int32_t* red, cudaStream_t st);

// y = H_K x on reduced complex128 vectors (gather form of apply_orbit_k_block).
cudaError_t orbit_apply(const OrbitApplyDev& A, const double2* x, double2* y, cudaStream_t st);

}  // namespace ftlm_b200
