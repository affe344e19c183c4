// Device-side view of a sector plan (see plan.hpp) and small helpers shared by the kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ftlm_b200 {

struct DevGauge {
  const uint32_t* ent;  // entries, [group] rounds of 32
  const int4* grp;      // [ngroups]: entry offset, real-section rounds, table-section rounds, 0
  const double2* tab;   // [nt] table-section coefficients
  int nt;
  double real2[2];      // real-section coefficients
  int phase;            // 1: table-section coefficients are real2[cls] * (pc, +-ps) (entry bits 30, 27)
  double pc, ps;
  int xor_real;         // 1: real-section coefficient = real2[0] with its high word ^ (entry & 0xFFFC0000)
  const uint8_t* perm;  // [ngroups * 32]: lane L of group g serves string g*32 + perm[g*32 + L]
};

// The output string served by table position c (group c / 32, lane c % 32).
__device__ __forceinline__ int gauge_string(const DevGauge& G, int c) { return (c & ~31) | G.perm[c]; }

struct DevSector {
  int n;
  int64_t Du, Dd, dim;
  double U, V;
  const uint32_t* umask;   // [Du]
  const uint32_t* dmask;   // [Dd]
  const int32_t* cnt_uu;   // [Du]
  const int32_t* cnt_dd;   // [Dd]
  const uint4* wpl;        // [Du]
  const int32_t* up_ptr;   // [Du+1]
  const int32_t* up_src;   // [nnz_up]
  const double2* up_coef;  // [nnz_up]
  const uint32_t* up_lohi; // [nnz_up]
  // Packed up list of the column pass (SectorPlan::up_pk), nullptr when the sector has none:
  // src | lo<<14 | hi<<19 | conj<<28 | phase<<29 | cls<<30 | s<<31.
  const uint32_t* up_pk;   // [nnz_up]
  double up_real2[2];
  double up_pc, up_ps;
  const int64_t* dn_gptr;  // [ngroups+1]
  const uint32_t* dn_ent;  // ELL entries
  const int64_t* dn_csr_ptr;   // [Dd+1] unpadded down-hop lists (batched path)
  const uint32_t* dn_csr_ent;
  const float2* up_coef32;     // [nnz_up] complex64 copies for the batched path
  const float2* dn_coef32;     // [n_dn_hops+1]
  const float2* dn_coef32s;    // [2*(n_dn_hops+1)]: [2*hop + s] = (-1)^s coef (the gauge-basis row pass)
  const double2* dn_coef;  // [n_dn_hops+1]
  const uint32_t* dn_nmask;// [n_dn_hops+1]
  int n_dn_hops;           // == pad hop id
  int* flags;              // [0]: input has a non-zero entry with |x|^2 < 1e-28
  // Gauge-basis down-hop table of the row pass (plan.hpp, GaugeTable); dn_g.ent == nullptr when the
  // sector has none or the launch uses the per-row table instead.
  DevGauge dn_g;
  int bt_cols;              // batched column-pass variant: 0/1/2 = 16/8/4-column chunks
};

// The reference skips source columns with std::norm(x) < 1e-28
// (src/hubbard_hamiltonian.cpp:62); a skipped source contributes exactly nothing.
__device__ __forceinline__ bool tiny(double2 v) { return v.x * v.x + v.y * v.y < 1e-28; }

// Inclusive prefix XOR of the down string, shifted left by one: bit k = parity(#dn in [0,k)).
__device__ __forceinline__ uint32_t prefix_parity_shifted(uint32_t d) {
  uint32_t p = d;
  p ^= p << 1;
  p ^= p << 2;
  p ^= p << 4;
  p ^= p << 8;
  p ^= p << 16;
  return p << 1;
}

__device__ __forceinline__ double diag_value(const DevSector& S, uint32_t u, uint32_t d, int cuu, int cdd, uint4 w) {
  const int cross = __popc(d & w.x) + 2 * __popc(d & w.y) + 4 * __popc(d & w.z) + 8 * __popc(d & w.w);
  return S.U * static_cast<double>(__popc(u & d)) + S.V * static_cast<double>(cuu + cdd + cross);
}

// Sign of the basis state (u, d) in the spin-ordered ("gauge") basis: with
// g = (-1)^{#(up site, down site) pairs with the down site below the up site}, G H G (G = diag g)
// is diag + U x 1 + 1 x D, the up-hop part independent of the down string and the down-hop part
// independent of the up string (each keeps only its own species' Jordan-Wigner signs).
__device__ __forceinline__ uint32_t gauge_sign(uint32_t u, uint32_t d) {
  return static_cast<uint32_t>(__popc(u & prefix_parity_shifted(d))) & 1u;
}

// acc += (neg ? -c : c) * v   (complex)
__device__ __forceinline__ void cmac(double2& acc, double2 c, double2 v, uint32_t neg) {
  if (neg) {
    c.x = -c.x;
    c.y = -c.y;
  }
  acc.x = fma(c.x, v.x, acc.x);
  acc.x = fma(-c.y, v.y, acc.x);
  acc.y = fma(c.x, v.y, acc.y);
  acc.y = fma(c.y, v.x, acc.y);
}

// (H x)[idx] in gather form from the sector tables: diagonal, down hops (ELL group of the column,
// sources in the same row), up hops (CSR of the row, sources in the same column), with the
// reference's source-skip rule.  The generic H·v kernel and the fused small-sector Lanczos use it.
__device__ __forceinline__ double2 hv_element(const DevSector& S, const double2* __restrict__ x, int64_t idx) {
  const int64_t r = idx / S.Dd;
  const int64_t c = idx - r * S.Dd;
  const uint32_t u = S.umask[r];
  const uint32_t d = S.dmask[c];
  double2 acc = make_double2(0.0, 0.0);
  const double2 xv = x[idx];
  if (!tiny(xv)) {
    const double dg = diag_value(S, u, d, S.cnt_uu[r], S.cnt_dd[c], S.wpl[r]);
    acc.x = dg * xv.x;
    acc.y = dg * xv.y;
  }
  const double2* xrow = x + r * S.Dd;
  const int64_t g = c >> 5;
  const int lane = static_cast<int>(c & 31);
  const int64_t e_end = S.dn_gptr[g + 1];
  for (int64_t p = S.dn_gptr[g] + lane; p < e_end; p += 32) {
    const uint32_t ent = S.dn_ent[p];
    const int h = static_cast<int>((ent >> 1) & 511u);
    if (h == S.n_dn_hops) continue;
    const double2 xs = xrow[ent >> 10];
    if (tiny(xs)) continue;
    const uint32_t neg = (ent & 1u) ^ (static_cast<uint32_t>(__popc(u & S.dn_nmask[h])) & 1u);
    cmac(acc, S.dn_coef[h], xs, neg);
  }
  const uint32_t q = prefix_parity_shifted(d);
  const int j_end = S.up_ptr[r + 1];
  for (int j = S.up_ptr[r]; j < j_end; ++j) {
    const double2 xs = x[static_cast<int64_t>(S.up_src[j]) * S.Dd + c];
    if (tiny(xs)) continue;
    const uint32_t lh = S.up_lohi[j];
    const uint32_t neg = ((q >> (lh & 255u)) ^ (q >> (lh >> 8))) & 1u;
    cmac(acc, S.up_coef[j], xs, neg);
  }
  return acc;
}

}  // namespace ftlm_b200
