// H·v kernels for one (N_up, N_dn) sector, complex128.  State (ru, rd) lives at ru*Dd + rd,
// so the vector is a Du x Dd row-major matrix X[up string][down string].
//
//   H X = diag o X  +  (down hops: mix columns inside a row)  +  (up hops: mix rows, column-wise)
//
// Paths:
//   hv_generic  one thread per output element, everything gathered from global memory.  Any size.
//   hv_rows     pass 1 of the fast path: persistent CTAs, one output row at a time; the input
//               row is staged in shared memory (down hops gather inside it); writes
//               y = diag o x + down part.  Requires a down row (+ coefficient table) to fit in SMEM.
//               Two forms: hv_rows (per-row coefficient table in shared memory; any hop list)
//               and hv_rows_gauge (the row computed in the spin-ordered basis, where down-hop
//               coefficients do not depend on the up string: register-held real coefficients,
//               one shared-memory load per hop; the default where the sector has the table).
//   hv_cols     pass 2: CTA = (output row, 256-column chunk, two columns per thread), chunk-major so that
//               the 256-column slab of x stays resident in L2 while all rows read it; adds the
//               up part: y[r, c] += sum_j coef_j * s_j(c) * x[src_j, c].
// Reference: src/hubbard_hamiltonian.cpp:51-108 (apply_extended_hubbard).
#include <algorithm>

#include "device.cuh"
#include "hv.cuh"

namespace ftlm_b200 {

namespace {

__global__ void __launch_bounds__(256) hv_generic_kernel(DevSector S, const double2* __restrict__ x,
                                                         double2* __restrict__ y) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < S.dim; idx += stride)
    y[idx] = hv_element(S, x, idx);
}

constexpr int kRowThreads = 1024;

// Warm L2 with a row another pass of this CTA reads next (bulk prefetch, no completion to wait on).
__device__ __forceinline__ void prefetch_row_l2(const double2* row, int64_t n) {
  const char* p = reinterpret_cast<const char*>(row);
  const uint32_t bytes = static_cast<uint32_t>(n * static_cast<int64_t>(sizeof(double2)));
  for (uint32_t off = 0; off < bytes; off += 32768u) {
    const uint32_t sz = min(32768u, bytes - off);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p + off), "r"(sz) : "memory");
  }
}

__device__ __forceinline__ double flip_sign(double v, uint32_t neg) {
  return __hiloint2double(__double2hiint(v) ^ static_cast<int>(neg << 31), __double2loint(v));
}

__global__ void __launch_bounds__(kRowThreads, 1) hv_rows_kernel(DevSector S, const double2* __restrict__ x,
                                                                   double2* __restrict__ y, double sx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Dd = static_cast<int>(S.Dd);
  double2* xs = reinterpret_cast<double2*>(smem_raw);
  double2* coef = xs + Dd;
  const int tid = threadIdx.x;
  for (int64_t r = blockIdx.x; r < S.Du; r += gridDim.x) {
    if (tid == 0 && r + gridDim.x < S.Du) prefetch_row_l2(x + (r + gridDim.x) * S.Dd, S.Dd);
    const uint32_t u = S.umask[r];
    const int cuu = S.cnt_uu[r];
    const uint4 w = S.wpl[r];
    const double2* xrow = x + r * S.Dd;
    int saw_tiny = 0;
    for (int c = tid; c < Dd; c += kRowThreads) {
      double2 v = xrow[c];
      v.x *= sx;  // the input is sx * x (sx = 1: unchanged)
      v.y *= sx;
      if (tiny(v)) {
        saw_tiny |= (v.x != 0.0 || v.y != 0.0);
        v = make_double2(0.0, 0.0);
      }
      xs[c] = v;
    }
    // Per-row down-hop coefficients (c_h times the up-string JW factor), 8 copies so that the
    // 8 lanes of a quarter-warp (lane % 8 = copy) never share a bank group.
    for (int i = tid; i < (S.n_dn_hops + 1) * 8; i += kRowThreads) {
      const int h = i >> 3;
      double2 cf = S.dn_coef[h];
      if (__popc(u & S.dn_nmask[h]) & 1) {
        cf.x = -cf.x;
        cf.y = -cf.y;
      }
      coef[i] = cf;
    }
    if (saw_tiny) atomicOr(S.flags, 1);
    __syncthreads();
    double2* yrow = y + r * S.Dd;
    for (int c = tid; c < Dd; c += kRowThreads) {
      const double2 xv = xs[c];
      const double dg = diag_value(S, u, S.dmask[c], cuu, S.cnt_dd[c], w);
      double2 acc = make_double2(dg * xv.x, dg * xv.y);
      const int g = c >> 5;
      const int64_t e_end = S.dn_gptr[g + 1];
#pragma unroll 4
      for (int64_t p = S.dn_gptr[g] + (c & 31); p < e_end; p += 32) {
        const uint32_t ent = __ldg(S.dn_ent + p);
        cmac(acc, coef[((ent >> 1) & 511u) * 8 + (c & 7)], xs[ent >> 10], ent & 1u);
      }
      yrow[c] = acc;
    }
    __syncthreads();
  }
}

using RowsKernel = void (*)(DevSector, const double2*, double2*, double);

// Column pass: two columns per thread, chunk = 2 * threads columns (variants: 64 / 128 / 256
// threads = 128 / 256 / 512-column slabs of Du * chunk * 16 bytes kept in L2; the autotuner picks).
constexpr int kMaxUpDeg = 128;

// acc += (-1)^neg c v, the sign applied to c's sign bits.
__device__ __forceinline__ void cmac_xor(double2& acc, double2 c, double2 v, uint32_t neg) {
  const int flip = static_cast<int>(neg << 31);
  c.x = __hiloint2double(__double2hiint(c.x) ^ flip, __double2loint(c.x));
  c.y = __hiloint2double(__double2hiint(c.y) ^ flip, __double2loint(c.y));
  acc.x = fma(c.x, v.x, acc.x);
  acc.x = fma(-c.y, v.y, acc.x);
  acc.y = fma(c.x, v.y, acc.y);
  acc.y = fma(c.y, v.x, acc.y);
}

// One real-section entry of a gauge table: the coefficient is one of two register-held values with
// the entry's sign (cls<<30 | s<<31), or, in the XOR form (kXor), real2[0] with the high word's bits
// 18..31 flipped by the entry's own bits 18..31 (one XOR: the builder checked that this gives exactly
// (-1)^s real2[cls]).
template <bool kXor>
__device__ __forceinline__ void gauge_real(double2& acc, uint32_t e, const unsigned char* line, double a0, double a1) {
  const double2 v = *reinterpret_cast<const double2*>(line + (e & 0x3FFF0u));
  const double cf = kXor ? __hiloint2double(__double2hiint(a0) ^ static_cast<int>(e & 0xFFFC0000u), __double2loint(a0))
                         : flip_sign((e & 0x40000000u) ? a1 : a0, e >> 31);
  acc.x = fma(cf, v.x, acc.x);
  acc.y = fma(cf, v.y, acc.y);
}

// One table-section entry: the coefficient from the 8-copy table (copy i % 8: the 8 lanes of a
// quarter-warp hit 8 bank groups), or, in the phase form (kPhase), real2[cls] times the unit phase
// (pc, +-ps): the product equals the table value bit for bit (checked when the table is built), so
// both forms give identical sums, and the phase form spends no shared-memory load on the coefficient.
template <bool kPhase>
__device__ __forceinline__ void gauge_cplx(double2& acc, uint32_t e, int i, const unsigned char* line,
                                           const double2* tab, double a0, double a1, double pc, double ps) {
  const double2 v = *reinterpret_cast<const double2*>(line + (e & 0x3FFF0u));
  if (kPhase) {
    const double cf = flip_sign((e & 0x40000000u) ? a1 : a0, e >> 31);
    const double cr = cf * pc;
    const double ci = flip_sign(cf * ps, (e >> 27) & 1u);
    acc.x = fma(cr, v.x, acc.x);
    acc.x = fma(-ci, v.y, acc.x);
    acc.y = fma(cr, v.y, acc.y);
    acc.y = fma(ci, v.x, acc.y);
  } else {
    cmac_xor(acc, tab[((e >> 18) & 511u) * 8 + (i & 7)], v, e >> 31);
  }
}

// acc += sum over the gauge-table entries of output string i (one warp = 32 consecutive strings, so
// the round counts are warp-uniform).  Both sections are whole 4-entry loads, so each runs as its own
// loop with no per-entry test; the last load of a section holds kr % 4 (kt % 4) rounds before its
// padding, and only those are gathered.  Entry loads run two ahead of use (the table ends with two
// padding loads, so the look-ahead needs no bound check).
template <bool kPhase, bool kXor>
__device__ __forceinline__ void gauge_hops(double2& acc, const DevGauge& G, int i, const unsigned char* line,
                                           const double2* tab, double a0, double a1) {
  const int4 gp = G.grp[i >> 5];
  const int kr = gp.w & 0xFFFF, kt = gp.w >> 16;  // rounds before the padding to whole loads
  const double pc = G.pc, ps = G.ps;
  const uint4* ep = reinterpret_cast<const uint4*>(G.ent + gp.x) + (i & 31);
  uint4 cur = __ldg(ep);
  uint4 nxt = __ldg(ep + 32);
  int q = 0;
  auto next = [&]() {
    const uint4 e = cur;
    cur = nxt;
    nxt = __ldg(ep + (q + 2) * 32);
    ++q;
    return e;
  };
  for (int n = kr >> 2; n > 0; --n) {
    const uint4 e = next();
    gauge_real<kXor>(acc, e.x, line, a0, a1);
    gauge_real<kXor>(acc, e.y, line, a0, a1);
    gauge_real<kXor>(acc, e.z, line, a0, a1);
    gauge_real<kXor>(acc, e.w, line, a0, a1);
  }
  if (kr & 3) {
    const uint4 e = next();
    gauge_real<kXor>(acc, e.x, line, a0, a1);
    if ((kr & 3) > 1) gauge_real<kXor>(acc, e.y, line, a0, a1);
    if ((kr & 3) > 2) gauge_real<kXor>(acc, e.z, line, a0, a1);
  }
  for (int n = kt >> 2; n > 0; --n) {
    const uint4 e = next();
    gauge_cplx<kPhase>(acc, e.x, i, line, tab, a0, a1, pc, ps);
    gauge_cplx<kPhase>(acc, e.y, i, line, tab, a0, a1, pc, ps);
    gauge_cplx<kPhase>(acc, e.z, i, line, tab, a0, a1, pc, ps);
    gauge_cplx<kPhase>(acc, e.w, i, line, tab, a0, a1, pc, ps);
  }
  if (kt & 3) {
    const uint4 e = next();
    gauge_cplx<kPhase>(acc, e.x, i, line, tab, a0, a1, pc, ps);
    if ((kt & 3) > 1) gauge_cplx<kPhase>(acc, e.y, i, line, tab, a0, a1, pc, ps);
    if ((kt & 3) > 2) gauge_cplx<kPhase>(acc, e.z, i, line, tab, a0, a1, pc, ps);
  }
}

// Row pass in the spin-ordered basis.  With g(u, d) = (-1)^popc(u & prefix_parity_shifted(d)), the
// down-hop part of row u is  y[u, d] = g(u, d) sum_h (-1)^s_h c_h g(u, d_h) x[u, d_h]  with s_h the
// down-string sign alone, so the row is staged as xs[d] = g(u, d) x[u, d] and every coefficient is
// the same for all rows: real ones come from two registers (an entry bit picks one), the others from
// a small table copied once per CTA (8 copies, one per bank group).  Each hop then costs one 16-byte
// shared load of x (plus one for table hops outside the phase form) instead of two.  Entries:
// GaugeTable (plan.hpp).
template <bool kPhase, bool kXor>
__global__ void __launch_bounds__(kRowThreads, 1) hv_rows_gauge_kernel(DevSector S, const double2* __restrict__ x,
                                                                         double2* __restrict__ y, double sx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Dd = static_cast<int>(S.Dd);
  double2* xs = reinterpret_cast<double2*>(smem_raw);
  double2* tab = xs + Dd + 8;
  const int tid = threadIdx.x;
  const DevGauge G = S.dn_g;
  if (!kPhase)
    for (int i = tid; i < G.nt * 8; i += kRowThreads) tab[i] = G.tab[i >> 3];
  if (tid < 8) xs[Dd + tid] = make_double2(0.0, 0.0);  // zero sentinels for padding entries
  const double a0 = G.real2[0], a1 = G.real2[1];
  for (int64_t r = blockIdx.x; r < S.Du; r += gridDim.x) {
    if (tid == 0 && r + gridDim.x < S.Du) prefetch_row_l2(x + (r + gridDim.x) * S.Dd, S.Dd);
    const uint32_t u = S.umask[r];
    const int cuu = S.cnt_uu[r];
    const uint4 w = S.wpl[r];
    const double2* xrow = x + r * S.Dd;
    int saw_tiny = 0;
    for (int c = tid; c < Dd; c += kRowThreads) {
      double2 v = xrow[c];
      v.x *= sx;  // the input is sx * x (sx = 1: unchanged)
      v.y *= sx;
      if (tiny(v)) {
        saw_tiny |= (v.x != 0.0 || v.y != 0.0);
        v = make_double2(0.0, 0.0);
      }
      if (gauge_sign(u, S.dmask[c])) v = make_double2(-v.x, -v.y);
      xs[c] = v;
    }
    if (saw_tiny) atomicOr(S.flags, 1);
    __syncthreads();
    double2* yrow = y + r * S.Dd;
    for (int c = tid; c < Dd; c += kRowThreads) {
      const int d = gauge_string(G, c);  // table position c serves output string d
      const uint32_t dm = S.dmask[d];
      const double2 xv = xs[d];
      const double dg = diag_value(S, u, dm, cuu, S.cnt_dd[d], w);
      double2 acc = make_double2(dg * xv.x, dg * xv.y);
      gauge_hops<kPhase, kXor>(acc, G, c, smem_raw, tab, a0, a1);
      if (gauge_sign(u, dm)) acc = make_double2(-acc.x, -acc.y);
      yrow[d] = acc;
    }
    __syncthreads();
  }
}

// kFused: the input is sx * x; the up-hop sum is formed on its own and added as
// y = y_rows + sx * sum, and the thread's share of <sx x, y> over its columns goes to dot
// (the Lanczos step's alpha without a separate pass: x[r, c] is in the L2-resident slab).
template <int kColThreads, bool kFilter, bool kFused>
__device__ __forceinline__ void cols_body(const DevSector& S, const double2* __restrict__ x, double2* __restrict__ y,
                                          int64_t r, int64_t c0, int deg, const int64_t* s_off, const double2* s_coef,
                                          const uint32_t* s_lh, double sx, double (&dot)[2]) {
  const int64_t c1 = c0 + kColThreads;
  const bool has1 = c1 < S.Dd;
  const int64_t c1s = has1 ? c1 : c0;  // in-bounds column for the second lane slot
  const uint32_t q0 = prefix_parity_shifted(S.dmask[c0]);
  const uint32_t q1 = prefix_parity_shifted(S.dmask[c1s]);
  double2* y0 = y + r * S.Dd + c0;
  double2 acc0 = kFused ? make_double2(0.0, 0.0) : *y0;
  double2 acc1 = (has1 && !kFused) ? y[r * S.Dd + c1] : make_double2(0.0, 0.0);
  const double2* x0 = x + c0;
  const double2* x1 = x + c1s;
  auto skip = [sx](double2 v) { return kFused ? tiny(make_double2(sx * v.x, sx * v.y)) : tiny(v); };
  int j = 0;
  for (; j + 4 <= deg; j += 4) {
    double2 v0[4], v1[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int64_t off = s_off[j + t];
      v0[t] = x0[off];
      v1[t] = x1[off];
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const uint32_t lh = s_lh[j + t];
      const uint32_t lo = lh & 255u, hi = lh >> 8;
      const double2 cf = s_coef[j + t];
      if (!kFilter || !skip(v0[t])) cmac_xor(acc0, cf, v0[t], ((q0 >> lo) ^ (q0 >> hi)) & 1u);
      if (!kFilter || !skip(v1[t])) cmac_xor(acc1, cf, v1[t], ((q1 >> lo) ^ (q1 >> hi)) & 1u);
    }
  }
  for (; j < deg; ++j) {
    const int64_t off = s_off[j];
    const double2 v0 = x0[off], v1 = x1[off];
    const uint32_t lh = s_lh[j];
    const uint32_t lo = lh & 255u, hi = lh >> 8;
    const double2 cf = s_coef[j];
    if (!kFilter || !skip(v0)) cmac_xor(acc0, cf, v0, ((q0 >> lo) ^ (q0 >> hi)) & 1u);
    if (!kFilter || !skip(v1)) cmac_xor(acc1, cf, v1, ((q1 >> lo) ^ (q1 >> hi)) & 1u);
  }
  if constexpr (kFused) {
    const double2 r0 = *y0;
    acc0 = make_double2(fma(sx, acc0.x, r0.x), fma(sx, acc0.y, r0.y));
    const double2 xq0 = x[r * S.Dd + c0];
    const double qx = sx * xq0.x, qy = sx * xq0.y;  // conj(q) * y
    dot[0] += qx * acc0.x + qy * acc0.y;
    dot[1] += qx * acc0.y - qy * acc0.x;
    if (has1) {
      const double2 r1 = y[r * S.Dd + c1];
      acc1 = make_double2(fma(sx, acc1.x, r1.x), fma(sx, acc1.y, r1.y));
      const double2 xq1 = x[r * S.Dd + c1];
      const double px = sx * xq1.x, py = sx * xq1.y;
      dot[0] += px * acc1.x + py * acc1.y;
      dot[1] += px * acc1.y - py * acc1.x;
    }
  }
  *y0 = acc0;
  if (has1) y[r * S.Dd + c1] = acc1;
}

// The column pass over the packed up list (SectorPlan::up_pk): one 4-byte word per source, read
// four at a time from shared memory, gives the source row, the (lo, hi) of the column-dependent sign
// and the coefficient (-1)^s real2[cls] (times (pc, +-ps) for a phase hop).  A real coefficient costs
// two FMAs per column instead of a complex multiply, and the list costs a quarter of a shared load per
// source instead of three.  The kind of each source is the same for every thread of the block, so
// the phase test does not diverge.  Same products and sums as cols_body on the CSR list.
template <int kColThreads, bool kFilter, bool kFused>
__device__ __forceinline__ void cols_body_packed(const DevSector& S, const double2* __restrict__ x,
                                                 double2* __restrict__ y, int64_t r, int64_t c0, int deg,
                                                 const uint32_t* s_pk, double sx, double (&dot)[2]) {
  const int64_t c1 = c0 + kColThreads;
  const bool has1 = c1 < S.Dd;
  const int64_t c1s = has1 ? c1 : c0;
  const uint32_t q0 = prefix_parity_shifted(S.dmask[c0]);
  const uint32_t q1 = prefix_parity_shifted(S.dmask[c1s]);
  double2* y0 = y + r * S.Dd + c0;
  double2 acc0 = kFused ? make_double2(0.0, 0.0) : *y0;
  double2 acc1 = (has1 && !kFused) ? y[r * S.Dd + c1] : make_double2(0.0, 0.0);
  const double2* x0 = x + c0;
  const double2* x1 = x + c1s;
  const int64_t Dd = S.Dd;
  const double a0 = S.up_real2[0], a1 = S.up_real2[1], pc = S.up_pc, ps = S.up_ps;
  auto skip = [sx](double2 v) { return kFused ? tiny(make_double2(sx * v.x, sx * v.y)) : tiny(v); };
  auto term = [&](uint32_t pk, double2 v0, double2 v1) {
    const uint32_t lo = (pk >> 14) & 31u, hi = (pk >> 19) & 31u;
    const double cf = flip_sign((pk & 0x40000000u) ? a1 : a0, pk >> 31);
    const uint32_t f0 = ((q0 >> lo) ^ (q0 >> hi)) & 1u, f1 = ((q1 >> lo) ^ (q1 >> hi)) & 1u;
    if (pk & 0x20000000u) {  // phase hop: cf * (pc, +-ps), the column sign on both parts
      const double cr = cf * pc;
      const double ci = flip_sign(cf * ps, (pk >> 28) & 1u);
      const double2 c = make_double2(cr, ci);
      if (!kFilter || !skip(v0)) cmac_xor(acc0, c, v0, f0);
      if (!kFilter || !skip(v1)) cmac_xor(acc1, c, v1, f1);
    } else {
      if (!kFilter || !skip(v0)) {
        const double c = flip_sign(cf, f0);
        acc0.x = fma(c, v0.x, acc0.x);
        acc0.y = fma(c, v0.y, acc0.y);
      }
      if (!kFilter || !skip(v1)) {
        const double c = flip_sign(cf, f1);
        acc1.x = fma(c, v1.x, acc1.x);
        acc1.y = fma(c, v1.y, acc1.y);
      }
    }
  };
  int j = 0;
  for (; j + 4 <= deg; j += 4) {
    const uint4 pk = *reinterpret_cast<const uint4*>(s_pk + j);
    const uint32_t p[4] = {pk.x, pk.y, pk.z, pk.w};
    double2 v0[4], v1[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int64_t off = static_cast<int64_t>(p[t] & 0x3FFFu) * Dd;
      v0[t] = x0[off];
      v1[t] = x1[off];
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) term(p[t], v0[t], v1[t]);
  }
  for (; j < deg; ++j) {
    const uint32_t pk = s_pk[j];
    const int64_t off = static_cast<int64_t>(pk & 0x3FFFu) * Dd;
    term(pk, x0[off], x1[off]);
  }
  if constexpr (kFused) {
    const double2 r0 = *y0;
    acc0 = make_double2(fma(sx, acc0.x, r0.x), fma(sx, acc0.y, r0.y));
    const double2 xq0 = x[r * S.Dd + c0];
    const double qx = sx * xq0.x, qy = sx * xq0.y;  // conj(q) * y
    dot[0] += qx * acc0.x + qy * acc0.y;
    dot[1] += qx * acc0.y - qy * acc0.x;
    if (has1) {
      const double2 r1 = y[r * S.Dd + c1];
      acc1 = make_double2(fma(sx, acc1.x, r1.x), fma(sx, acc1.y, r1.y));
      const double2 xq1 = x[r * S.Dd + c1];
      const double px = sx * xq1.x, py = sx * xq1.y;
      dot[0] += px * acc1.x + py * acc1.y;
      dot[1] += px * acc1.y - py * acc1.x;
    }
  }
  *y0 = acc0;
  if (has1) y[r * S.Dd + c1] = acc1;
}

// At least 896 resident threads per SM (28 warps): the L2 gathers need the bytes in flight, and the
// fused form would otherwise take a few registers more and drop to 24 warps.
template <int kColThreads, bool kFused, bool kPacked>
__global__ void __launch_bounds__(kColThreads, 896 / kColThreads) hv_cols_kernel(DevSector S, const double2* __restrict__ x,
                                                              double2* __restrict__ y, double sx,
                                                              double* __restrict__ dotp) {
  constexpr int kColChunk = 2 * kColThreads;
  constexpr int kListDeg = kPacked ? 4 : kMaxUpDeg;  // the list arrays of the form this launch does not use
  __shared__ int64_t s_off[kListDeg];
  __shared__ double2 s_coef[kListDeg];
  __shared__ uint32_t s_lh[kListDeg];
  __shared__ __align__(16) uint32_t s_pk[kPacked ? kMaxUpDeg : 4];
  const int64_t b = blockIdx.x;
  const int64_t chunk = b / S.Du;
  const int64_t r = b - chunk * S.Du;
  const int j0 = S.up_ptr[r];
  const int deg = S.up_ptr[r + 1] - j0;
  for (int j = threadIdx.x; j < deg; j += kColThreads) {
    if constexpr (kPacked) {
      s_pk[j] = S.up_pk[j0 + j];
    } else {
      s_off[j] = static_cast<int64_t>(S.up_src[j0 + j]) * S.Dd;
      s_coef[j] = S.up_coef[j0 + j];
      s_lh[j] = S.up_lohi[j0 + j];
    }
  }
  const bool filt = (*S.flags) != 0;
  __syncthreads();
  const int64_t c0 = chunk * kColChunk + threadIdx.x;
  double dot[2] = {0.0, 0.0};
  if (c0 < S.Dd) {
    if constexpr (kPacked) {
      if (filt)
        cols_body_packed<kColThreads, true, kFused>(S, x, y, r, c0, deg, s_pk, sx, dot);
      else
        cols_body_packed<kColThreads, false, kFused>(S, x, y, r, c0, deg, s_pk, sx, dot);
    } else {
      if (filt)
        cols_body<kColThreads, true, kFused>(S, x, y, r, c0, deg, s_off, s_coef, s_lh, sx, dot);
      else
        cols_body<kColThreads, false, kFused>(S, x, y, r, c0, deg, s_off, s_coef, s_lh, sx, dot);
    }
  }
  if constexpr (kFused) {  // fixed tree over the block (warp shuffles, then warps in order): one partial
    constexpr int kWarps = kColThreads / 32;
    __shared__ double red[2][kWarps];
#pragma unroll
    for (int h = 16; h > 0; h >>= 1) {
      dot[0] += __shfl_down_sync(0xFFFFFFFFu, dot[0], h);
      dot[1] += __shfl_down_sync(0xFFFFFFFFu, dot[1], h);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
      red[0][warp] = dot[0];
      red[1][warp] = dot[1];
    }
    __syncthreads();
    if (threadIdx.x == 0 && dotp) {
      double s0 = red[0][0], s1 = red[1][0];
#pragma unroll
      for (int w = 1; w < kWarps; ++w) {
        s0 += red[0][w];
        s1 += red[1][w];
      }
      dotp[2 * b] = s0;
      dotp[2 * b + 1] = s1;
    }
  }
}

int g_num_sms = 0;

}  // namespace

size_t hv_rows_smem_bytes(const DevSector& S) {
  if (S.dn_g.ent) return static_cast<size_t>(S.Dd + 8 + (S.dn_g.phase ? 0 : 8 * S.dn_g.nt)) * sizeof(double2);
  return static_cast<size_t>(S.Dd) * sizeof(double2) + static_cast<size_t>(S.n_dn_hops + 1) * 8 * sizeof(double2);
}

bool hv_fast_path_ok(const DevSector& S, int max_up_deg) {
  return hv_rows_smem_bytes(S) <= 227 * 1024 && max_up_deg <= kMaxUpDeg && S.dim >= (1 << 16) && S.Dd >= 64;
}

void init_sm_count() {
  if (g_num_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
}

template <int kThreads>
cudaError_t launch_cols(const DevSector& S, const double2* x, double2* y, cudaStream_t st, double sx, double* dotp) {
  const int64_t nchunks = (S.Dd + 2 * kThreads - 1) / (2 * kThreads);
  const unsigned grid = static_cast<unsigned>(nchunks * S.Du);
  const bool fused = dotp || sx != 1.0;
  if (S.up_pk) {
    if (fused)
      hv_cols_kernel<kThreads, true, true><<<grid, kThreads, 0, st>>>(S, x, y, sx, dotp);
    else
      hv_cols_kernel<kThreads, false, true><<<grid, kThreads, 0, st>>>(S, x, y, sx, dotp);
  } else {
    if (fused)
      hv_cols_kernel<kThreads, true, false><<<grid, kThreads, 0, st>>>(S, x, y, sx, dotp);
    else
      hv_cols_kernel<kThreads, false, false><<<grid, kThreads, 0, st>>>(S, x, y, sx, dotp);
  }
  return cudaGetLastError();
}

int64_t hv_cols_blocks(const DevSector& S, int cols_variant) {
  cols_variant %= 3;  // 3..5: the same slabs over the packed list
  const int threads = cols_variant == 1 ? 64 : (cols_variant == 2 ? 256 : 128);
  return (S.Dd + 2 * threads - 1) / (2 * threads) * S.Du;
}

cudaError_t hv_launch_pass(const DevSector& S, const double2* x, double2* y, int pass, cudaStream_t st,
                           int cols_variant, double sx, double* dotp) {
  if (S.dim <= 0) return cudaSuccess;
  init_sm_count();
  if (pass == 0) {
    cudaError_t e = cudaMemsetAsync(S.flags, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    const size_t sm = hv_rows_smem_bytes(S);
    const RowsKernel k = !S.dn_g.ent ? hv_rows_kernel
                         : S.dn_g.phase ? (S.dn_g.xor_real ? hv_rows_gauge_kernel<true, true> : hv_rows_gauge_kernel<true, false>)
                                        : (S.dn_g.xor_real ? hv_rows_gauge_kernel<false, true> : hv_rows_gauge_kernel<false, false>);
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm));
    if (e != cudaSuccess) return e;
    const int grid_r = static_cast<int>(std::min<int64_t>(S.Du, g_num_sms));
    k<<<grid_r, kRowThreads, sm, st>>>(S, x, y, sx);
    return cudaGetLastError();
  }
  cols_variant %= 3;  // 3..5: the same slabs; the list form comes with S (S.up_pk)
  if (cols_variant == 1) return launch_cols<64>(S, x, y, st, sx, dotp);
  if (cols_variant == 2) return launch_cols<256>(S, x, y, st, sx, dotp);
  return launch_cols<128>(S, x, y, st, sx, dotp);
}

cudaError_t hv_launch(const DevSector& S, const double2* x, double2* y, int path, cudaStream_t st, int cols_variant) {
  if (S.dim <= 0) return cudaSuccess;
  init_sm_count();
  if (path == 2) {
    cudaError_t e = hv_launch_pass(S, x, y, 0, st, cols_variant);
    if (e != cudaSuccess) return e;
    return hv_launch_pass(S, x, y, 1, st, cols_variant);
  }
  const int64_t blocks = std::min<int64_t>((S.dim + 255) / 256, static_cast<int64_t>(g_num_sms) * 16);
  hv_generic_kernel<<<static_cast<unsigned>(blocks), 256, 0, st>>>(S, x, y);
  return cudaGetLastError();
}

}  // namespace ftlm_b200
