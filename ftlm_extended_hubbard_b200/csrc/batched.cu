// Batched FTLM (complex64 vectors, FP64 scalars): the 32 Lanczos chains of one sector advance
// together.  Block vectors are V[state][chain] (32 complex64 = 256 bytes per basis state), one
// warp per basis state and lane = chain, so every gather is one coalesced 256-byte segment and the
// index / JW-sign work of a hop is shared by the 32 chains.  Same hop tables as the complex128
// path (plan.hpp), same recurrence as src/lanczos.cpp:180-205, with these changes of form:
//
//   * vectors are kept unnormalised: W_k = beta_{k-1} q_k (W_0 = raw start, beta_{-1} = ||raw||),
//     and the 1/beta_{k-1} factor is applied in FP64 after the H·v, never rounded to FP32:
//       Y = H W_k                              (FP32, unscaled)
//       z = <q_k, H q_k> = <W_k, Y> / beta_{k-1}^2,  alpha_k = Re z
//       W_{k+1} = Y / beta_{k-1} - (z / beta_{k-1}) W_k - (beta_{k-1} / beta_{k-2}) W_{k-1},  beta_k = ||W_{k+1}||
//     so no normalisation pass exists, and no per-step FP32 rounding of the scale enters alpha;
//   * alpha/beta stay on the device; a chain whose ||w||^2 < 1e-24 stops (reference breakdown
//     rule) and its later scale factors are 0;
//   * H·v in FP32 (FMA), dot products and norms accumulated in FP64 with Neumaier compensation,
//     the vector update evaluated in FP64 and rounded to complex64;
//   * every kernel is persistent with a fixed grid (kBtBlocks) and fixed per-block work order, so
//     the FP64 reductions are bitwise repeatable.
#include <algorithm>
#include <cstdio>

#include "batched.cuh"
#include "device.cuh"
#include "orbit.cuh"

namespace ftlm_b200 {

namespace {

constexpr int kBtThreads = 256;  // 8 warps = 8 basis states per work item
constexpr int kBtWarps = kBtThreads / 32;
constexpr int kMaxUpDegB = 128;

struct Neu {  // Neumaier-compensated FP64 sum
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double v) {
    const double t = s + v;
    c += (fabs(s) >= fabs(v)) ? ((s - t) + v) : ((v - t) + s);
    s = t;
  }
  __device__ __forceinline__ double value() const { return s + c; }
};

// |v|^2 < 1e-28 in FP32 (squares below FLT_MIN flush towards zero, which is still below the bound).
__device__ __forceinline__ bool tinyf(float2 v) { return fmaf(v.x, v.x, v.y * v.y) < 1e-28f; }

__device__ __forceinline__ void cmacf(float2& acc, float cr, float ci, float2 v, uint32_t neg) {
  if (neg) {
    cr = -cr;
    ci = -ci;
  }
  acc.x = fmaf(cr, v.x, acc.x);
  acc.x = fmaf(-ci, v.y, acc.x);
  acc.y = fmaf(cr, v.y, acc.y);
  acc.y = fmaf(ci, v.x, acc.y);
}

// Block-wide per-lane sum of NV doubles over the 8 warps; result valid in warp 0.
template <int NV>
__device__ __forceinline__ void lane_block_sum(double (&v)[NV], double* sh /* NV*kBtThreads */) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < NV; ++i) sh[i * kBtThreads + t] = v[i];
  __syncthreads();
  if (t < 32) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double s = 0.0;
      for (int w = 0; w < kBtWarps; ++w) s += sh[i * kBtThreads + w * 32 + t];
      v[i] = s;
    }
  }
  __syncthreads();
}

// Start vectors: chain r uses Philox4x32-10 with key seed + r*100003 and counter = state index,
// the same stream as the complex128 path's FTLM_START_PHILOX, rounded to complex64.
__device__ __forceinline__ uint4 philox(uint4 c, uint2 k) {
  constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += W0;
    k.y += W1;
  }
  return c;
}

__global__ void __launch_bounds__(kBtThreads) bt_start_kernel(float2* __restrict__ W, int64_t dim, unsigned seed,
                                                              double* __restrict__ partial, int* __restrict__ flag,
                                                              const uint32_t* __restrict__ umask,
                                                              const uint32_t* __restrict__ dmask, int64_t Dd) {
  __shared__ double sh[kBtThreads];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned key = seed + static_cast<unsigned>(lane) * 100003u;
  Neu acc;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * kBtWarps + warp; i < dim; i += static_cast<int64_t>(gridDim.x) * kBtWarps) {
    const uint4 r = philox(make_uint4(static_cast<uint32_t>(i), static_cast<uint32_t>(i >> 32), 0u, 0u),
                           make_uint2(key, 0x7F4A7C15u));
    const uint64_t a = (static_cast<uint64_t>(r.x) << 21) ^ (r.y >> 11);
    const uint64_t b = (static_cast<uint64_t>(r.z) << 21) ^ (r.w >> 11);
    const double u1 = (static_cast<double>(a & ((1ull << 53) - 1)) + 0.5) * 0x1.0p-53;
    const double u2 = (static_cast<double>(b & ((1ull << 53) - 1)) + 0.5) * 0x1.0p-53;
    const double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    float2 z = make_float2(static_cast<float>(rad * c), static_cast<float>(rad * s));
    if (umask) {  // the start vector expressed in the gauge basis: W = G r
      const int64_t r = i / Dd;
      if (gauge_sign(umask[r], dmask[i - r * Dd])) z = make_float2(-z.x, -z.y);
    }
    if (tinyf(z) && (z.x != 0.f || z.y != 0.f)) *flag = 1;
    W[i * 32 + lane] = z;
    acc.add(static_cast<double>(z.x) * z.x + static_cast<double>(z.y) * z.y);
  }
  double v[1] = {acc.value()};
  lane_block_sum<1>(v, sh);
  if (threadIdx.x < 32) partial[blockIdx.x * 32 + lane] = v[0];
}

constexpr int kBtUnroll = 4;  // hop pairs per batch: 8 independent 256-byte gathers per warp

__device__ __forceinline__ float2 filt(float2 v) { return tinyf(v) ? make_float2(0.f, 0.f) : v; }
__device__ __forceinline__ float4 filt4(float4 v) {
  const float2 a = filt(make_float2(v.x, v.y)), b = filt(make_float2(v.z, v.w));
  return make_float4(a.x, a.y, b.x, b.y);
}

// acc (two chains) += (-1)^neg c v with the sign applied to c's sign bits.
__device__ __forceinline__ void cmac4(float4& acc, float2 c, float4 v, uint32_t neg) {
  const uint32_t f = neg << 31;
  c.x = __uint_as_float(__float_as_uint(c.x) ^ f);
  c.y = __uint_as_float(__float_as_uint(c.y) ^ f);
  acc.x = fmaf(c.x, v.x, acc.x);
  acc.x = fmaf(-c.y, v.y, acc.x);
  acc.y = fmaf(c.x, v.y, acc.y);
  acc.y = fmaf(c.y, v.x, acc.y);
  acc.z = fmaf(c.x, v.z, acc.z);
  acc.z = fmaf(-c.y, v.w, acc.z);
  acc.w = fmaf(c.x, v.w, acc.w);
  acc.w = fmaf(c.y, v.z, acc.w);
}

__device__ __forceinline__ float4 fold_halves(float4 a) {
  a.x += __shfl_down_sync(0xffffffffu, a.x, 16);
  a.y += __shfl_down_sync(0xffffffffu, a.y, 16);
  a.z += __shfl_down_sync(0xffffffffu, a.z, 16);
  a.w += __shfl_down_sync(0xffffffffu, a.w, 16);
  return a;
}

// Thread layout of both H·v passes: one warp per basis state; half-warp hv = lane >> 4 takes every
// other hop, and lane l = lane & 15 holds chains 2l and 2l+1 (one float4), so one warp instruction
// gathers two hops (2 x 256 bytes) and the per-hop index work is shared by 32 chains.

// The walks below keep (row, column) as 32-bit counters advanced by the warp stride, so no
// division runs per basis state; vector offsets are counted in float4 units (< 2^32 up to a
// 68 GB block vector).

// Row pass (gauge basis): Y[r, c, :] = diag * W + down hops.  Warp-persistent over basis states in
// row-major order (all warps of the grid walk the same row together, so the row of W — Dd * 256
// bytes — is served from L2).  In the gauge basis the down-hop coefficients do not depend on the
// up string: entry (2*hop + down-string sign) indexes one global signed table (dn_coef32s).
template <bool kFilter>
__device__ __forceinline__ void bt_rows_body(const DevSector& S, const float4* __restrict__ Wrow,
                                             float4* __restrict__ Yrow, uint32_t u, int cuu, uint4 wp, int c,
                                             int lane) {
  const int hv = lane >> 4;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (hv == 0) {
    float4 xv = Wrow[static_cast<uint32_t>(c) * 16u];
    if (kFilter) xv = filt4(xv);
    const float dg = static_cast<float>(diag_value(S, u, S.dmask[c], cuu, S.cnt_dd[c], wp));
    acc = make_float4(dg * xv.x, dg * xv.y, dg * xv.z, dg * xv.w);
  }
  // padded to a multiple of 8 entries: each half-warp takes 4 of every 8, no tail
  const int64_t p0 = S.dn_csr_ptr[c];
  const uint32_t* ent = S.dn_csr_ent + p0 + hv;
  const int K = static_cast<int>(S.dn_csr_ptr[c + 1] - p0);
  for (int k0 = 0; k0 < K; k0 += 8) {
    uint32_t e[4];
    float4 v[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) e[t] = ent[k0 + 2 * t];
#pragma unroll
    for (int t = 0; t < 4; ++t) v[t] = Wrow[(e[t] >> 9) << 4];
#pragma unroll
    for (int t = 0; t < 4; ++t) cmac4(acc, __ldg(S.dn_coef32s + (e[t] & 511u)), kFilter ? filt4(v[t]) : v[t], 0u);
  }
  acc = fold_halves(acc);
  if (hv == 0) Yrow[static_cast<uint32_t>(c) * 16u] = acc;
}

__global__ void __launch_bounds__(kBtThreads, kBtBlocksPerSm) bt_rows_kernel(DevSector S, const float2* __restrict__ W,
                                                                             float2* __restrict__ Y,
                                                                             const int* __restrict__ flag) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int l = lane & 15;
  const bool filter = *flag != 0;
  const int Dd = static_cast<int>(S.Dd), Du = static_cast<int>(S.Du);
  const int gw = blockIdx.x * kBtWarps + warp;
  const int nw = gridDim.x * kBtWarps;
  int r = gw / Dd, c = gw - (gw / Dd) * Dd;
  while (r < Du) {
    const uint32_t u = S.umask[r];
    const int cuu = S.cnt_uu[r];
    const uint4 wp = S.wpl[r];
    const float4* Wrow = reinterpret_cast<const float4*>(W) + static_cast<int64_t>(r) * Dd * 16 + l;
    float4* Yrow = reinterpret_cast<float4*>(Y) + static_cast<int64_t>(r) * Dd * 16 + l;
    if (filter)
      bt_rows_body<true>(S, Wrow, Yrow, u, cuu, wp, c, lane);
    else
      bt_rows_body<false>(S, Wrow, Yrow, u, cuu, wp, c, lane);
    c += nw;
    while (c >= Dd) {
      c -= Dd;
      ++r;
    }
  }
}

// Staged row pass (the default where the sector has the gauge-basis row table, plan.hpp GaugeTable):
// one work item = (up row r, chain pair p).  The row's slice of the two chains, W[r, :, 2p..2p+1]
// (16 bytes per basis state, 206 KB at 4x4 (8,8)), is staged in shared memory, and the down hops are
// gathered there with the complex128 row pass's table and schedule (the same 16-byte element size,
// so the same bank-group-free rounds): one 16-byte shared load serves two chains, instead of the
// 256-byte L2 gather of bt_rows_kernel for 32 chains.  Coefficients are the double-precision table
// values rounded to FP32 (what bt_rows_kernel's signed FP32 table holds); sums in FP32.
constexpr int kBtsThreads = 1024;

__device__ __forceinline__ double flip_d(double v, uint32_t neg) {
  return __hiloint2double(__double2hiint(v) ^ static_cast<int>(neg << 31), __double2loint(v));
}

template <bool kXor>
__device__ __forceinline__ void bts_real(float4& acc, uint32_t e, const unsigned char* line, double a0, double a1) {
  const float4 v = *reinterpret_cast<const float4*>(line + (e & 0x3FFF0u));
  const double cd = kXor ? __hiloint2double(__double2hiint(a0) ^ static_cast<int>(e & 0xFFFC0000u), __double2loint(a0))
                         : flip_d((e & 0x40000000u) ? a1 : a0, e >> 31);
  const float c = __double2float_rn(cd);
  acc.x = fmaf(c, v.x, acc.x);
  acc.y = fmaf(c, v.y, acc.y);
  acc.z = fmaf(c, v.z, acc.z);
  acc.w = fmaf(c, v.w, acc.w);
}

// Complex-section entry: the coefficient from the CTA's copy of the table in FP32 (8 copies, copy i % 8:
// the 8 lanes of a quarter-warp read 8 different bank groups), with the entry's sign.
__device__ __forceinline__ void bts_cplx(float4& acc, uint32_t e, int i, const unsigned char* line, const float2* tab) {
  const float4 v = *reinterpret_cast<const float4*>(line + (e & 0x3FFF0u));
  float2 c = tab[((e >> 18) & 511u) * 8 + (i & 7)];
  const uint32_t f = (e >> 31) << 31;
  c = make_float2(__uint_as_float(__float_as_uint(c.x) ^ f), __uint_as_float(__float_as_uint(c.y) ^ f));
  cmac4(acc, c, v, 0u);
}

// The gauge-table walk of hv.cu's row pass for output string i (sections as whole 4-entry loads, the
// padding rounds of each section's last load skipped, entry loads two ahead of use).
template <bool kXor>
__device__ __forceinline__ void bts_hops(float4& acc, const DevGauge& G, int i, const unsigned char* line,
                                         const float2* tab, double a0, double a1) {
  const int4 gp = G.grp[i >> 5];
  const int kr = gp.w & 0xFFFF, kt = gp.w >> 16;
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
    bts_real<kXor>(acc, e.x, line, a0, a1);
    bts_real<kXor>(acc, e.y, line, a0, a1);
    bts_real<kXor>(acc, e.z, line, a0, a1);
    bts_real<kXor>(acc, e.w, line, a0, a1);
  }
  if (kr & 3) {
    const uint4 e = next();
    bts_real<kXor>(acc, e.x, line, a0, a1);
    if ((kr & 3) > 1) bts_real<kXor>(acc, e.y, line, a0, a1);
    if ((kr & 3) > 2) bts_real<kXor>(acc, e.z, line, a0, a1);
  }
  for (int n = kt >> 2; n > 0; --n) {
    const uint4 e = next();
    bts_cplx(acc, e.x, i, line, tab);
    bts_cplx(acc, e.y, i, line, tab);
    bts_cplx(acc, e.z, i, line, tab);
    bts_cplx(acc, e.w, i, line, tab);
  }
  if (kt & 3) {
    const uint4 e = next();
    bts_cplx(acc, e.x, i, line, tab);
    if ((kt & 3) > 1) bts_cplx(acc, e.y, i, line, tab);
    if ((kt & 3) > 2) bts_cplx(acc, e.z, i, line, tab);
  }
}

template <bool kXor>
__global__ void __launch_bounds__(kBtsThreads, 1) bt_rows_staged_kernel(DevSector S, const float2* __restrict__ W,
                                                                         float2* __restrict__ Y,
                                                                         const int* __restrict__ flag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Dd = static_cast<int>(S.Dd);
  float4* xs = reinterpret_cast<float4*>(smem_raw);
  float2* tab = reinterpret_cast<float2*>(xs + Dd + 8);
  const int tid = threadIdx.x;
  const DevGauge G = S.dn_g;
  const bool filter = *flag != 0;
  for (int i = tid; i < G.nt * 8; i += kBtsThreads) {
    const double2 c = G.tab[i >> 3];
    tab[i] = make_float2(__double2float_rn(c.x), __double2float_rn(c.y));
  }
  if (tid < 8) xs[Dd + tid] = make_float4(0.f, 0.f, 0.f, 0.f);  // zero sentinels for padding entries
  const double a0 = G.real2[0], a1 = G.real2[1];
  const float4* W4 = reinterpret_cast<const float4*>(W);
  float4* Y4 = reinterpret_cast<float4*>(Y);
  const int64_t items = S.Du * (kBtChains / 2);
  for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const int64_t r = it / (kBtChains / 2);
    const int p = static_cast<int>(it - r * (kBtChains / 2));
    const uint32_t u = S.umask[r];
    const int cuu = S.cnt_uu[r];
    const uint4 wp = S.wpl[r];
    const int64_t base = r * S.Dd * (kBtChains / 2) + p;  // float4 index of state (r, 0), chains 2p, 2p+1
    for (int c = tid; c < Dd; c += kBtsThreads) {
      float4 v = W4[base + static_cast<int64_t>(c) * (kBtChains / 2)];
      if (filter) v = filt4(v);
      xs[c] = v;
    }
    __syncthreads();
    for (int c = tid; c < Dd; c += kBtsThreads) {
      const int d = gauge_string(G, c);  // table position c serves output string d
      const float4 xv = xs[d];
      const float dg = static_cast<float>(diag_value(S, u, S.dmask[d], cuu, S.cnt_dd[d], wp));
      float4 acc = make_float4(dg * xv.x, dg * xv.y, dg * xv.z, dg * xv.w);
      bts_hops<kXor>(acc, G, c, smem_raw, tab, a0, a1);
      Y4[base + static_cast<int64_t>(d) * (kBtChains / 2)] = acc;
    }
    __syncthreads();
  }
}

// Gathers of the orbit pass: two half-warps take every other source of the warp's list.
template <bool kFilter>
__device__ __forceinline__ float4 bt_cols_sum(const float4* Wc, const uint32_t* s_off, const float2* s_cf, int deg8,
                                              int hv) {
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int j0 = hv; j0 < deg8; j0 += 8) {
    float4 v[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) v[t] = Wc[s_off[j0 + 2 * t]];
#pragma unroll
    for (int t = 0; t < 4; ++t) cmac4(acc, s_cf[j0 + 2 * t], kFilter ? filt4(v[t]) : v[t], 0u);
  }
  return fold_halves(acc);
}

// Column pass (gauge basis): Y[r, c, :] += sum_j u_j W[src_j, c, :] with the coefficients u_j of
// output up string r the same for every column (the down string no longer enters the sign), then
// the fused <W_k, Y> per chain.  Work item = (kCols-column chunk, group of kRows output rows), walked
// chunk-major by a persistent grid so that the chunk's slab of W (Du x kCols x 256 bytes) stays in
// L2; in an item, thread (row t / (16 kCols), column t / 16 % kCols, lane t % 16) owns chains 2l,
// 2l+1 of one element and every source row is read as one contiguous kCols x 256-byte segment.
// kCols = 16 / 8 / 4 (slabs of 52.7 / 26.4 / 13.2 MB at 4x4 (8,8)) are the variants the batched
// autotuner chooses from.  Each block keeps its items' dot sums in registers and writes one partial
// per chain (fixed work order: bitwise repeatable for a given variant).
template <bool kFilter>
__device__ __forceinline__ float4 bg_cols_sum(const float4* __restrict__ Wc, const uint32_t* s_off,
                                              const float2* s_cf, int deg) {
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  int j = 0;
  for (; j + 4 <= deg; j += 4) {
    float4 v[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) v[t] = Wc[s_off[j + t]];
#pragma unroll
    for (int t = 0; t < 4; ++t) cmac4(acc, s_cf[j + t], kFilter ? filt4(v[t]) : v[t], 0u);
  }
  for (; j < deg; ++j) {
    const float4 v = Wc[s_off[j]];
    cmac4(acc, s_cf[j], kFilter ? filt4(v) : v, 0u);
  }
  return acc;
}

template <int kCols>
__global__ void __launch_bounds__(kBtThreads, kBtBlocksPerSm) bt_cols_kernel(DevSector S, const float2* __restrict__ W,
                                                                             float2* __restrict__ Y,
                                                                             double* __restrict__ partial,
                                                                             const int* __restrict__ flag) {
  constexpr int kRows = kBtThreads / (16 * kCols);
  __shared__ uint32_t s_off[kRows][kMaxUpDegB];
  __shared__ float2 s_cf[kRows][kMaxUpDegB];
  __shared__ double sh[4 * kBtThreads];
  const int t = threadIdx.x;
  const int ri = t / (16 * kCols), col = (t >> 4) % kCols, l = t & 15;
  const bool filter = *flag != 0;
  const int Dd = static_cast<int>(S.Dd), Du = static_cast<int>(S.Du);
  const uint32_t row_stride = static_cast<uint32_t>(Dd) * 16u;  // float4 units per row
  const float4* W4 = reinterpret_cast<const float4*>(W);
  float4* Y4 = reinterpret_cast<float4*>(Y);
  const int64_t nchunks = (Dd + kCols - 1) / kCols;
  const int64_t ngroups = (Du + kRows - 1) / kRows;
  const int64_t items = nchunks * ngroups;
  double d0r = 0.0, d0i = 0.0, d1r = 0.0, d1i = 0.0;  // chains 2l and 2l+1
  for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const int64_t chunk = it / ngroups;
    const int r0 = static_cast<int>(it - chunk * ngroups) * kRows;
    __syncthreads();  // the previous item's lists are no longer read
#pragma unroll
    for (int q = 0; q < kRows; ++q) {
      if (r0 + q >= Du) break;
      const int j0 = S.up_ptr[r0 + q];
      const int dq = S.up_ptr[r0 + q + 1] - j0;
      for (int j = t; j < dq; j += kBtThreads) {
        s_off[q][j] = static_cast<uint32_t>(S.up_src[j0 + j]) * row_stride;
        s_cf[q][j] = S.up_coef32[j0 + j];
      }
    }
    __syncthreads();
    const int r = r0 + ri;
    const int c = static_cast<int>(chunk) * kCols + col;
    if (r < Du && c < Dd) {
      const int deg = S.up_ptr[r + 1] - S.up_ptr[r];
      const float4* Wc = W4 + static_cast<uint32_t>(c) * 16u + l;
      const float4 acc = filter ? bg_cols_sum<true>(Wc, s_off[ri], s_cf[ri], deg)
                                : bg_cols_sum<false>(Wc, s_off[ri], s_cf[ri], deg);
      const int64_t o = static_cast<int64_t>(r) * row_stride + static_cast<uint32_t>(c) * 16u + l;
      float4 y = Y4[o];
      y.x += acc.x;
      y.y += acc.y;
      y.z += acc.z;
      y.w += acc.w;
      Y4[o] = y;
      const float4 w = W4[o];
      // conj(w) * y per chain
      const double wx = w.x, wy = w.y, wz = w.z, ww = w.w;
      const double yx = y.x, yy = y.y, yz = y.z, yw = y.w;
      d0r = fma(wx, yx, fma(wy, yy, d0r));
      d0i = fma(wx, yy, fma(-wy, yx, d0i));
      d1r = fma(wz, yz, fma(ww, yw, d1r));
      d1i = fma(wz, yw, fma(-ww, yz, d1i));
    }
  }
  // per-chain block sums: thread t holds chains 2l, 2l+1 of one element
  sh[0 * kBtThreads + t] = d0r;
  sh[1 * kBtThreads + t] = d0i;
  sh[2 * kBtThreads + t] = d1r;
  sh[3 * kBtThreads + t] = d1i;
  __syncthreads();
  if (t < 32) {
    const int ll = t & 15, which = t >> 4;  // thread t reduces chain 2*ll + which
    double re = 0.0, im = 0.0;
    for (int k = 0; k < kBtThreads / 16; ++k) {
      re += sh[(2 * which) * kBtThreads + k * 16 + ll];
      im += sh[(2 * which + 1) * kBtThreads + k * 16 + ll];
    }
    const int chain = 2 * ll + which;
    partial[(blockIdx.x * 32 + chain) * 2] = re;
    partial[(blockIdx.x * 32 + chain) * 2 + 1] = im;
  }
}

// Row pass of the batched H·V: the staged kernel where the sector has the gauge table and the
// staged slice fits shared memory, else bt_rows_kernel.
cudaError_t launch_bt_rows(const DevSector& S, const float2* W, float2* Y, const int* flag, cudaStream_t s) {
  if (S.dn_g.ent) {
    const size_t sm = static_cast<size_t>(S.Dd + 8) * sizeof(float4) + static_cast<size_t>(S.dn_g.nt) * 8 * sizeof(float2);
    if (sm <= 227 * 1024) {
      using K = void (*)(DevSector, const float2*, float2*, const int*);
      const K k = S.dn_g.xor_real ? bt_rows_staged_kernel<true> : bt_rows_staged_kernel<false>;
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm));
      if (e != cudaSuccess) return e;
      int dev = 0, nsm = 148;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      const int64_t items = S.Du * (kBtChains / 2);
      const int grid = static_cast<int>(std::min<int64_t>(items, nsm));
      k<<<grid, kBtsThreads, sm, s>>>(S, W, Y, flag);
      return cudaGetLastError();
    }
  }
  bt_rows_kernel<<<kBtBlocks, kBtThreads, 0, s>>>(S, W, Y, flag);
  return cudaGetLastError();
}

cudaError_t launch_bt_cols(int cols_variant, const DevSector& S, const float2* W, float2* Y, double* partial,
                           const int* flag, cudaStream_t s) {
  if (cols_variant == 1)
    bt_cols_kernel<8><<<kBtBlocks, kBtThreads, 0, s>>>(S, W, Y, partial, flag);
  else if (cols_variant == 2)
    bt_cols_kernel<4><<<kBtBlocks, kBtThreads, 0, s>>>(S, W, Y, partial, flag);
  else
    bt_cols_kernel<16><<<kBtBlocks, kBtThreads, 0, s>>>(S, W, Y, partial, flag);
  return cudaGetLastError();
}

// W_{k+1} = s_in Y - c1 W_k - c2 W_{k-1} (in Y's buffer, FP64 then rounded), ||W_{k+1}||^2 partials per chain.
__global__ void __launch_bounds__(kBtThreads, kBtBlocksPerSm) bt_update_kernel(float2* __restrict__ Y,
                                                                               const float2* __restrict__ Wk,
                                                                               const float2* __restrict__ Wkm1,
                                                                               int64_t dim, const double* __restrict__ st,
                                                                               int use_prev, double* __restrict__ partial,
                                                                               int* __restrict__ flag) {
  __shared__ double sh[kBtThreads];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double s_in = st[kBtSin * 32 + lane];
  const double c1r = st[kBtC1r * 32 + lane], c1i = st[kBtC1i * 32 + lane];
  const double c2 = use_prev ? st[kBtC2 * 32 + lane] : 0.0;
  Neu acc;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kBtWarps;
  for (int64_t i0 = static_cast<int64_t>(blockIdx.x) * kBtWarps + warp; i0 < dim; i0 += 4 * stride) {
    float2 y[4], a[4], b[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int64_t i = i0 + t * stride;
      const int64_t o = (i < dim ? i : i0) * 32 + lane;
      y[t] = Y[o];
      a[t] = Wk[o];
      b[t] = use_prev ? Wkm1[o] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int64_t i = i0 + t * stride;
      if (i >= dim) continue;
      double wr = s_in * static_cast<double>(y[t].x) - (c1r * a[t].x - c1i * a[t].y);
      double wi = s_in * static_cast<double>(y[t].y) - (c1r * a[t].y + c1i * a[t].x);
      wr -= c2 * b[t].x;
      wi -= c2 * b[t].y;
      const float2 w = make_float2(static_cast<float>(wr), static_cast<float>(wi));
      if (tinyf(w) && (w.x != 0.f || w.y != 0.f)) *flag = 1;
      Y[i * 32 + lane] = w;
      acc.add(static_cast<double>(w.x) * w.x + static_cast<double>(w.y) * w.y);
    }
  }
  double v[1] = {acc.value()};
  lane_block_sum<1>(v, sh);
  if (threadIdx.x < 32) partial[blockIdx.x * 32 + lane] = v[0];
}

// One warp: chain lane.  mode 0: start norms -> s_in = 1/||raw||, c2 = 0.
// mode 1: dot partials <W_k, H W_k> -> z = s_in^2 <W_k, H W_k>, alpha_k, c1 = z * s_in.  mode 2: norm partials -> beta_k, next
// s_in = 1/beta_k, c2 = beta_k * s_in (old), breakdown bookkeeping.
__global__ void bt_scalar_kernel(const double* __restrict__ partial, int nblocks, int mode, int k,
                                 double* __restrict__ st, double* __restrict__ alpha, double* __restrict__ beta,
                                 int* __restrict__ used) {
  const int lane = threadIdx.x;
  if (lane >= 32) return;
  if (mode == 1) {
    Neu sr, si;
    for (int b = 0; b < nblocks; ++b) {
      sr.add(partial[(b * 32 + lane) * 2]);
      si.add(partial[(b * 32 + lane) * 2 + 1]);
    }
    const double s_in = st[kBtSin * 32 + lane];
    const double zr = sr.value() * s_in * s_in, zi = si.value() * s_in * s_in;
    st[kBtC1r * 32 + lane] = zr * s_in;
    st[kBtC1i * 32 + lane] = zi * s_in;
    if (st[kBtActive * 32 + lane] != 0.0) alpha[k * 32 + lane] = zr;
    return;
  }
  Neu s;
  for (int b = 0; b < nblocks; ++b) s.add(partial[b * 32 + lane]);
  const double n2 = s.value();
  if (mode == 0) {
    const double n0 = sqrt(n2);
    st[kBtSin * 32 + lane] = (n0 < 1e-18) ? 0.0 : 1.0 / n0;
    st[kBtC2 * 32 + lane] = 0.0;
    st[kBtActive * 32 + lane] = (n0 < 1e-18) ? 0.0 : 1.0;
    used[lane] = 0;
    return;
  }
  const bool active = st[kBtActive * 32 + lane] != 0.0;
  const double s_in = st[kBtSin * 32 + lane];
  if (!active) {
    st[kBtSin * 32 + lane] = 0.0;
    st[kBtC2 * 32 + lane] = 0.0;
    return;
  }
  used[lane] = k + 1;
  if (n2 < 1e-24) {  // breakdown (src/lanczos.cpp:187): alpha_k kept, no beta_k
    st[kBtActive * 32 + lane] = 0.0;
    st[kBtSin * 32 + lane] = 0.0;
    st[kBtC2 * 32 + lane] = 0.0;
    return;
  }
  const double b = sqrt(n2);
  beta[k * 32 + lane] = b;
  st[kBtC2 * 32 + lane] = b * s_in;
  st[kBtSin * 32 + lane] = 1.0 / b;
}

// Orbit momentum block, 32 chains: Y[a, :] = H_K W[a, :] (complex64 block vectors over the
// block's representatives) and the fused <W_k, Y> per chain.  Warp per representative: the lanes
// walk the representative's sources in the sector's gather tables 32 at a time (table lookup and
// coefficient <rep a|H|s> eta conj(chi(R)) sqrt|A_b| / sqrt|A_a| in FP64, rounded to complex64) and
// compact the surviving ones into the warp's shared-memory list; then the half-warps gather the
// 256-byte rows W[b, :] as in the column pass.  Same algebra as the complex128 apply_tables kernel.
constexpr int kOrbTerms = 256;

__device__ __forceinline__ void orb_push(bool ok, uint32_t off, float2 cf, int lane, int& cnt, uint32_t* s_off,
                                         float2* s_cf) {
  const uint32_t m = __ballot_sync(0xffffffffu, ok);
  if (ok) {
    const int pos = cnt + __popc(m & ((1u << lane) - 1u));
    s_off[pos] = off;
    s_cf[pos] = cf;
  }
  cnt += __popc(m);
}

__device__ __forceinline__ float2 orb_coef(const OrbitApplyDev& A, double2 c, uint32_t e, double inv_sa) {
  const double2 ch = A.chi_tab[(e >> 24) & 15u];
  const double f = (((e >> 28) & 1u) ? -1.0 : 1.0) * A.sqrtA[e & 0xFFFFFFu] * inv_sa;
  return make_float2(static_cast<float>(f * (c.x * ch.x + c.y * ch.y)), static_cast<float>(f * (c.y * ch.x - c.x * ch.y)));
}

__global__ void __launch_bounds__(kBtThreads, kBtBlocksPerSm) bt_orbit_kernel(OrbitApplyDev A, const float2* __restrict__ W,
                                                                              float2* __restrict__ Y,
                                                                              const double* __restrict__ st,
                                                                              double* __restrict__ partial,
                                                                              const int* __restrict__ flag) {
  __shared__ uint32_t s_off[kBtWarps][kOrbTerms];
  __shared__ float2 s_cf[kBtWarps][kOrbTerms];
  __shared__ double sh[4 * kBtThreads];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int hv = lane >> 4, l = lane & 15;
  const bool filter = *flag != 0;
  const DevSector& S = A.S;
  const int64_t Dd = S.Dd;
  const float4* W4 = reinterpret_cast<const float4*>(W);
  float4* Y4 = reinterpret_cast<float4*>(Y);
  uint32_t* off = s_off[warp];
  float2* cfs = s_cf[warp];
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  double d0r = 0.0, d0i = 0.0, d1r = 0.0, d1i = 0.0;
  for (int64_t a = static_cast<int64_t>(blockIdx.x) * kBtWarps + warp; a < A.dk;
       a += static_cast<int64_t>(gridDim.x) * kBtWarps) {
    const uint32_t pk = A.reps[a];
    const uint32_t u = pk >> 16, d = pk & 0xFFFFu;
    const int32_t ru = A.O.rank_u[u], rd = A.O.rank_d[d];
    const double inv_sa = 1.0 / A.sqrtA[a];
    int cnt = 0;
    __syncwarp();
    const uint32_t q = prefix_parity_shifted(d);
    const int p1 = S.up_ptr[ru + 1];
    for (int p0 = S.up_ptr[ru]; p0 < p1; p0 += 32) {
      const int p = p0 + lane;
      bool ok = false;
      uint32_t o = 0;
      float2 cf = make_float2(0.f, 0.f);
      if (p < p1) {
        const uint32_t e = __ldg(A.table + static_cast<int64_t>(S.up_src[p]) * Dd + rd);
        if (e != kNone) {
          const uint32_t lh = S.up_lohi[p];
          double2 c = S.up_coef[p];
          if (((q >> (lh & 255u)) ^ (q >> (lh >> 8))) & 1u) c = make_double2(-c.x, -c.y);
          ok = true;
          o = (e & 0xFFFFFFu) * 16u;
          cf = orb_coef(A, c, e, inv_sa);
        }
      }
      orb_push(ok, o, cf, lane, cnt, off, cfs);
    }
    const int64_t rowbase = static_cast<int64_t>(ru) * Dd;
    const int64_t d1 = S.dn_csr_ptr[rd + 1];
    for (int64_t p0 = S.dn_csr_ptr[rd]; p0 < d1; p0 += 32) {
      const int64_t p = p0 + lane;
      bool ok = false;
      uint32_t o = 0;
      float2 cf = make_float2(0.f, 0.f);
      if (p < d1) {
        const uint32_t ent = S.dn_csr_ent[p];
        const int h = static_cast<int>((ent >> 1) & 255u);
        if (h != S.n_dn_hops) {
          const uint32_t e = __ldg(A.table + rowbase + (ent >> 9));
          if (e != kNone) {
            double2 c = S.dn_coef[h];
            if ((ent & 1u) ^ (static_cast<uint32_t>(__popc(u & S.dn_nmask[h])) & 1u)) c = make_double2(-c.x, -c.y);
            ok = true;
            o = (e & 0xFFFFFFu) * 16u;
            cf = orb_coef(A, c, e, inv_sa);
          }
        }
      }
      orb_push(ok, o, cf, lane, cnt, off, cfs);
    }
    const int deg8 = (cnt + 7) & ~7;
    for (int j = cnt + lane; j < deg8; j += 32) {  // padding: a valid row, zero coefficient
      off[j] = static_cast<uint32_t>(a) * 16u;
      cfs[j] = make_float2(0.f, 0.f);
    }
    __syncwarp();
    const float4* Wc = W4 + l;
    const float4 acc = filter ? bt_cols_sum<true>(Wc, off, cfs, deg8, hv) : bt_cols_sum<false>(Wc, off, cfs, deg8, hv);
    if (hv == 0) {
      float4 w = W4[static_cast<uint32_t>(a) * 16u + l];
      const float4 wf = filter ? filt4(w) : w;
      const float dg = static_cast<float>(diag_value(S, u, d, S.cnt_uu[ru], S.cnt_dd[rd], S.wpl[ru]));
      float4 y;
      y.x = acc.x + dg * wf.x;
      y.y = acc.y + dg * wf.y;
      y.z = acc.z + dg * wf.z;
      y.w = acc.w + dg * wf.w;
      Y4[static_cast<uint32_t>(a) * 16u + l] = y;
      const double wx = w.x, wy = w.y, wz = w.z, ww = w.w;
      const double yx = y.x, yy = y.y, yz = y.z, yw = y.w;
      d0r = fma(wx, yx, fma(wy, yy, d0r));
      d0i = fma(wx, yy, fma(-wy, yx, d0i));
      d1r = fma(wz, yz, fma(ww, yw, d1r));
      d1i = fma(wz, yw, fma(-ww, yz, d1i));
    }
  }
  const int t = threadIdx.x;
  sh[0 * kBtThreads + t] = d0r;
  sh[1 * kBtThreads + t] = d0i;
  sh[2 * kBtThreads + t] = d1r;
  sh[3 * kBtThreads + t] = d1i;
  __syncthreads();
  if (t < 32) {
    const int ll = t & 15, which = t >> 4;
    double re = 0.0, im = 0.0;
    for (int w = 0; w < kBtWarps; ++w) {
      re += sh[(2 * which) * kBtThreads + w * 32 + ll];
      im += sh[(2 * which + 1) * kBtThreads + w * 32 + ll];
    }
    const int chain = 2 * ll + which;
    partial[(blockIdx.x * 32 + chain) * 2] = re;
    partial[(blockIdx.x * 32 + chain) * 2 + 1] = im;
  }
}

}  // namespace

cudaError_t bt_start(float2* W, int64_t dim, unsigned seed, double* st, double* partial, int* used, int* flags,
                     cudaStream_t s, const DevSector* gauge) {
  cudaError_t e = cudaMemsetAsync(flags, 0, 2 * sizeof(int), s);
  if (e != cudaSuccess) return e;
  bt_start_kernel<<<kBtBlocks, kBtThreads, 0, s>>>(W, dim, seed, partial, flags, gauge ? gauge->umask : nullptr,
                                                   gauge ? gauge->dmask : nullptr, gauge ? gauge->Dd : 1);
  bt_scalar_kernel<<<1, 32, 0, s>>>(partial, kBtBlocks, 0, 0, st, nullptr, nullptr, used);
  return cudaGetLastError();
}

cudaError_t bt_step(const DevSector& S, const float2* Wk, const float2* Wkm1, float2* Y, int k, double* st,
                    double* partial, double* alpha, double* beta, int* used, int* flags, cudaStream_t s) {
  // flags[k % 2]: written vector W_k has a tiny non-zero entry; flags[(k+1) % 2] is cleared for W_{k+1}.
  int* fin = flags + (k & 1);
  int* fout = flags + ((k + 1) & 1);
  cudaError_t e = cudaMemsetAsync(fout, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  launch_bt_rows(S, Wk, Y, fin, s);
  launch_bt_cols(S.bt_cols, S, Wk, Y, partial, fin, s);
  bt_scalar_kernel<<<1, 32, 0, s>>>(partial, kBtBlocks, 1, k, st, alpha, beta, used);
  bt_update_kernel<<<kBtBlocks, kBtThreads, 0, s>>>(Y, Wk, Wkm1, S.dim, st, k > 0, partial, fout);
  bt_scalar_kernel<<<1, 32, 0, s>>>(partial, kBtBlocks, 2, k, st, alpha, beta, used);
  return cudaGetLastError();
}

cudaError_t bt_orbit_step(const OrbitApplyDev& A, const float2* Wk, const float2* Wkm1, float2* Y, int k, double* st,
                          double* partial, double* alpha, double* beta, int* used, int* flags, cudaStream_t s) {
  int* fin = flags + (k & 1);
  int* fout = flags + ((k + 1) & 1);
  cudaError_t e = cudaMemsetAsync(fout, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  bt_orbit_kernel<<<kBtBlocks, kBtThreads, 0, s>>>(A, Wk, Y, st, partial, fin);
  bt_scalar_kernel<<<1, 32, 0, s>>>(partial, kBtBlocks, 1, k, st, alpha, beta, used);
  bt_update_kernel<<<kBtBlocks, kBtThreads, 0, s>>>(Y, Wk, Wkm1, A.dk, st, k > 0, partial, fout);
  bt_scalar_kernel<<<1, 32, 0, s>>>(partial, kBtBlocks, 2, k, st, alpha, beta, used);
  return cudaGetLastError();
}

cudaError_t bt_apply(const DevSector& S, const float2* X, float2* Y, const double* st_unit, double* partial,
                     const int* zero_flag, cudaStream_t s) {
  (void)st_unit;
  launch_bt_rows(S, X, Y, zero_flag, s);
  launch_bt_cols(S.bt_cols, S, X, Y, partial, zero_flag, s);
  return cudaGetLastError();
}

}  // namespace ftlm_b200
