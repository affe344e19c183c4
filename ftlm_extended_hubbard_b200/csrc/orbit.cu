// Translation-orbit k-block kernels; conventions in orbit.cuh.
//
// Canonical representative = the translation image with the smallest packed (up<<16 | dn)
// (include/ftlm/symmetry/orbit.hpp:115-119).  For a state s, R is the first translation in the
// reference's search order (dx outer, dy inner; src/orbit_k_block_basis.cpp:225-236) with
// T_R rep = s, and eta = (-1)^(inversions of the occupied modes 2*site+spin, listed in site order,
// after translation) (include/ftlm/symmetry/fermionic_translation.hpp:32-54).
#include "orbit.cuh"

namespace ftlm_b200 {

namespace {

__device__ __forceinline__ uint32_t translate(const OrbitDev& O, int R, uint32_t m) {
  const uint16_t* t = O.tlut + R * 512;
  return static_cast<uint32_t>(t[m & 255u]) | static_cast<uint32_t>(t[256 + (m >> 8)]);
}

// Parity of the inversions of T_R on the occupied modes of (u, d).
__device__ __forceinline__ uint32_t translation_sign(const OrbitDev& O, int R, uint32_t u, uint32_t d) {
  const uint8_t* ts = O.tsite + R * 16;
  uint64_t seen = 0;
  uint32_t inv = 0;
  for (int s = 0; s < O.n; ++s) {
    const uint32_t tsite = ts[s];
    if ((u >> s) & 1u) {
      const uint32_t tm = 2u * tsite;
      inv += __popcll(seen >> (tm + 1));
      seen |= 1ull << tm;
    }
    if ((d >> s) & 1u) {
      const uint32_t tm = 2u * tsite + 1u;
      inv += __popcll(seen >> (tm + 1));
      seen |= 1ull << tm;
    }
  }
  return inv & 1u;
}

__global__ void canon_kernel(OrbitDev O, int32_t* __restrict__ rep_full, uint8_t* __restrict__ reta) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < O.dim; i += stride) {
    const int64_t ru = i / O.Dd;
    const uint32_t u = O.umask[ru], d = O.dmask[i - ru * O.Dd];
    uint32_t best = (u << 16) | d;
    for (int R = 1; R < O.G; ++R) {
      const uint32_t p = (translate(O, R, u) << 16) | translate(O, R, d);
      best = min(best, p);
    }
    const uint32_t bu = best >> 16, bd = best & 0xFFFFu;
    int Rf = 0;
    for (int k = 0; k < O.G; ++k) {
      const int R = O.rorder[k];
      if (translate(O, R, bu) == u && translate(O, R, bd) == d) {
        Rf = R;
        break;
      }
    }
    rep_full[i] = static_cast<int32_t>(static_cast<int64_t>(O.rank_u[bu]) * O.Dd + O.rank_d[bd]);
    reta[i] = static_cast<uint8_t>(Rf | (translation_sign(O, Rf, bu, bd) << 4));
  }
}

__global__ void absA_kernel(OrbitDev O, const uint32_t* __restrict__ reps, int64_t nreps,
                            const double2* __restrict__ chi_tab, double* __restrict__ absA, double2* __restrict__ Aout,
                            int* __restrict__ stab) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b < nreps; b += stride) {
    const uint32_t u = reps[b] >> 16, d = reps[b] & 0xFFFFu;
    double ar = 0.0, ai = 0.0;
    int ns = 0;
    for (int R = 0; R < O.G; ++R) {  // dy outer, dx inner: R = dy * Lx + dx ascending
      if (translate(O, R, u) != u || translate(O, R, d) != d) continue;
      ++ns;
      const double eta = translation_sign(O, R, u, d) ? -1.0 : 1.0;
      ar += eta * chi_tab[R].x;
      ai += eta * chi_tab[R].y;
    }
    absA[b] = hypot(ar, ai);
    if (Aout) Aout[b] = make_double2(ar, ai);
    if (stab) stab[b] = ns;
  }
}

__global__ void table_kernel(OrbitDev O, const int32_t* __restrict__ rep_full, const uint8_t* __restrict__ reta,
                             const int32_t* __restrict__ red_of_full, uint32_t* __restrict__ table) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < O.dim; i += stride) {
    const int32_t b = red_of_full[rep_full[i]];
    table[i] = (b < 0) ? 0xFFFFFFFFu : (static_cast<uint32_t>(b) | (static_cast<uint32_t>(reta[i]) << 24));
  }
}

__device__ __forceinline__ void orbit_term(const OrbitApplyDev& A, int64_t j, double2 hval, double sa,
                                           const double2* __restrict__ x, double2& acc) {
  const uint32_t e = A.table[j];
  if (e == 0xFFFFFFFFu) return;
  const uint32_t beta = e & 0xFFFFFFu;
  const double2 xb = x[beta];
  if (tiny(xb)) return;
  const int R = static_cast<int>((e >> 24) & 15u);
  const double eta = ((e >> 28) & 1u) ? -1.0 : 1.0;
  const double2 ch = A.chi_tab[R];
  // h * eta * chi(R) * sqrt(|A_beta| / |A_alpha|), then conjugated (gather from the Hermitian H_K)
  const double f = eta * A.sqrtA[beta] * sa;
  const double cr = f * (hval.x * ch.x - hval.y * ch.y);
  const double ci = -f * (hval.x * ch.y + hval.y * ch.x);
  acc.x = fma(cr, xb.x, acc.x);
  acc.x = fma(-ci, xb.y, acc.x);
  acc.y = fma(cr, xb.y, acc.y);
  acc.y = fma(ci, xb.x, acc.y);
}

__global__ void __launch_bounds__(256) apply_kernel(OrbitApplyDev A, const double2* __restrict__ x,
                                                    double2* __restrict__ y) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t a = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; a < A.dk; a += stride) {
    const uint32_t u = A.reps[a] >> 16, d = A.reps[a] & 0xFFFFu;
    const int32_t ru = A.O.rank_u[u], rd = A.O.rank_d[d];
    double2 acc = make_double2(0.0, 0.0);
    const double2 xa = x[a];
    if (!tiny(xa)) {
      const double dg = diag_value(A.S, u, d, A.S.cnt_uu[ru], A.S.cnt_dd[rd], A.S.wpl[ru]);
      acc.x = dg * xa.x;
      acc.y = dg * xa.y;
    }
    const double sa = 1.0 / A.sqrtA[a];
    for (int h = 0; h < A.n_uhops; ++h) {
      const int f = A.uhop_from[h], t = A.uhop_to[h];
      if (!((u >> f) & 1u) || ((u >> t) & 1u)) continue;
      const uint32_t u2 = u ^ (1u << f) ^ (1u << t);
      const uint32_t neg = (__popc(u & A.uhop_own[h]) + __popc(d & A.uhop_oth[h])) & 1u;
      double2 hv = A.uhop_c[h];
      if (neg) hv = make_double2(-hv.x, -hv.y);
      orbit_term(A, static_cast<int64_t>(A.O.rank_u[u2]) * A.O.Dd + rd, hv, sa, x, acc);
    }
    for (int h = 0; h < A.n_dhops; ++h) {
      const int f = A.dhop_from[h], t = A.dhop_to[h];
      if (!((d >> f) & 1u) || ((d >> t) & 1u)) continue;
      const uint32_t d2 = d ^ (1u << f) ^ (1u << t);
      const uint32_t neg = (__popc(d & A.dhop_own[h]) + __popc(u & A.dhop_oth[h])) & 1u;
      double2 hv = A.dhop_c[h];
      if (neg) hv = make_double2(-hv.x, -hv.y);
      orbit_term(A, static_cast<int64_t>(ru) * A.O.Dd + A.O.rank_d[d2], hv, sa, x, acc);
    }
    y[a] = acc;
  }
}

// sqrt(|A_b|) x_b with the reference's source-skip rule applied (a skipped source contributes
// exactly nothing, and a zero contributes exactly nothing to the gathers below).
__global__ void prescale_kernel(int64_t dk, const double* __restrict__ sqrtA, const double2* __restrict__ x,
                                double2* __restrict__ xs) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b < dk; b += stride) {
    const double2 v = x[b];
    const double f = sqrtA[b];
    xs[b] = tiny(v) ? make_double2(0.0, 0.0) : make_double2(f * v.x, f * v.y);
  }
}

// Thread per representative alpha, driven by the sector's own gather tables: the up sources of
// rep(alpha) are the CSR row of its up string, the down sources the padded list of its down
// string, each with the matrix element <rep alpha|H|s>.  By Hermiticity of H_K,
//   H_K[alpha, beta] = sum_{s in orbit beta} <rep alpha|H|s> eta(beta, R_s) conj(chi(R_s)) sqrt|A_beta| / sqrt|A_alpha|,
// so y_alpha = diag x_alpha + (1/sqrt|A_alpha|) sum <rep alpha|H|s> eta conj(chi) xs_beta.
// Sources are taken four at a time: four table lookups, then four gathers of xs, in flight together.
constexpr int kOrbBatch = 4;

__device__ __forceinline__ void orbit_acc(double2 c, uint32_t e, double2 xb, double2& acc, const double2* chi) {
  const double2 ch = chi[(e >> 24) & 15u];
  const double eta = ((e >> 28) & 1u) ? -1.0 : 1.0;
  const double cr = eta * (c.x * ch.x + c.y * ch.y);
  const double ci = eta * (c.y * ch.x - c.x * ch.y);
  acc.x = fma(cr, xb.x, acc.x);
  acc.x = fma(-ci, xb.y, acc.x);
  acc.y = fma(cr, xb.y, acc.y);
  acc.y = fma(ci, xb.x, acc.y);
}

__global__ void __launch_bounds__(256) apply_tables_kernel(OrbitApplyDev A, const double2* __restrict__ x,
                                                           double2* __restrict__ y) {
  const DevSector& S = A.S;
  const int64_t Dd = A.O.Dd;
  const double2* __restrict__ xs = A.xs;
  const uint32_t* __restrict__ table = A.table;
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t a = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; a < A.dk; a += stride) {
    const uint32_t pk = A.reps[a];
    const uint32_t u = pk >> 16, d = pk & 0xFFFFu;
    const int32_t ru = A.O.rank_u[u], rd = A.O.rank_d[d];
    double2 acc = make_double2(0.0, 0.0);
    // up sources: same down string, rows up_src
    const uint32_t q = prefix_parity_shifted(d);
    const int p1 = S.up_ptr[ru + 1];
    for (int p = S.up_ptr[ru]; p < p1; p += kOrbBatch) {
      uint32_t e[kOrbBatch];
      double2 c[kOrbBatch], xv[kOrbBatch];
#pragma unroll
      for (int k = 0; k < kOrbBatch; ++k) {
        e[k] = kNone;
        if (p + k < p1) {
          const uint32_t lh = S.up_lohi[p + k];
          const uint32_t neg = ((q >> (lh & 255u)) ^ (q >> (lh >> 8))) & 1u;
          c[k] = S.up_coef[p + k];
          if (neg) c[k] = make_double2(-c[k].x, -c[k].y);
          e[k] = __ldg(table + static_cast<int64_t>(S.up_src[p + k]) * Dd + rd);
        }
      }
#pragma unroll
      for (int k = 0; k < kOrbBatch; ++k) xv[k] = e[k] != kNone ? xs[e[k] & 0xFFFFFFu] : make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < kOrbBatch; ++k)
        if (e[k] != kNone) orbit_acc(c[k], e[k], xv[k], acc, A.chi_tab);
    }
    // down sources: same up string, columns from the padded down list
    const int64_t rowbase = static_cast<int64_t>(ru) * Dd;
    const int64_t d1 = S.dn_csr_ptr[rd + 1];
    for (int64_t p = S.dn_csr_ptr[rd]; p < d1; p += kOrbBatch) {
      uint32_t e[kOrbBatch];
      double2 c[kOrbBatch], xv[kOrbBatch];
#pragma unroll
      for (int k = 0; k < kOrbBatch; ++k) {
        e[k] = kNone;
        const uint32_t ent = S.dn_csr_ent[p + k];  // lists are padded to a multiple of 8
        const int h = static_cast<int>((ent >> 1) & 255u);
        if (h != S.n_dn_hops) {
          const uint32_t neg = (ent & 1u) ^ (static_cast<uint32_t>(__popc(u & S.dn_nmask[h])) & 1u);
          c[k] = S.dn_coef[h];
          if (neg) c[k] = make_double2(-c[k].x, -c[k].y);
          e[k] = __ldg(table + rowbase + (ent >> 9));
        }
      }
#pragma unroll
      for (int k = 0; k < kOrbBatch; ++k) xv[k] = e[k] != kNone ? xs[e[k] & 0xFFFFFFu] : make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < kOrbBatch; ++k)
        if (e[k] != kNone) orbit_acc(c[k], e[k], xv[k], acc, A.chi_tab);
    }
    const double sa = 1.0 / A.sqrtA[a];
    double2 out = make_double2(acc.x * sa, acc.y * sa);
    const double2 xa = x[a];
    if (!tiny(xa)) {
      const double dg = diag_value(S, u, d, S.cnt_uu[ru], S.cnt_dd[rd], S.wpl[ru]);
      out.x = fma(dg, xa.x, out.x);
      out.y = fma(dg, xa.y, out.y);
    }
    y[a] = out;
  }
}

__global__ void scatter_kernel(const int64_t* __restrict__ full, int64_t n, int32_t* __restrict__ red) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b < n; b += stride)
    red[full[b]] = static_cast<int32_t>(b);
}

int g_sms = 0;
// Order-preserving stream compaction: kCompactItems consecutive items per block (4 per thread, in
// thread order), block counts, one-block exclusive scan of the counts, then each block writes its
// flagged items at offset + in-block prefix.  Pred(p) -> bool, Emit(p, pos).
constexpr int kCompactThreads = 1024;
constexpr int kCompactItems = 4 * kCompactThreads;

template <class Pred>
__global__ void __launch_bounds__(kCompactThreads) compact_count_kernel(Pred pred, int64_t n, int32_t* counts) {
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kCompactItems + 4 * threadIdx.x;
  int c = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) c += (base + k < n && pred(base + k)) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  __shared__ int ws[kCompactThreads / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kCompactThreads / 32; ++w) t += ws[w];
    counts[blockIdx.x] = t;
  }
}

// counts[0..nb) -> exclusive offsets in place, total in counts[nb] (one block, chunks of 1024).
__global__ void __launch_bounds__(kCompactThreads) compact_scan_kernel(int32_t* counts, int64_t nb) {
  __shared__ int32_t buf[kCompactThreads];
  __shared__ int32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t b0 = 0; b0 < nb; b0 += kCompactThreads) {
    const int64_t b = b0 + threadIdx.x;
    const int32_t v = b < nb ? counts[b] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kCompactThreads; o <<= 1) {  // Hillis-Steele inclusive scan
      const int32_t add = threadIdx.x >= static_cast<unsigned>(o) ? buf[threadIdx.x - o] : 0;
      __syncthreads();
      buf[threadIdx.x] += add;
      __syncthreads();
    }
    if (b < nb) counts[b] = carry + buf[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 0) carry += buf[kCompactThreads - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) counts[nb] = carry;
}

template <class Pred, class Emit>
__global__ void __launch_bounds__(kCompactThreads) compact_write_kernel(Pred pred, Emit emit, int64_t n,
                                                                         const int32_t* offsets) {
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kCompactItems + 4 * threadIdx.x;
  bool f[4];
  int c = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    f[k] = base + k < n && pred(base + k);
    c += f[k] ? 1 : 0;
  }
  // exclusive prefix of c over the block (thread order)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  __shared__ int ws[kCompactThreads / 32];
  if (lane == 31) ws[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int v = ws[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    ws[lane] = v;
  }
  __syncthreads();
  int pos = offsets[blockIdx.x] + (warp > 0 ? ws[warp - 1] : 0) + incl - c;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (f[k]) emit(base + k, pos++);
}

// Phase 1: per-block counts, their exclusive scan and the total (synchronises st to read it back).
template <class Pred>
cudaError_t compact_count(Pred pred, int64_t n, int32_t* counts /* >= nb + 1 */, int64_t* total, cudaStream_t st) {
  *total = 0;
  if (n <= 0) return cudaSuccess;
  const int64_t nb = (n + kCompactItems - 1) / kCompactItems;
  compact_count_kernel<<<static_cast<unsigned>(nb), kCompactThreads, 0, st>>>(pred, n, counts);
  compact_scan_kernel<<<1, kCompactThreads, 0, st>>>(counts, nb);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  int32_t t = 0;
  e = cudaMemcpyAsync(&t, counts + nb, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  *total = t;
  return e;
}

// Phase 2: the flagged items, in order, to the outputs sized by phase 1.
template <class Pred, class Emit>
cudaError_t compact_write(Pred pred, Emit emit, int64_t n, const int32_t* counts, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t nb = (n + kCompactItems - 1) / kCompactItems;
  compact_write_kernel<<<static_cast<unsigned>(nb), kCompactThreads, 0, st>>>(pred, emit, n, counts);
  return cudaGetLastError();
}

// Position p of the packed order (up strings by mask value, then down strings by mask value) is the
// full state inv_u[p / Dd] * Dd + inv_d[p % Dd]; it is listed when it is its orbit's representative.
struct RepPred {
  const int32_t* rep_full;
  const int32_t* inv_u;
  const int32_t* inv_d;
  int64_t Dd;
  __device__ bool operator()(int64_t p) const {
    const int64_t i = static_cast<int64_t>(inv_u[p / Dd]) * Dd + inv_d[p % Dd];
    return rep_full[i] == i;
  }
};
struct RepEmit {
  const int32_t* inv_u;
  const int32_t* inv_d;
  const uint32_t* umask;
  const uint32_t* dmask;
  int64_t Dd;
  uint32_t* packed;
  int64_t* full;
  __device__ void operator()(int64_t p, int pos) const {
    const int32_t ru = inv_u[p / Dd], rd = inv_d[p % Dd];
    packed[pos] = (umask[ru] << 16) | dmask[rd];
    full[pos] = static_cast<int64_t>(ru) * Dd + rd;
  }
};

struct SurvivePred {
  const double* absA;
  double tol;
  __device__ bool operator()(int64_t b) const { return absA[b] > tol; }
};
struct SurviveEmit {
  OrbitBlockIn in;
  OrbitBlockOut out;
  __device__ void operator()(int64_t b, int pos) const {
    out.reps[pos] = in.reps[b];
    out.absA[pos] = in.absA[b];
    out.A[pos] = in.A[b];
    out.stab[pos] = in.stab[b];
    out.orbit_idx[pos] = b;
    out.full[pos] = in.full[b];
    out.sqrtA[pos] = sqrt(in.absA[b]);
  }
};

unsigned grid_for(int64_t n) {
  if (g_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_sms <= 0) g_sms = 148;
  }
  const int64_t b = (n + 255) / 256;
  return static_cast<unsigned>(b < 16 * g_sms ? (b > 0 ? b : 1) : 16 * g_sms);
}

}  // namespace

int64_t orbit_compact_counts(int64_t n) { return (n + kCompactItems - 1) / kCompactItems + 1; }

cudaError_t orbit_count_reps(const OrbitDev& O, const int32_t* rep_full, const int32_t* inv_u, const int32_t* inv_d,
                             int32_t* counts, int64_t* nreps, cudaStream_t st) {
  return compact_count(RepPred{rep_full, inv_u, inv_d, O.Dd}, O.dim, counts, nreps, st);
}

cudaError_t orbit_write_reps(const OrbitDev& O, const int32_t* rep_full, const int32_t* inv_u, const int32_t* inv_d,
                             const int32_t* counts, uint32_t* packed, int64_t* full, cudaStream_t st) {
  return compact_write(RepPred{rep_full, inv_u, inv_d, O.Dd},
                       RepEmit{inv_u, inv_d, O.umask, O.dmask, O.Dd, packed, full}, O.dim, counts, st);
}

cudaError_t orbit_count_survivors(const double* absA, int64_t nreps, double tol, int32_t* counts, int64_t* dk,
                                  cudaStream_t st) {
  return compact_count(SurvivePred{absA, tol}, nreps, counts, dk, st);
}

cudaError_t orbit_write_survivors(const OrbitBlockIn& in, int64_t nreps, double tol, const int32_t* counts,
                                  const OrbitBlockOut& out, cudaStream_t st) {
  return compact_write(SurvivePred{in.absA, tol}, SurviveEmit{in, out}, nreps, counts, st);
}

cudaError_t orbit_canon(const OrbitDev& O, int32_t* rep_full, uint8_t* reta, cudaStream_t st) {
  canon_kernel<<<grid_for(O.dim), 256, 0, st>>>(O, rep_full, reta);
  return cudaGetLastError();
}

cudaError_t orbit_absA(const OrbitDev& O, const uint32_t* reps, int64_t nreps, const double2* chi_tab, double* absA,
                       double2* A, int* stab, cudaStream_t st) {
  if (nreps <= 0) return cudaSuccess;
  absA_kernel<<<grid_for(nreps), 256, 0, st>>>(O, reps, nreps, chi_tab, absA, A, stab);
  return cudaGetLastError();
}

cudaError_t orbit_table(const OrbitDev& O, const int32_t* rep_full, const uint8_t* reta, const int32_t* red_of_full,
                        uint32_t* table, cudaStream_t st) {
  table_kernel<<<grid_for(O.dim), 256, 0, st>>>(O, rep_full, reta, red_of_full, table);
  return cudaGetLastError();
}

cudaError_t orbit_scatter_index(const int64_t* full, int64_t n, int32_t* red, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  scatter_kernel<<<grid_for(n), 256, 0, st>>>(full, n, red);
  return cudaGetLastError();
}

cudaError_t orbit_apply(const OrbitApplyDev& A, const double2* x, double2* y, cudaStream_t st) {
  if (A.dk <= 0) return cudaSuccess;
  if (A.path == 1 && A.xs != nullptr) {
    prescale_kernel<<<grid_for(A.dk), 256, 0, st>>>(A.dk, A.sqrtA, x, A.xs);
    apply_tables_kernel<<<grid_for(A.dk), 256, 0, st>>>(A, x, y);
    return cudaGetLastError();
  }
  apply_kernel<<<grid_for(A.dk), 256, 0, st>>>(A, x, y);
  return cudaGetLastError();
}

}  // namespace ftlm_b200
