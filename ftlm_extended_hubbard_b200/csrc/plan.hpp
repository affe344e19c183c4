// Host-side sector plan: the (N_up, N_dn) Fock basis in factorised form and the gather
// tables the device kernels read.  Pure C++ (no CUDA), so its integer work is checkable on CPU.
//
// Basis (reference src/fock_basis.cpp:17-42): strings of one spin species are the k-subsets
// of the n sites in lexicographic order of their sorted site lists; state index =
// rank_up * C(n, n_dn) + rank_dn.  Here the two string lists are kept separately (the state
// is never materialised as a dim-long mask pair) and ranks come from a closed form instead of
// a hash map: lex_rank(m) = C(n,k) - 1 - colex_rank(bitreverse_n(m)).
//
// Operator (reference src/hubbard_hamiltonian.cpp:51-108), gather form, per spin species:
//   up hop  f->t (lo<hi the two sites): JW sign = (-1)^(#up in (lo,hi) + #dn in [lo,hi))
//   dn hop  f->t                      : JW sign = (-1)^(#up in (lo,hi] + #dn in (lo,hi))
// The factor that depends only on the moving species' string is folded into the table
// coefficient; the factor that depends on the other species' string is applied per element
// (up part: from the prefix parity of the down string; down part: per up row, per hop).
// Duplicate directed hops (same spin, from, to) are merged by summing their coefficients in
// list order — the JW sign depends only on (spin, from, to), so the operator is unchanged.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ftlm_b200 {

struct HopIn {
  int from, to, spin;
  double cre, cim;
};
struct PairIn {
  int i, j;
};

uint64_t binom(int n, int k);

struct SpinSpace {
  int n = 0, k = 0;
  int64_t D = 0;
  std::vector<uint32_t> masks;  // lexicographic order
  void build(int n_, int k_);
  int64_t rank(uint32_t m) const;  // -1 if m is not a k-subset of the n sites
};

// One merged directed hop of one spin species.
struct MergedHop {
  int from, to;
  double cre, cim;
  uint32_t own_mask;    // sites of the same species strictly between lo and hi
  uint32_t other_mask;  // sites of the other species counted by the JW sign
  int lo, hi;
};

// Hop gather table of one spin in the spin-ordered (gauge) basis g(u, d) = (-1)^popc(u & pps(d)),
// pps(d) = prefix parity of d shifted by one site.  In that basis a hop's coefficient is (-1)^s c_h,
// s the JW sign of the hopping species' own string alone, so the same table serves every string of
// the other species.  Built when D + 8 <= 16384, n_sites <= 32 and at most 512 hops need a table
// coefficient.  Per group of 32 output strings (grp[4g..4g+3] = entry offset, KR, KT, KR0 | KT0<<16),
// rounds k = 0 .. KR+KT-1 (KR and KT each padded to a multiple of 4 with sentinel rounds; KR0 and KT0
// are the rounds before that padding),
// entry of round k for lane l at grp[4g] + ((k / 4) * 32 + l) * 4 + k % 4 (one 16-byte load per
// lane brings 4 rounds):
//   real section  (rounds k < KR = grp[4g+1]): hops with c_h = real2[cls], cls in {0, 1};
//                 entry = src<<4 | cls<<30 | s<<31
//   table section (KR <= k < KR + KT, KT = grp[4g+2]): any other hop; entry = src<<4 | t<<18 | s<<31
//                 with c_h = (tab[2t], tab[2t+1])
// src << 4 is the byte offset of the 16-byte element in the staged line; src >= D addresses one of 8
// zero sentinels after it (padding, one per bank group).  Each section is scheduled so that the 8
// lanes of a quarter-warp read 8 different bank groups in every round.
// Phase form (phase = true): every table coefficient is one of the two real values times a single
// unit phase p = (pc, ps) or its conjugate, bit for bit (tab[t] == real2[k] * (pc, +-ps) in double
// arithmetic) — the case of one Peierls phase, e.g. phi_x != 0 and phi_y == 0.  Table-section entries
// then also carry cls<<30 and conj<<27, so the row pass forms the coefficient from registers instead
// of loading it from the shared-memory table (same product, same rounding).
// XOR form (xor_real = true): real-section entries carry, instead of cls<<30 | s<<31, the bits 18..31
// by which the high word of (-1)^s real2[cls] differs from that of real2[0] (possible when real2[0]
// and real2[1] share their low words and their high words differ only in bits 18..31), so the row
// pass forms the coefficient with one XOR.  Both sections are padded to whole 4-entry loads.
struct GaugeTable {
  bool ok = false;
  bool phase = false;
  bool xor_real = false;
  uint32_t xor_d = 0;
  double pc = 1.0, ps = 0.0;
  double real2[2] = {0.0, 0.0};
  std::vector<double> tab;
  std::vector<int32_t> grp;
  std::vector<uint32_t> ent;
  // lane permutation, 32 per group: the entries of lane L of group g belong to output string
  // g*32 + perm[32g + L] (the bank-group loads of the quarter-warps balanced; identity on the last,
  // partial group)
  std::vector<uint8_t> perm;
};

struct SectorPlan {
  int n = 0, nu = 0, nd = 0;
  double U = 0.0, V = 0.0;
  SpinSpace up, dn;
  std::vector<MergedHop> hu, hd;
  std::vector<PairIn> pairs;
  int64_t dim = 0;

  // Diagonal: H_ii = U*popc(u&d) + V*(cnt_uu[ru] + cnt_dd[rd] + sum_b 2^b popc(d & wpl[ru][b])).
  std::vector<int32_t> cnt_uu, cnt_dd;
  std::vector<uint32_t> wpl;  // 4 per up string: bit-planes of #pair partners occupied by up

  // Up part (gather CSR over output up ranks): sources, coefficient with the up-string JW
  // factor folded in, and packed (lo | hi<<8) for the per-element down-string factor.
  std::vector<int32_t> up_ptr, up_src;
  std::vector<double> up_coef;  // 2 per entry
  std::vector<uint32_t> up_lohi;
  // The same list packed into one word per entry for the column pass (built when Du <= 16384, at
  // most 32 sites, and every coefficient is (-1)^s real2[cls], or that times (pc, +-ps) for one unit
  // phase, bit for bit): src | lo<<14 | hi<<19 | conj<<28 | phase<<29 | cls<<30 | s<<31.
  bool up_pk_ok = false;
  double up_real2[2] = {0.0, 0.0};
  double up_pc = 1.0, up_ps = 0.0;
  std::vector<uint32_t> up_pk;

  // Down part (ELL, 32 consecutive output down ranks per group, entry k of lane l at
  // dn_gptr[g] + 32k + l): entry = src_rank<<10 | hop_id<<1 | dn_string_sign.  Padding
  // entries carry hop_id == dn_pad_hop.  Per down hop: coefficient and the up-site mask of
  // its per-row sign.
  std::vector<int64_t> dn_gptr;
  std::vector<uint32_t> dn_ent;
  int dn_pad_hop = 0;
  // Batched path: per output down string, entries src<<9 | (2*hop_id + sign), padded to a multiple
  // of 8 with (self, pad hop) entries: dn_csr_ptr[Dd+1], dn_csr_ent.
  std::vector<int64_t> dn_csr_ptr;
  std::vector<uint32_t> dn_csr_ent;
  std::vector<double> dn_coef;     // 2 per hop id (pad hop id has 0)
  std::vector<uint32_t> dn_nmask;  // per hop id

  // Down-hop gather table of the row pass in the spin-ordered (gauge) basis (see GaugeTable).
  GaugeTable dn_g;

  double mean_up_sources = 0.0, mean_dn_sources = 0.0;
  int max_dn_deg = 0, max_up_deg = 0;
};

// Builds the plan; returns "" on success or an error message (reference argument errors:
// src/fock_basis.cpp:19-24).
std::string build_plan(int n_sites, int n_up, int n_dn, double U, double V, const std::vector<HopIn>& hops,
                       const std::vector<PairIn>& pairs, SectorPlan* out);

// Diagonal entry from the plan tables (host).
double plan_diag(const SectorPlan& p, int64_t ru, int64_t rd);

// build_hubbard_geometry (reference src/lattice.cpp:38-110), host.
void build_geometry(int Lx, int Ly, double t, double tp, double phix, double phiy, std::vector<HopIn>* hops,
                    std::vector<PairIn>* pairs);

}  // namespace ftlm_b200
