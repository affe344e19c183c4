// Host-side sector plan; see plan.hpp for the conventions.
#include "plan.hpp"

#include <algorithm>
#include <cstdint>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <utility>

namespace ftlm_b200 {

namespace {

uint64_t g_binom[65][65];
bool g_binom_ready = false;

void init_binom() {
  if (g_binom_ready) return;
  for (int n = 0; n <= 64; ++n) {
    for (int k = 0; k <= 64; ++k) g_binom[n][k] = 0;
    g_binom[n][0] = 1;
    for (int k = 1; k <= n; ++k) g_binom[n][k] = g_binom[n - 1][k - 1] + (k <= n - 1 ? g_binom[n - 1][k] : 0);
  }
  g_binom_ready = true;
}

// Reference src/fock_basis.cpp:7-15: lexicographic k-subsets (lowest free position first).
void enumerate(int n, int k, int pos, uint32_t cur, std::vector<uint32_t>* out) {
  if (k == 0) {
    out->push_back(cur);
    return;
  }
  for (int i = pos; i <= n - k; ++i) enumerate(n, k - 1, i + 1, cur | (1u << i), out);
}

inline int popc(uint32_t x) { return __builtin_popcount(x); }

inline uint32_t range_mask(int a, int b) {  // sites a..b-1 (a <= b)
  const uint64_t hi = (b >= 32) ? 0xFFFFFFFFull : ((1ull << b) - 1);
  const uint64_t lo = (a >= 32) ? 0xFFFFFFFFull : ((1ull << a) - 1);
  return static_cast<uint32_t>(hi & ~lo);
}

// Merge directed hops of one spin by (from, to), summing coefficients in list order.
std::vector<MergedHop> merge_hops(const std::vector<HopIn>& hops, int spin) {
  std::vector<MergedHop> out;
  std::map<std::pair<int, int>, size_t> where;
  for (const auto& h : hops) {
    if (h.spin != spin) continue;
    const auto key = std::make_pair(h.from, h.to);
    auto it = where.find(key);
    if (it == where.end()) {
      where[key] = out.size();
      MergedHop m{};
      m.from = h.from;
      m.to = h.to;
      m.cre = h.cre;
      m.cim = h.cim;
      out.push_back(m);
    } else {
      out[it->second].cre += h.cre;
      out[it->second].cim += h.cim;
    }
  }
  for (auto& m : out) {
    m.lo = std::min(m.from, m.to);
    m.hi = std::max(m.from, m.to);
    m.own_mask = range_mask(m.lo + 1, m.hi);
    // up hop: other species (down) counted on [lo, hi); down hop: up counted on (lo, hi].
    m.other_mask = (spin == 0) ? range_mask(m.lo, m.hi) : range_mask(m.lo + 1, m.hi + 1);
  }
  return out;
}

// Orders the down-hop entries of one quarter-warp (8 lanes) into rounds so that in every round
// the 8 lanes read 8 different shared-memory bank groups: an entry's group is src % 8 (16-byte
// elements).  Edge-colouring of the bipartite multigraph lanes x groups with Delta colours
// (Konig's theorem; alternating-path recolouring), Delta = max lane or group degree.  A lane idle
// in a round reads an element of a group that round leaves free, with a zero coefficient.
void schedule_quarter(const std::vector<uint32_t>* in, std::vector<uint32_t>* out, uint32_t pad_hop, int64_t Dd) {
  struct Edge {
    int lane, grp;
    uint32_t ent;
  };
  std::vector<Edge> edges;
  int degL[8] = {0}, degG[8] = {0};
  for (int l = 0; l < 8; ++l)
    for (uint32_t ent : in[l]) {
      const int g = static_cast<int>((ent >> 10) & 7u);
      edges.push_back(Edge{l, g, ent});
      ++degL[l];
      ++degG[g];
    }
  int D = 0;
  for (int i = 0; i < 8; ++i) D = std::max(D, std::max(degL[i], degG[i]));
  std::vector<int> atL(static_cast<size_t>(8 * std::max(D, 1)), -1), atG(static_cast<size_t>(8 * std::max(D, 1)), -1);
  auto L = [&](int l, int c) -> int& { return atL[static_cast<size_t>(l * D + c)]; };
  auto G = [&](int g, int c) -> int& { return atG[static_cast<size_t>(g * D + c)]; };
  std::vector<int> col(edges.size(), -1);
  for (size_t e = 0; e < edges.size(); ++e) {
    const int l = edges[e].lane, g = edges[e].grp;
    int a = 0, b = 0;
    while (L(l, a) != -1) ++a;  // free at the lane
    while (G(g, b) != -1) ++b;  // free at the group
    if (G(g, a) != -1) {
      // Swap colours a and b along the alternating path that leaves g on colour a.
      std::vector<int> path;
      bool at_group = true;
      int v = g, c = a;
      while (true) {
        const int ed = at_group ? G(v, c) : L(v, c);
        if (ed < 0) break;
        path.push_back(ed);
        v = at_group ? edges[static_cast<size_t>(ed)].lane : edges[static_cast<size_t>(ed)].grp;
        at_group = !at_group;
        c = (c == a) ? b : a;
      }
      for (int ed : path) {
        const Edge& E = edges[static_cast<size_t>(ed)];
        L(E.lane, col[static_cast<size_t>(ed)]) = -1;
        G(E.grp, col[static_cast<size_t>(ed)]) = -1;
      }
      for (int ed : path) {
        const Edge& E = edges[static_cast<size_t>(ed)];
        const int nc = (col[static_cast<size_t>(ed)] == a) ? b : a;
        col[static_cast<size_t>(ed)] = nc;
        L(E.lane, nc) = ed;
        G(E.grp, nc) = ed;
      }
    }
    col[e] = a;
    L(l, a) = static_cast<int>(e);
    G(g, a) = static_cast<int>(e);
  }
  for (int l = 0; l < 8; ++l) out[l].assign(static_cast<size_t>(D), 0u);
  for (int c = 0; c < D; ++c) {
    int free_groups[8], nf = 0;
    for (int g = 0; g < 8; ++g)
      if (G(g, c) < 0) free_groups[nf++] = g;
    int fi = 0;
    for (int l = 0; l < 8; ++l) {
      const int ed = L(l, c);
      if (ed >= 0) {
        out[l][static_cast<size_t>(c)] = edges[static_cast<size_t>(ed)].ent;
      } else {
        const int g = fi < nf ? free_groups[fi++] : 0;
        const uint32_t src = static_cast<uint32_t>(g < Dd ? g : 0);
        out[l][static_cast<size_t>(c)] = (src << 10) | pad_hop;
      }
    }
  }
}

// The gauge-basis gather table of one spin (see GaugeTable): per group of 32 output strings, the
// hops split into the real section (coefficient one of two register-held values) and the table
// section, each scheduled by schedule_quarter, then re-encoded with byte offsets and sentinels.
void build_gauge_table(const SpinSpace& sp, const std::vector<MergedHop>& hops, int n_sites, GaugeTable* out) {
  GaugeTable& G = *out;
  G = GaugeTable{};
  const int64_t D = sp.D;
  if (n_sites > 32 || D < 1 || D + 8 > (1 << 14)) return;
  const int nh = static_cast<int>(hops.size());
  if (nh >= 511) return;
  // class of each hop: 0/1 = real value real2[0/1], 2 + t = table entry t
  std::vector<int> cls(static_cast<size_t>(nh), 0);
  int nreal = 0;
  for (int h = 0; h < nh; ++h) {
    const MergedHop& m = hops[static_cast<size_t>(h)];
    int k = -1;
    if (m.cim == 0.0) {
      for (int i = 0; i < nreal; ++i)
        if (G.real2[i] == m.cre) k = i;
      if (k < 0 && nreal < 2) {
        G.real2[nreal] = m.cre;
        k = nreal++;
      }
    }
    if (k < 0) {
      k = 2 + static_cast<int>(G.tab.size() / 2);
      G.tab.push_back(m.cre);
      G.tab.push_back(m.cim);
    }
    cls[static_cast<size_t>(h)] = k;
  }
  if (nreal == 1) G.real2[1] = G.real2[0];
  if (G.tab.size() / 2 > 512) return;
  // XOR form of the real section: when the two real values share their low words and their high
  // words differ only in bits 18..31, the signed coefficient (-1)^s real2[cls] is real2[0] with
  // bits 18..31 of its high word flipped by the entry's own bits 18..31.
  {
    uint64_t b0, b1;
    std::memcpy(&b0, &G.real2[0], 8);
    std::memcpy(&b1, &G.real2[1], 8);
    G.xor_real = static_cast<uint32_t>(b0) == static_cast<uint32_t>(b1) &&
                 ((static_cast<uint32_t>(b0 >> 32) ^ static_cast<uint32_t>(b1 >> 32)) & 0x3FFFFu) == 0u;
    G.xor_d = static_cast<uint32_t>(b0 >> 32) ^ static_cast<uint32_t>(b1 >> 32);
  }
  // Phase form: find p from the first table value and one of the real values, then require every
  // table value to be reproduced exactly as real2[k] * (pc, +-ps).
  const size_t nt = G.tab.size() / 2;
  std::vector<uint32_t> tab_bits(nt, 0u);  // cls<<30 | conj<<27 per table entry in the phase form
  for (int k0 = 0; k0 < 2 && nt > 0 && !G.phase; ++k0) {
    const double a = G.real2[k0];
    if (a == 0.0) continue;
    const double pc = G.tab[0] / a, ps = G.tab[1] / a;
    bool all = true;
    for (size_t t = 0; t < nt && all; ++t) {
      bool found = false;
      for (int k = 0; k < 2 && !found; ++k)
        for (int cj = 0; cj < 2 && !found; ++cj)
          if (G.real2[k] * pc == G.tab[2 * t] && G.real2[k] * (cj ? -ps : ps) == G.tab[2 * t + 1]) {
            tab_bits[t] = (static_cast<uint32_t>(k) << 30) | (static_cast<uint32_t>(cj) << 27);
            found = true;
          }
      all = found;
    }
    if (all) {
      G.phase = true;
      G.pc = pc;
      G.ps = ps;
    }
  }
  auto sentinel = [D](uint32_t group) {
    return static_cast<uint32_t>(D + static_cast<int64_t>((group + 8u - static_cast<uint32_t>(D & 7)) & 7u)) << 4;
  };
  const uint32_t pad_hop = static_cast<uint32_t>(nh) << 1;
  // old-format entry (src<<10 | hop<<1 | s) -> section entry; pads become sentinels of their bank group
  auto encode = [&](uint32_t e) -> uint32_t {
    const uint32_t src = e >> 10, h = (e >> 1) & 511u, sg = e & 1u;
    if (static_cast<int>(h) == nh) return sentinel(src & 7u);
    const int k = cls[h];
    if (k < 2 && G.xor_real) return (src << 4) | (((k ? G.xor_d : 0u) ^ (sg << 31)) & 0xFFFC0000u);
    if (k < 2) return (src << 4) | (static_cast<uint32_t>(k) << 30) | (sg << 31);
    const uint32_t extra = G.phase ? tab_bits[static_cast<size_t>(k - 2)] : 0u;
    return (src << 4) | (static_cast<uint32_t>(k - 2) << 18) | extra | (sg << 31);
  };
  const int64_t ngroups = (D + 31) / 32;
  std::vector<std::vector<uint32_t>> lr(32), lt(32), sr(32), st(32);
  for (int64_t g = 0; g < ngroups; ++g) {
    for (int l = 0; l < 32; ++l) {
      lr[l].clear();
      lt[l].clear();
      const int64_t r = g * 32 + l;
      if (r >= D) continue;
      const uint32_t m2 = sp.masks[static_cast<size_t>(r)];
      for (int h = 0; h < nh; ++h) {
        const auto& hp = hops[static_cast<size_t>(h)];
        if (!((m2 >> hp.to) & 1u) || ((m2 >> hp.from) & 1u)) continue;
        const uint32_t m = m2 ^ (1u << hp.from) ^ (1u << hp.to);
        const int64_t src = sp.rank(m);
        if (src < 0) return;
        const uint32_t sg = static_cast<uint32_t>(popc(m & hp.own_mask) & 1);
        const uint32_t e = (static_cast<uint32_t>(src) << 10) | (static_cast<uint32_t>(h) << 1) | sg;
        (cls[static_cast<size_t>(h)] < 2 ? lr[l] : lt[l]).push_back(e);
      }
    }
    // Lane permutation of a full group: the rounds of a section are set by the worst quarter-warp,
    // max(its longest lane, its busiest bank group), so move strings between quarters to balance the
    // bank-group loads (local search over swaps, deterministic per group); lane L serves string
    // g*32 + perm[L].  The last, partial group keeps the identity.
    uint8_t perm[32];
    for (int l = 0; l < 32; ++l) perm[l] = static_cast<uint8_t>(l);
    if (g * 32 + 32 <= D) {
      int dl[2][32], dgp[2][32][8];
      for (int l = 0; l < 32; ++l)
        for (int sct = 0; sct < 2; ++sct) {
          const auto& lst = sct ? lt[l] : lr[l];
          dl[sct][l] = static_cast<int>(lst.size());
          for (int b = 0; b < 8; ++b) dgp[sct][l][b] = 0;
          for (uint32_t e : lst) ++dgp[sct][l][(e >> 10) & 7u];
        }
      auto cost = [&](const uint8_t* pm) {
        int tot = 0;
        for (int sct = 0; sct < 2; ++sct) {
          int dm = 0;
          for (int q = 0; q < 4; ++q) {
            int m = 0, gs[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int k = 0; k < 8; ++k) {
              const int l = pm[q * 8 + k];
              m = std::max(m, dl[sct][l]);
              for (int b = 0; b < 8; ++b) gs[b] += dgp[sct][l][b];
            }
            for (int b = 0; b < 8; ++b) m = std::max(m, gs[b]);
            dm = std::max(dm, m);
          }
          tot += dm;
        }
        return tot;
      };
      uint64_t st64 = 0x9E3779B97F4A7C15ull ^ static_cast<uint64_t>(g);
      auto rnd = [&st64]() {  // splitmix64
        uint64_t z = (st64 += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
      };
      int best = cost(perm);
      for (int it = 0; it < 1500; ++it) {
        const int a = static_cast<int>(rnd() % 32), b = static_cast<int>(rnd() % 32);
        if (a / 8 == b / 8) continue;
        std::swap(perm[a], perm[b]);
        const int c = cost(perm);
        if (c <= best)
          best = c;
        else
          std::swap(perm[a], perm[b]);
      }
      std::vector<std::vector<uint32_t>> tr(32), tt(32);
      for (int l = 0; l < 32; ++l) {
        tr[l].swap(lr[perm[l]]);
        tt[l].swap(lt[perm[l]]);
      }
      for (int l = 0; l < 32; ++l) {
        lr[l].swap(tr[l]);
        lt[l].swap(tt[l]);
      }
    }
    for (int l = 0; l < 32; ++l) G.perm.push_back(perm[l]);
    size_t KR = 0, KT = 0;
    for (int qw = 0; qw < 4; ++qw) {
      schedule_quarter(&lr[8 * qw], &sr[8 * qw], pad_hop, D);
      schedule_quarter(&lt[8 * qw], &st[8 * qw], pad_hop, D);
      KR = std::max(KR, sr[8 * qw].size());
      KT = std::max(KT, st[8 * qw].size());
    }
    // each section padded to whole 4-entry loads: the row pass runs one loop per section with no
    // per-entry section test, and skips the padding rounds of each section's last load
    const size_t KR0 = KR, KT0 = KT;
    KR = (KR + 3) / 4 * 4;
    KT = (KT + 3) / 4 * 4;
    const size_t K4 = KR + KT;
    const size_t off = G.ent.size();
    if (off + K4 * 32 > static_cast<size_t>(INT32_MAX) || KR0 > 0xFFFF || KT0 > 0x7FFF) return;
    G.grp.push_back(static_cast<int32_t>(off));
    G.grp.push_back(static_cast<int32_t>(KR));
    G.grp.push_back(static_cast<int32_t>(KT));
    G.grp.push_back(static_cast<int32_t>(KR0 | (KT0 << 16)));
    // round k of lane l at off + ((k / 4) * 32 + l) * 4 + k % 4: a lane loads 4 rounds with one
    // 16-byte load.  Rounds a quarter does not need, and the rounds that pad the group to a
    // multiple of 4: lane l reads the sentinel of bank group l % 8.
    G.ent.resize(off + K4 * 32);
    for (size_t k = 0; k < K4; ++k)
      for (int l = 0; l < 32; ++l) {
        uint32_t e = sentinel(static_cast<uint32_t>(l) & 7u);
        if (k < KR) {
          if (k < sr[l].size()) e = encode(sr[l][k]);
        } else if (k < KR + KT) {
          if (k - KR < st[l].size()) e = encode(st[l][k - KR]);
        }
        G.ent[off + ((k / 4) * 32 + static_cast<size_t>(l)) * 4 + k % 4] = e;
      }
  }
  // two all-sentinel loads after the last group: the row pass loads two ahead of use unconditionally
  G.ent.resize(G.ent.size() + 2 * 32 * 4, sentinel(0u));
  G.ok = true;
}

}  // namespace

uint64_t binom(int n, int k) {
  init_binom();
  if (n < 0 || k < 0 || k > n || n > 64) return 0;
  return g_binom[n][k];
}

void SpinSpace::build(int n_, int k_) {
  init_binom();
  n = n_;
  k = k_;
  masks.clear();
  masks.reserve(static_cast<size_t>(binom(n, k)));
  enumerate(n, k, 0, 0u, &masks);
  D = static_cast<int64_t>(masks.size());
}

int64_t SpinSpace::rank(uint32_t m) const {
  if (n < 32 && (m >> n) != 0) return -1;
  if (popc(m) != k) return -1;
  // colex rank of the bit-reversed set: sum_j C(q_j, j), q ascending, j = 1..k.
  uint64_t colex = 0;
  int j = 0;
  for (int q = 0; q < n; ++q) {
    const int p = n - 1 - q;
    if ((m >> p) & 1u) {
      ++j;
      colex += g_binom[q][j];
    }
  }
  return static_cast<int64_t>(binom(n, k) - 1 - colex);
}

void build_geometry(int Lx, int Ly, double t, double tp, double phix, double phiy, std::vector<HopIn>* hops,
                    std::vector<PairIn>* pairs) {
  hops->clear();
  pairs->clear();
  auto site = [Lx](int x, int y) { return y * Lx + x; };
  auto bond = [hops](int from, int to, std::complex<double> phase, double ts) {
    if (std::abs(ts) < 1e-15) return;
    const std::complex<double> cij = -ts * phase, cji = -ts * std::conj(phase);
    for (int s = 0; s < 2; ++s) {
      hops->push_back(HopIn{from, to, s, cij.real(), cij.imag()});
      hops->push_back(HopIn{to, from, s, cji.real(), cji.imag()});
    }
  };
  auto phase = [phix, phiy](int wx, int wy) {
    return std::polar(1.0, static_cast<double>(wx) * phix + static_cast<double>(wy) * phiy);
  };
  auto nn = [pairs](int a, int b) {
    if (a == b) return;
    if (a > b) std::swap(a, b);
    pairs->push_back(PairIn{a, b});
  };
  for (int y = 0; y < Ly; ++y) {
    for (int x = 0; x < Lx; ++x) {
      const int i = site(x, y);
      if (Lx > 1) {
        const bool w = x + 1 >= Lx;
        const int j = site(w ? 0 : x + 1, y);
        if (i != j) {
          nn(i, j);
          bond(i, j, phase(w ? 1 : 0, 0), t);
        }
      }
      if (Ly > 1) {
        const bool w = y + 1 >= Ly;
        const int j = site(x, w ? 0 : y + 1);
        if (i != j) {
          nn(i, j);
          bond(i, j, phase(0, w ? 1 : 0), t);
        }
      }
      static const int dd[4][2] = {{1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
      for (const auto& d : dd) {
        int nx = x + d[0], ny = y + d[1], wx = 0, wy = 0;
        if (nx >= Lx) {
          nx -= Lx;
          wx = 1;
        } else if (nx < 0) {
          nx += Lx;
          wx = -1;
        }
        if (ny >= Ly) {
          ny -= Ly;
          wy = 1;
        } else if (ny < 0) {
          ny += Ly;
          wy = -1;
        }
        const int j = site(nx, ny);
        if (i != j) bond(i, j, phase(wx, wy), tp);
      }
    }
  }
}

double plan_diag(const SectorPlan& p, int64_t ru, int64_t rd) {
  const uint32_t u = p.up.masks[static_cast<size_t>(ru)], d = p.dn.masks[static_cast<size_t>(rd)];
  const uint32_t* w = &p.wpl[static_cast<size_t>(ru) * 4];
  const int cross = popc(d & w[0]) + 2 * popc(d & w[1]) + 4 * popc(d & w[2]) + 8 * popc(d & w[3]);
  const int vcount = p.cnt_uu[static_cast<size_t>(ru)] + p.cnt_dd[static_cast<size_t>(rd)] + cross;
  return p.U * static_cast<double>(popc(u & d)) + p.V * static_cast<double>(vcount);
}

namespace {

// Packed up-hop list (see SectorPlan::up_pk): every merged up hop's coefficient must be one of two
// real values, or one of them times a single unit phase p or its conjugate, exactly.
void build_up_packed(SectorPlan* Pp) {
  SectorPlan& P = *Pp;
  P.up_pk_ok = false;
  P.up_pk.clear();
  if (P.up.D > (1 << 14) || P.n > 32) return;
  const int nh = static_cast<int>(P.hu.size());
  std::vector<uint32_t> hbits(static_cast<size_t>(nh), 0u);  // cls<<30 | phase<<29 | conj<<28
  int nreal = 0;
  for (int h = 0; h < nh && nreal <= 2; ++h) {
    const MergedHop& m = P.hu[static_cast<size_t>(h)];
    if (m.cim != 0.0) continue;
    int k = -1;
    for (int i = 0; i < nreal; ++i)
      if (P.up_real2[i] == m.cre) k = i;
    if (k < 0) {
      if (nreal == 2) return;
      P.up_real2[nreal] = m.cre;
      k = nreal++;
    }
    hbits[static_cast<size_t>(h)] = static_cast<uint32_t>(k) << 30;
  }
  if (nreal == 1) P.up_real2[1] = P.up_real2[0];
  // p from the first complex hop and one of the real values; every complex hop must then be
  // real2[k] * (pc, +-ps) exactly
  int first = -1;
  for (int h = 0; h < nh && first < 0; ++h)
    if (P.hu[static_cast<size_t>(h)].cim != 0.0) first = h;
  bool all = true;
  for (int k0 = 0; k0 < 2 && first >= 0; ++k0) {
    const double a = P.up_real2[k0];
    if (a == 0.0) continue;
    P.up_pc = P.hu[static_cast<size_t>(first)].cre / a;
    P.up_ps = P.hu[static_cast<size_t>(first)].cim / a;
    all = true;
    for (int h = 0; h < nh && all; ++h) {
      const MergedHop& m = P.hu[static_cast<size_t>(h)];
      if (m.cim == 0.0) continue;
      bool found = false;
      for (int k = 0; k < 2 && !found; ++k)
        for (int cj = 0; cj < 2 && !found; ++cj)
          if (P.up_real2[k] * P.up_pc == m.cre && P.up_real2[k] * (cj ? -P.up_ps : P.up_ps) == m.cim) {
            hbits[static_cast<size_t>(h)] = (static_cast<uint32_t>(k) << 30) | (1u << 29) | (static_cast<uint32_t>(cj) << 28);
            found = true;
          }
      all = found;
    }
    if (all) break;
  }
  if (!all) return;
  P.up_pk.reserve(P.up_src.size());
  for (int64_t r = 0; r < P.up.D; ++r) {
    const uint32_t u2 = P.up.masks[static_cast<size_t>(r)];
    for (int h = 0; h < nh; ++h) {  // the CSR builder's order
      const MergedHop& m = P.hu[static_cast<size_t>(h)];
      if (!((u2 >> m.to) & 1u) || ((u2 >> m.from) & 1u)) continue;
      const uint32_t u = u2 ^ (1u << m.from) ^ (1u << m.to);
      const uint32_t src = static_cast<uint32_t>(P.up.rank(u));
      const uint32_t sg = static_cast<uint32_t>(popc(u & m.own_mask) & 1);
      P.up_pk.push_back(src | (static_cast<uint32_t>(m.lo) << 14) | (static_cast<uint32_t>(m.hi) << 19) |
                        hbits[static_cast<size_t>(h)] | (sg << 31));
    }
  }
  P.up_pk_ok = P.up_pk.size() == P.up_src.size();
  if (!P.up_pk_ok) P.up_pk.clear();
}

}  // namespace

std::string build_plan(int n_sites, int n_up, int n_dn, double U, double V, const std::vector<HopIn>& hops,
                       const std::vector<PairIn>& pairs, SectorPlan* out) {
  init_binom();
  if (n_sites <= 0 || n_sites > 32) return "FockBasis: require 1 <= n_sites <= 32 (bit packing)";
  if (n_up < 0 || n_dn < 0 || n_up > n_sites || n_dn > n_sites) return "FockBasis: particle numbers out of range";
  for (const auto& h : hops) {
    if (h.from < 0 || h.to < 0 || h.from >= n_sites || h.to >= n_sites || (h.spin != 0 && h.spin != 1))
      return "hopping out of range";
    if (h.from == h.to) return "on-site hopping entries are not supported";
  }
  for (const auto& pr : pairs)
    if (pr.i < 0 || pr.j < 0 || pr.i >= n_sites || pr.j >= n_sites) return "nn pair out of range";
  const uint64_t Du = binom(n_sites, n_up), Dd = binom(n_sites, n_dn);
  if (Du > (1u << 22) || Dd > (1u << 22)) return "spin space larger than 2^22 strings is not supported";
  if (Du * Dd >= (1ull << 31)) return "sector dimension must fit the reference's int index (< 2^31)";

  SectorPlan& P = *out;
  P = SectorPlan{};
  P.n = n_sites;
  P.nu = n_up;
  P.nd = n_dn;
  P.U = U;
  P.V = V;
  P.pairs = pairs;
  P.up.build(n_sites, n_up);
  P.dn.build(n_sites, n_dn);
  P.dim = P.up.D * P.dn.D;
  P.hu = merge_hops(hops, 0);
  P.hd = merge_hops(hops, 1);
  if (P.hd.size() + 1 > 256) return "more than 255 distinct down hoppings are not supported";

  // Diagonal tables.  sum_pairs (u_i+d_i)(u_j+d_j) = uu + dd + sum_s d_s * c_u(s).
  P.cnt_uu.resize(static_cast<size_t>(P.up.D));
  P.cnt_dd.resize(static_cast<size_t>(P.dn.D));
  P.wpl.assign(static_cast<size_t>(P.up.D) * 4, 0u);
  for (int64_t r = 0; r < P.up.D; ++r) {
    const uint32_t u = P.up.masks[static_cast<size_t>(r)];
    int uu = 0;
    int cu[32] = {0};
    for (const auto& pr : pairs) {
      const int ui = (u >> pr.i) & 1u, uj = (u >> pr.j) & 1u;
      uu += ui * uj;
      cu[pr.i] += uj;
      cu[pr.j] += ui;
    }
    P.cnt_uu[static_cast<size_t>(r)] = uu;
    for (int s = 0; s < n_sites; ++s) {
      if (cu[s] > 15) return "more than 15 nn pairs on one site are not supported";
      for (int b = 0; b < 4; ++b)
        if ((cu[s] >> b) & 1) P.wpl[static_cast<size_t>(r) * 4 + b] |= (1u << s);
    }
  }
  for (int64_t r = 0; r < P.dn.D; ++r) {
    const uint32_t d = P.dn.masks[static_cast<size_t>(r)];
    int dd = 0;
    for (const auto& pr : pairs) dd += static_cast<int>(((d >> pr.i) & 1u) * ((d >> pr.j) & 1u));
    P.cnt_dd[static_cast<size_t>(r)] = dd;
  }

  // Up part: for output up string u', hop f->t contributes from source u = u' ^ f ^ t when
  // u' has t and not f; the up-string factor (-1)^#up(lo,hi) is the same on u and u'.
  P.up_ptr.assign(static_cast<size_t>(P.up.D) + 1, 0);
  for (int64_t r = 0; r < P.up.D; ++r) {
    const uint32_t u2 = P.up.masks[static_cast<size_t>(r)];
    int deg = 0;
    for (const auto& h : P.hu) {
      if (!((u2 >> h.to) & 1u) || ((u2 >> h.from) & 1u)) continue;
      const uint32_t u = u2 ^ (1u << h.from) ^ (1u << h.to);
      const int64_t src = P.up.rank(u);
      if (src < 0) return "internal: up source rank";
      const double sg = (popc(u & h.own_mask) & 1) ? -1.0 : 1.0;
      P.up_src.push_back(static_cast<int32_t>(src));
      P.up_coef.push_back(sg * h.cre);
      P.up_coef.push_back(sg * h.cim);
      P.up_lohi.push_back(static_cast<uint32_t>(h.lo) | (static_cast<uint32_t>(h.hi) << 8));
      ++deg;
    }
    P.max_up_deg = std::max(P.max_up_deg, deg);
    P.up_ptr[static_cast<size_t>(r) + 1] = static_cast<int32_t>(P.up_src.size());
  }
  P.mean_up_sources = P.up.D ? static_cast<double>(P.up_src.size()) / static_cast<double>(P.up.D) : 0.0;
  build_up_packed(&P);

  // Down part: per output down string d', hop f->t contributes from d = d' ^ f ^ t; the
  // down-string factor (-1)^#dn(lo,hi) goes into the entry, the up-string factor per row.
  const int nh = static_cast<int>(P.hd.size());
  P.dn_pad_hop = nh;
  P.dn_coef.assign(static_cast<size_t>(nh + 1) * 2, 0.0);
  P.dn_nmask.assign(static_cast<size_t>(nh + 1), 0u);
  for (int h = 0; h < nh; ++h) {
    P.dn_coef[2 * h] = P.hd[h].cre;
    P.dn_coef[2 * h + 1] = P.hd[h].cim;
    P.dn_nmask[h] = P.hd[h].other_mask;
  }
  const int64_t ngroups = (P.dn.D + 31) / 32;
  P.dn_gptr.assign(static_cast<size_t>(ngroups) + 1, 0);
  P.dn_csr_ptr.assign(static_cast<size_t>(P.dn.D) + 1, 0);
  std::vector<std::vector<uint32_t>> lane(32);
  std::vector<std::vector<uint32_t>> sched(32);
  int64_t total_src = 0;
  const uint32_t pad_hop = static_cast<uint32_t>(P.dn_pad_hop) << 1;
  for (int64_t g = 0; g < ngroups; ++g) {
    for (int l = 0; l < 32; ++l) {
      lane[l].clear();
      const int64_t r = g * 32 + l;
      if (r >= P.dn.D) continue;
      const uint32_t d2 = P.dn.masks[static_cast<size_t>(r)];
      for (int h = 0; h < nh; ++h) {
        const auto& hp = P.hd[h];
        if (!((d2 >> hp.to) & 1u) || ((d2 >> hp.from) & 1u)) continue;
        const uint32_t d = d2 ^ (1u << hp.from) ^ (1u << hp.to);
        const int64_t src = P.dn.rank(d);
        if (src < 0) return "internal: down source rank";
        const uint32_t sg = static_cast<uint32_t>(popc(d & hp.own_mask) & 1);
        lane[l].push_back((static_cast<uint32_t>(src) << 10) | (static_cast<uint32_t>(h) << 1) | sg);
      }
      total_src += static_cast<int64_t>(lane[l].size());
      P.max_dn_deg = std::max(P.max_dn_deg, static_cast<int>(lane[l].size()));
      for (uint32_t en : lane[l]) P.dn_csr_ent.push_back(((en >> 10) << 9) | (((en >> 1) & 511u) << 1) | (en & 1u));
      while ((P.dn_csr_ent.size() - static_cast<size_t>(P.dn_csr_ptr[static_cast<size_t>(r)])) % 8 != 0)
        P.dn_csr_ent.push_back((static_cast<uint32_t>(r) << 9) | (static_cast<uint32_t>(P.dn_pad_hop) << 1));
      P.dn_csr_ptr[static_cast<size_t>(r) + 1] = static_cast<int64_t>(P.dn_csr_ent.size());
    }
    // Per quarter-warp (8 lanes), order the entries so that in every round the 8 lanes read
    // 8 different shared-memory bank groups (a 16-byte element src sits in group src % 8).
    size_t K = 0;
    for (int qw = 0; qw < 4; ++qw) {
      schedule_quarter(&lane[8 * qw], &sched[8 * qw], pad_hop, P.dn.D);
      K = std::max(K, sched[8 * qw].size());
    }
    for (int l = 0; l < 32; ++l) {
      // Rounds a quarter does not need: every lane reads its own element (distinct groups).
      const int64_t r = g * 32 + l;
      const uint32_t self = static_cast<uint32_t>(r < P.dn.D ? r : std::min<int64_t>(l & 7, P.dn.D - 1));
      while (sched[l].size() < K) sched[l].push_back((self << 10) | pad_hop);
    }
    for (size_t k = 0; k < K; ++k)
      for (int l = 0; l < 32; ++l) P.dn_ent.push_back(sched[l][k]);
    P.dn_gptr[static_cast<size_t>(g) + 1] = static_cast<int64_t>(P.dn_ent.size());
  }
  P.mean_dn_sources = P.dn.D ? static_cast<double>(total_src) / static_cast<double>(P.dn.D) : 0.0;
  build_gauge_table(P.dn, P.hd, P.n, &P.dn_g);
  return "";
}

}  // namespace ftlm_b200
