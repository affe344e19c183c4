// A caller of the reference's orbit k-block API (include/ftlm/symmetry/orbit_k_block_basis.hpp),
// compiled against the C++ drop-in by tests/test_gpu_orbit_dropin.py.
//   dropin_orbit facts          the facts tests/test_orbit_k_block_basis.cpp checks
//   dropin_orbit apply Lx Ly t tp U V nu nd kx ky x.bin out.bin
//       writes dk, then per row: packed rep (u32), |A|, orbit size (i32), orbit index (i64), then y.
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ftlm/fock_basis.hpp"
#include "ftlm/hubbard_params.hpp"
#include "ftlm/lattice.hpp"
#include "ftlm/symmetry/orbit_k_block_basis.hpp"

using namespace ftlm;
using namespace ftlm::symmetry;

static int facts() {
  FockBasis fb(4, 2, 2);
  OrbitKBlockBasis b0;
  b0.build(fb, MomentumSector{0, 0, 2, 2});
  if (b0.dim() != 12) return 2;
  std::size_t sum_sizes = 0;
  for (const auto& e : b0.entries()) {
    sum_sizes += e.orbit_size;
    if (std::abs(e.abs_A - e.stabilizer_size) > 1e-9 * (1.0 + e.abs_A)) return 3;
  }
  int mapped = 0;
  for (int i = 0; i < fb.dim(); ++i) {
    const RawState s{static_cast<std::uint16_t>(fb.up_mask(i)), static_cast<std::uint16_t>(fb.down_mask(i))};
    int ri = 0, dx = 0, dy = 0;
    double eta = 0.0;
    if (!b0.map_raw_to_rep(s, &ri, &dx, &dy, &eta)) continue;
    ++mapped;
    const RawState r = b0.entries()[static_cast<std::size_t>(ri)].rep;
    if (r == s && (dx != 0 || dy != 0 || eta != 1.0)) return 4;
  }
  if (static_cast<std::size_t>(mapped) != sum_sizes) return 5;
  FockBasis fb32(6, 3, 3);
  OrbitKBlockBasis b32;
  b32.build(fb32, MomentumSector{1, 0, 3, 2});
  if (b32.dim() != 66) return 6;
  std::printf("ok orbit dims %d %d\n", b0.dim(), b32.dim());
  return 0;
}

int main(int argc, char** argv) {
  if (argc >= 2 && std::strcmp(argv[1], "facts") == 0) return facts();
  if (argc != 14 || std::strcmp(argv[1], "apply") != 0) return 1;
  HubbardParams p;
  p.Lx = std::atoi(argv[2]);
  p.Ly = std::atoi(argv[3]);
  p.t = std::atof(argv[4]);
  p.tp = std::atof(argv[5]);
  p.U = std::atof(argv[6]);
  p.V = std::atof(argv[7]);
  const int nu = std::atoi(argv[8]), nd = std::atoi(argv[9]);
  const MomentumSector K{std::atoi(argv[10]), std::atoi(argv[11]), p.Lx, p.Ly};
  FockBasis fb(p.Lx * p.Ly, nu, nd);
  RectLattice lat;
  lat.Lx = p.Lx;
  lat.Ly = p.Ly;
  std::vector<SpinfulHopping> hops;
  std::vector<NearestPair> pairs;
  build_hubbard_geometry(p, lat, &hops, &pairs);
  OrbitKBlockBasis basis;
  basis.build(fb, K);
  const int dk = basis.dim();
  std::vector<std::complex<double>> x(static_cast<std::size_t>(dk)), y(static_cast<std::size_t>(dk));
  FILE* f = std::fopen(argv[12], "rb");
  if (!f || std::fread(x.data(), sizeof(x[0]), x.size(), f) != x.size()) return 7;
  std::fclose(f);
  apply_orbit_k_block(p, fb, basis, hops, pairs, x.data(), y.data());
  apply_orbit_k_block(p, fb, basis, hops, pairs, x.data(), y.data());  // second call: cached device tables
  FILE* g = std::fopen(argv[13], "wb");
  if (!g) return 8;
  std::fwrite(&dk, sizeof(dk), 1, g);
  for (const auto& e : basis.entries()) {
    const std::uint32_t pk = pack_raw_state(e.rep);
    const int os = e.orbit_size;
    const long long oi = static_cast<long long>(e.orbit_index);
    std::fwrite(&pk, sizeof(pk), 1, g);
    std::fwrite(&e.abs_A, sizeof(double), 1, g);
    std::fwrite(&os, sizeof(os), 1, g);
    std::fwrite(&oi, sizeof(oi), 1, g);
  }
  std::fwrite(y.data(), sizeof(y[0]), y.size(), g);
  std::fclose(g);
  return 0;
}
