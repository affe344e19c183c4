// C ABI (include/ftlm_gpu.h): sector handles, H·v, Lanczos, quadrature, grand-canonical sweep.
// Host orchestration only; every floating-point operation on sector vectors runs in the
// kernels of hv.cu / lanczos.cu / quad.cu.  No exception crosses the ABI.  The batched path,
// the parameter gradient and the momentum blocks are in capi_batched.cu, capi_grad.cu and
// capi_orbit.cu.
#include <map>
#include <thread>

#include <atomic>

#include "capi_internal.hpp"
#include "chains.cuh"

using namespace ftlm_b200;
using namespace ftlm_b200::capi;

// Quadrature of the complex128 sector path (ftlm_gpu_set_quadrature).
static std::atomic<bool> g_quad_converged{false};

namespace {
thread_local std::string g_err;
}  // namespace

int ftlm_b200::capi::fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int ftlm_b200::set_error(int code, const char* msg) { return fail(code, msg); }

namespace ftlm_b200 {
namespace capi {

void reference_start(int64_t dim, unsigned seed, std::vector<std::complex<double>>* q) {
  std::mt19937 rng(seed);
  std::normal_distribution<double> gauss(0.0, 1.0);
  q->resize(static_cast<size_t>(dim));
  auto& v = *q;
  for (int64_t i = 0; i < dim; ++i) {
    const double re = gauss(rng);
    const double im = gauss(rng);
    v[static_cast<size_t>(i)] = {re, im};
  }
  double n0 = 0.0;
  for (const auto& z : v) n0 += std::norm(z);
  n0 = std::sqrt(n0);
  if (n0 < 1e-18) {
    std::fill(v.begin(), v.end(), std::complex<double>(0.0, 0.0));
    v[0] = {1.0, 0.0};
  } else {
    const std::complex<double> sc(1.0 / n0, 0.0);
    for (auto& z : v) z *= sc;
  }
}

// Device Lanczos workspace.
}  // namespace capi
}  // namespace ftlm_b200

namespace {

int upload_plan(ftlm_sector* s) {
  const SectorPlan& P = s->plan;
  DevSector& D = s->dev;
  CU_TRY(cudaGetDevice(&s->device));
  D.n = P.n;
  D.Du = P.up.D;
  D.Dd = P.dn.D;
  D.dim = P.dim;
  D.U = P.U;
  D.V = P.V;
  std::vector<uint4> w4(static_cast<size_t>(P.up.D));
  for (size_t i = 0; i < w4.size(); ++i) w4[i] = make_uint4(P.wpl[4 * i], P.wpl[4 * i + 1], P.wpl[4 * i + 2], P.wpl[4 * i + 3]);
  std::vector<double2> upc(P.up_src.size()), dnc(P.dn_coef.size() / 2);
  std::vector<float2> upc32(upc.size()), dnc32(dnc.size());
  for (size_t i = 0; i < upc.size(); ++i) {
    upc[i] = make_double2(P.up_coef[2 * i], P.up_coef[2 * i + 1]);
    upc32[i] = make_float2(static_cast<float>(upc[i].x), static_cast<float>(upc[i].y));
  }
  for (size_t i = 0; i < dnc.size(); ++i) {
    dnc[i] = make_double2(P.dn_coef[2 * i], P.dn_coef[2 * i + 1]);
    dnc32[i] = make_float2(static_cast<float>(dnc[i].x), static_cast<float>(dnc[i].y));
  }
  std::vector<float2> dnc32s(2 * dnc32.size());
  for (size_t i = 0; i < dnc32.size(); ++i) {
    dnc32s[2 * i] = dnc32[i];
    dnc32s[2 * i + 1] = make_float2(-dnc32[i].x, -dnc32[i].y);
  }
  float2 *ucf32, *dcf32, *dcf32s;
  CU_TRY(upload(upc32, &ucf32, &s->owned));
  CU_TRY(upload(dnc32, &dcf32, &s->owned));
  CU_TRY(upload(dnc32s, &dcf32s, &s->owned));
  uint32_t *um, *dm, *ulh, *dent, *dnm;
  int32_t *cuu, *cdd, *uptr, *usrc;
  uint4* wp;
  double2 *ucf, *dcf;
  int64_t* gptr;
  int64_t* cptr;
  uint32_t* cent;
  CU_TRY(upload(P.dn_csr_ptr, &cptr, &s->owned));
  CU_TRY(upload(P.dn_csr_ent, &cent, &s->owned));
  CU_TRY(upload(P.up.masks, &um, &s->owned));
  CU_TRY(upload(P.dn.masks, &dm, &s->owned));
  CU_TRY(upload(P.cnt_uu, &cuu, &s->owned));
  CU_TRY(upload(P.cnt_dd, &cdd, &s->owned));
  CU_TRY(upload(w4, &wp, &s->owned));
  CU_TRY(upload(P.up_ptr, &uptr, &s->owned));
  CU_TRY(upload(P.up_src, &usrc, &s->owned));
  CU_TRY(upload(upc, &ucf, &s->owned));
  CU_TRY(upload(P.up_lohi, &ulh, &s->owned));
  CU_TRY(upload(P.dn_gptr, &gptr, &s->owned));
  CU_TRY(upload(P.dn_ent, &dent, &s->owned));
  CU_TRY(upload(dnc, &dcf, &s->owned));
  CU_TRY(upload(P.dn_nmask, &dnm, &s->owned));
  std::vector<int> flags(4, 0);
  int* fl;
  CU_TRY(upload(flags, &fl, &s->owned));
  D.bt_cols = 1;  // 8-column chunks: the fastest at 4x4 (4,4), (6,6), (8,8) (ftlm_gpu_batched_autotune)
  auto upload_gauge = [&](const GaugeTable& G, DevGauge* out) -> cudaError_t {
    *out = DevGauge{};
    out->real2[0] = G.real2[0];
    out->real2[1] = G.real2[1];
    if (!G.ok) return cudaSuccess;
    uint32_t* ge;
    int32_t* gg;
    cudaError_t e = upload(G.ent, &ge, &s->owned);
    if (e == cudaSuccess) e = upload(G.grp, &gg, &s->owned);
    if (e != cudaSuccess) return e;
    out->ent = ge;
    out->grp = reinterpret_cast<const int4*>(gg);
    uint8_t* gp;
    if ((e = upload(G.perm, &gp, &s->owned)) != cudaSuccess) return e;
    out->perm = gp;
    out->nt = static_cast<int>(G.tab.size() / 2);
    out->phase = G.phase ? 1 : 0;
    out->xor_real = G.xor_real ? 1 : 0;
    out->pc = G.pc;
    out->ps = G.ps;
    if (out->nt > 0) {
      double* gt;
      if ((e = upload(G.tab, &gt, &s->owned)) != cudaSuccess) return e;
      out->tab = reinterpret_cast<const double2*>(gt);
    }
    return cudaSuccess;
  };
  CU_TRY(upload_gauge(P.dn_g, &D.dn_g));
  D.up_pk = nullptr;
  D.up_real2[0] = P.up_real2[0];
  D.up_real2[1] = P.up_real2[1];
  D.up_pc = P.up_pc;
  D.up_ps = P.up_ps;
  if (P.up_pk_ok) {
    uint32_t* upk;
    CU_TRY(upload(P.up_pk, &upk, &s->owned));
    D.up_pk = upk;
  }
  D.umask = um;
  D.dmask = dm;
  D.cnt_uu = cuu;
  D.cnt_dd = cdd;
  D.wpl = wp;
  D.up_ptr = uptr;
  D.up_src = usrc;
  D.up_coef = ucf;
  D.up_lohi = ulh;
  D.dn_gptr = gptr;
  D.dn_ent = dent;
  D.dn_csr_ptr = cptr;
  D.up_coef32 = ucf32;
  D.dn_coef32 = dcf32;
  D.dn_coef32s = dcf32s;
  D.dn_csr_ent = cent;
  D.dn_coef = dcf;
  D.dn_nmask = dnm;
  D.n_dn_hops = P.dn_pad_hop;
  D.flags = fl;
  CU_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  s->on_device = true;
  return FTLM_OK;
}

int create_common(int n_sites, int n_up, int n_dn, double U, double V, const ftlm_hop* hops, int n_hops,
                  const ftlm_pair* pairs, int n_pairs, bool device, ftlm_sector** out) {
  if (!out) return fail(FTLM_ERR_INVALID, "null output handle");
  *out = nullptr;
  if (n_hops < 0 || n_pairs < 0 || (n_hops > 0 && !hops) || (n_pairs > 0 && !pairs))
    return fail(FTLM_ERR_INVALID, "bad hopping/pair arrays");
  std::vector<HopIn> hv(static_cast<size_t>(n_hops));
  for (int i = 0; i < n_hops; ++i) hv[i] = HopIn{hops[i].from, hops[i].to, hops[i].spin, hops[i].coeff_re, hops[i].coeff_im};
  std::vector<PairIn> pv(static_cast<size_t>(n_pairs));
  for (int i = 0; i < n_pairs; ++i) pv[i] = PairIn{pairs[i].i, pairs[i].j};
  auto* s = new (std::nothrow) ftlm_sector();
  if (!s) return fail(FTLM_ERR_NOMEM, "host allocation failed");
  std::string err;
  try {
    err = build_plan(n_sites, n_up, n_dn, U, V, hv, pv, &s->plan);
  } catch (const std::bad_alloc&) {
    delete s;
    return fail(FTLM_ERR_NOMEM, "host allocation failed while building the sector plan");
  }
  if (!err.empty()) {
    delete s;
    const bool unsup = err.find("not supported") != std::string::npos || err.find("2^31") != std::string::npos;
    return fail(unsup ? FTLM_ERR_UNSUPPORTED : FTLM_ERR_INVALID, err);
  }
  if (device) {
    const int rc = upload_plan(s);
    if (rc != FTLM_OK) {
      delete s;
      return rc;
    }
  }
  *out = s;
  return FTLM_OK;
}


}  // namespace

int ftlm_b200::capi::need_device(const ftlm_sector* s) {
  if (!s) return fail(FTLM_ERR_INVALID, "null sector");
  if (!s->on_device) return fail(FTLM_ERR_INVALID, "sector was created host-only");
  return FTLM_OK;
}

extern "C" {

const char* ftlm_gpu_last_error(void) { return g_err.c_str(); }

const char* ftlm_gpu_version_string(void) { return "ftlm_extended_hubbard_b200 0.1.0 (sm_100a)"; }

int ftlm_gpu_device_count(int* n) {
  if (!n) return fail(FTLM_ERR_INVALID, "null");
  *n = 0;
  const cudaError_t e = cudaGetDeviceCount(n);
  if (e != cudaSuccess) {
    *n = 0;
    return fail(FTLM_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  }
  return FTLM_OK;
}

int ftlm_gpu_build_geometry(const ftlm_params* p, ftlm_hop* hops, int max_hops, int* n_hops, ftlm_pair* pairs,
                            int max_pairs, int* n_pairs) {
  if (!p || !n_hops || !n_pairs) return fail(FTLM_ERR_INVALID, "null argument");
  if (p->Lx <= 0 || p->Ly <= 0) return fail(FTLM_ERR_INVALID, "Lx, Ly must be positive");
  std::vector<HopIn> hv;
  std::vector<PairIn> pv;
  build_geometry(p->Lx, p->Ly, p->t, p->tp, p->phi_x, p->phi_y, &hv, &pv);
  *n_hops = static_cast<int>(hv.size());
  *n_pairs = static_cast<int>(pv.size());
  for (int i = 0; i < *n_hops && i < max_hops && hops; ++i)
    hops[i] = ftlm_hop{hv[i].from, hv[i].to, hv[i].spin, hv[i].cre, hv[i].cim};
  for (int i = 0; i < *n_pairs && i < max_pairs && pairs; ++i) pairs[i] = ftlm_pair{pv[i].i, pv[i].j};
  return FTLM_OK;
}

int ftlm_gpu_sector_create_hops(int n_sites, int n_up, int n_dn, double U, double V, const ftlm_hop* hops, int n_hops,
                                const ftlm_pair* pairs, int n_pairs, ftlm_sector** out) {
  return create_common(n_sites, n_up, n_dn, U, V, hops, n_hops, pairs, n_pairs, true, out);
}

int ftlm_gpu_sector_create_host(int n_sites, int n_up, int n_dn, double U, double V, const ftlm_hop* hops, int n_hops,
                                const ftlm_pair* pairs, int n_pairs, ftlm_sector** out) {
  return create_common(n_sites, n_up, n_dn, U, V, hops, n_hops, pairs, n_pairs, false, out);
}

int ftlm_gpu_sector_create(const ftlm_params* p, int n_up, int n_dn, ftlm_sector** out) {
  if (!p) return fail(FTLM_ERR_INVALID, "null params");
  if (p->Lx <= 0 || p->Ly <= 0) return fail(FTLM_ERR_INVALID, "Lx, Ly must be positive");
  std::vector<HopIn> hv;
  std::vector<PairIn> pv;
  build_geometry(p->Lx, p->Ly, p->t, p->tp, p->phi_x, p->phi_y, &hv, &pv);
  std::vector<ftlm_hop> h(hv.size());
  for (size_t i = 0; i < hv.size(); ++i) h[i] = ftlm_hop{hv[i].from, hv[i].to, hv[i].spin, hv[i].cre, hv[i].cim};
  std::vector<ftlm_pair> q(pv.size());
  for (size_t i = 0; i < pv.size(); ++i) q[i] = ftlm_pair{pv[i].i, pv[i].j};
  const int rc = create_common(p->Lx * p->Ly, n_up, n_dn, p->U, p->V, h.data(), static_cast<int>(h.size()), q.data(),
                               static_cast<int>(q.size()), true, out);
  if (rc == FTLM_OK) {
    (*out)->Lx = p->Lx;
    (*out)->Ly = p->Ly;
  }
  return rc;
}

int ftlm_gpu_sector_destroy(ftlm_sector* s) {
  delete s;
  return FTLM_OK;
}

int ftlm_gpu_sector_dim(const ftlm_sector* s, long long* dim) {
  if (!s || !dim) return fail(FTLM_ERR_INVALID, "null argument");
  *dim = s->plan.dim;
  return FTLM_OK;
}

int ftlm_gpu_sector_masks(const ftlm_sector* s, uint64_t* up, uint64_t* dn) {
  if (!s || !up || !dn) return fail(FTLM_ERR_INVALID, "null argument");
  const auto& P = s->plan;
  for (int64_t r = 0; r < P.up.D; ++r)
    for (int64_t c = 0; c < P.dn.D; ++c) {
      up[r * P.dn.D + c] = P.up.masks[static_cast<size_t>(r)];
      dn[r * P.dn.D + c] = P.dn.masks[static_cast<size_t>(c)];
    }
  return FTLM_OK;
}

int ftlm_gpu_sector_index_of(const ftlm_sector* s, uint64_t up, uint64_t dn, long long* index) {
  if (!s || !index) return fail(FTLM_ERR_INVALID, "null argument");
  *index = -1;
  if ((up >> 32) != 0 || (dn >> 32) != 0) return FTLM_OK;
  const int64_t ru = s->plan.up.rank(static_cast<uint32_t>(up));
  const int64_t rd = s->plan.dn.rank(static_cast<uint32_t>(dn));
  if (ru >= 0 && rd >= 0) *index = ru * s->plan.dn.D + rd;
  return FTLM_OK;
}

int ftlm_gpu_sector_state(const ftlm_sector* s, long long index, uint64_t* up, uint64_t* dn) {
  if (!s || !up || !dn) return fail(FTLM_ERR_INVALID, "null argument");
  if (index < 0 || index >= s->plan.dim) return fail(FTLM_ERR_INVALID, "FockBasis index out of range");
  *up = s->plan.up.masks[static_cast<size_t>(index / s->plan.dn.D)];
  *dn = s->plan.dn.masks[static_cast<size_t>(index % s->plan.dn.D)];
  return FTLM_OK;
}

int ftlm_gpu_sector_down_table_gauge(const ftlm_sector* s, int* available, long long* n_groups, long long* n_entries,
                                     int* n_table, int* groups, uint32_t* entries, double* table, double* real2) {
  if (!s || !available || !n_groups || !n_entries || !n_table) return fail(FTLM_ERR_INVALID, "null argument");
  const GaugeTable& G = s->plan.dn_g;
  *available = G.ok ? 1 : 0;
  *n_groups = G.ok ? static_cast<long long>(G.grp.size() / 4) : 0;
  *n_entries = G.ok ? static_cast<long long>(G.ent.size()) : 0;
  *n_table = G.ok ? static_cast<int>(G.tab.size() / 2) : 0;
  if (!G.ok) return FTLM_OK;
  if (groups) std::copy(G.grp.begin(), G.grp.end(), groups);
  if (entries) std::copy(G.ent.begin(), G.ent.end(), entries);
  if (table) std::copy(G.tab.begin(), G.tab.end(), table);
  if (real2) std::copy(G.real2, G.real2 + 2, real2);
  return FTLM_OK;
}

int ftlm_gpu_sector_down_table_form(const ftlm_sector* s, int* phase, double* pc_ps, int* xor_real,
                                    unsigned char* lane_perm) {
  if (!s || !phase) return fail(FTLM_ERR_INVALID, "null argument");
  const GaugeTable& G = s->plan.dn_g;
  *phase = (G.ok && G.phase) ? 1 : 0;
  if (xor_real) *xor_real = (G.ok && G.xor_real) ? 1 : 0;
  if (lane_perm && G.ok) std::copy(G.perm.begin(), G.perm.end(), lane_perm);
  if (pc_ps) {
    pc_ps[0] = G.pc;
    pc_ps[1] = G.ps;
  }
  return FTLM_OK;
}

int ftlm_gpu_sector_up_table_packed(const ftlm_sector* s, int* available, long long* n_entries, int32_t* ptr,
                                    uint32_t* entries, double* real2, double* pc_ps) {
  if (!s || !available || !n_entries) return fail(FTLM_ERR_INVALID, "null argument");
  const SectorPlan& P = s->plan;
  *available = P.up_pk_ok ? 1 : 0;
  *n_entries = P.up_pk_ok ? static_cast<long long>(P.up_pk.size()) : 0;
  if (!P.up_pk_ok) return FTLM_OK;
  if (ptr) std::copy(P.up_ptr.begin(), P.up_ptr.end(), ptr);
  if (entries) std::copy(P.up_pk.begin(), P.up_pk.end(), entries);
  if (real2) std::copy(P.up_real2, P.up_real2 + 2, real2);
  if (pc_ps) {
    pc_ps[0] = P.up_pc;
    pc_ps[1] = P.up_ps;
  }
  return FTLM_OK;
}

int ftlm_gpu_sector_stats(const ftlm_sector* s, double* mean_up, double* mean_dn, long long* du, long long* dd) {
  if (!s) return fail(FTLM_ERR_INVALID, "null sector");
  if (mean_up) *mean_up = s->plan.mean_up_sources;
  if (mean_dn) *mean_dn = s->plan.mean_dn_sources;
  if (du) *du = s->plan.up.D;
  if (dd) *dd = s->plan.dn.D;
  return FTLM_OK;
}

int ftlm_gpu_sector_down_table(const ftlm_sector* s, long long* n_groups, long long* n_entries, long long* gptr,
                               uint32_t* entries, int* pad_hop) {
  if (!s || !n_groups || !n_entries) return fail(FTLM_ERR_INVALID, "null argument");
  *n_groups = static_cast<long long>(s->plan.dn_gptr.size()) - 1;
  *n_entries = static_cast<long long>(s->plan.dn_ent.size());
  if (gptr) std::copy(s->plan.dn_gptr.begin(), s->plan.dn_gptr.end(), gptr);
  if (entries) std::copy(s->plan.dn_ent.begin(), s->plan.dn_ent.end(), entries);
  if (pad_hop) *pad_hop = s->plan.dn_pad_hop;
  return FTLM_OK;
}

int ftlm_gpu_sector_diag(const ftlm_sector* s, long long index, double* value) {
  if (!s || !value) return fail(FTLM_ERR_INVALID, "null argument");
  if (index < 0 || index >= s->plan.dim) return fail(FTLM_ERR_INVALID, "index out of range");
  *value = plan_diag(s->plan, index / s->plan.dn.D, index % s->plan.dn.D);
  return FTLM_OK;
}

int ftlm_gpu_set_apply_path(ftlm_sector* s, int path) {
  if (!s || path < 0 || path > 3) return fail(FTLM_ERR_INVALID, "bad path");
  s->apply_path = path;
  return FTLM_OK;
}

int ftlm_gpu_apply(ftlm_sector* s, const double* x, double* y, void* stream) {
  int rc = need_device(s);
  if (rc) return rc;
  if (!x || !y) return fail(FTLM_ERR_INVALID, "null vector");
  if (x == y) return fail(FTLM_ERR_INVALID, "x and y must not alias");
  return s->apply(reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y), static_cast<cudaStream_t>(stream));
}

int ftlm_gpu_apply_profiled(ftlm_sector* s, const double* x, double* y, void* stream, float* ms_passes, int* n_passes) {
  int rc = need_device(s);
  if (rc) return rc;
  if (!x || !y || !ms_passes || !n_passes) return fail(FTLM_ERR_INVALID, "null argument");
  if (x == y) return fail(FTLM_ERR_INVALID, "x and y must not alias");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int path = s->effective_path();
  const DevSector d = s->dev_for(path);
  cudaEvent_t ev[3];
  for (auto& e : ev) CU_TRY(cudaEventCreate(&e));
  CU_TRY(cudaEventRecord(ev[0], st));
  if (path >= 2) {
    CU_TRY(hv_launch_pass(d, reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y), 0, st,
                          s->cols_variant));
    CU_TRY(cudaEventRecord(ev[1], st));
    CU_TRY(hv_launch_pass(d, reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y), 1, st,
                          s->cols_variant));
  } else {
    CU_TRY(hv_launch(d, reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y), path, st));
    CU_TRY(cudaEventRecord(ev[1], st));
  }
  CU_TRY(cudaEventRecord(ev[2], st));
  CU_TRY(cudaEventSynchronize(ev[2]));
  CU_TRY(cudaEventElapsedTime(&ms_passes[0], ev[0], ev[1]));
  *n_passes = 1;
  if (path >= 2) {
    CU_TRY(cudaEventElapsedTime(&ms_passes[1], ev[1], ev[2]));
    *n_passes = 2;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return FTLM_OK;
}

int ftlm_gpu_apply_host(ftlm_sector* s, const double* x, double* y) {
  int rc = need_device(s);
  if (rc) return rc;
  if (!x || !y) return fail(FTLM_ERR_INVALID, "null vector");
  const size_t bytes = static_cast<size_t>(s->plan.dim) * sizeof(double2);
  if (!s->hx.p) {
    CU_TRY(s->hx.alloc(bytes));
    CU_TRY(s->hy.alloc(bytes));
  }
  CU_TRY(cudaMemcpyAsync(s->hx.p, x, bytes, cudaMemcpyHostToDevice, s->stream));
  rc = s->apply(s->hx.as<double2>(), s->hy.as<double2>(), s->stream);
  if (rc) return rc;
  CU_TRY(cudaMemcpyAsync(y, s->hy.p, bytes, cudaMemcpyDeviceToHost, s->stream));
  CU_TRY(cudaStreamSynchronize(s->stream));
  return FTLM_OK;
}

}  // extern "C"

namespace {

// The recurrence of src/lanczos.cpp:180-205 on a sector that runs the row + column-slab passes,
// with the BLAS-1 work folded into them: vectors are kept unnormalised (q_k = s_k W_k, s_k =
// 1/beta_{k-1}), the row pass stages s_k W_k, the column pass adds s_k times the up-hop sum and
// emits the partials of z = <q_k, H q_k>, and one pass forms w = H q_k - z q_k - beta_{k-1} q_{k-1}
// with ||w||^2.  Per step: 8 streaming vector passes instead of 12 and no normalisation pass.
// alpha and ||w||^2 are read back once per step for the reference's breakdown test.
int run_lanczos_fused(ftlm_sector* s, int max_steps, unsigned seed, int start_mode, std::vector<double>* alpha,
                      std::vector<double>* beta) {
  alpha->clear();
  beta->clear();
  const int64_t dim = s->plan.dim;
  if (dim <= 0 || max_steps <= 0) return FTLM_OK;
  LanczosWs& ws = s->ws;
  cudaStream_t st = s->stream;
  const int path = s->effective_path();
  const DevSector d = s->dev_for(path);
  if (hv_rows_smem_bytes(d) > 227 * 1024)
    return fail(FTLM_ERR_UNSUPPORTED, "row pass does not fit in shared memory for this sector");
  CU_TRY(ws.ensure(dim));
  const int64_t nblk = hv_cols_blocks(d, s->cols_variant);
  CU_TRY(ws.ensure_dotp(nblk));
  double* scr = ws.scratch.as<double>();
  if (start_mode == FTLM_START_PHILOX) {
    CU_TRY(lz_philox_start(ws.q.as<double2>(), dim, seed, scr, st));
    CU_TRY(lz_normalise_start(ws.q.as<double2>(), dim, scr, st));
  } else if (start_mode == FTLM_START_REFERENCE) {
    std::vector<std::complex<double>> h;
    reference_start(dim, seed, &h);
    CU_TRY(cudaMemcpyAsync(ws.q.p, h.data(), dim * sizeof(double2), cudaMemcpyHostToDevice, st));
    CU_TRY(cudaStreamSynchronize(st));
  } else {
    return fail(FTLM_ERR_INVALID, "unknown start_mode");
  }
  double2* Wk = ws.q.as<double2>();
  double2* Wkm1 = ws.qp.as<double2>();
  double2* Y = ws.w.as<double2>();
  double sk = 1.0, skm1 = 0.0, bprev = 0.0;
  double res[4];
  for (int k = 0; k < max_steps; ++k) {
    CU_TRY(hv_launch_pass(d, Wk, Y, 0, st, s->cols_variant, sk, nullptr));
    CU_TRY(hv_launch_pass(d, Wk, Y, 1, st, s->cols_variant, sk, ws.dotp.as<double>()));
    CU_TRY(lz_reduce_pairs(ws.dotp.as<double>(), nblk, scr, st));
    CU_TRY(lz_update_scaled(Y, Wk, sk, Wkm1, skm1, bprev, k > 0, dim, scr, st));
    CU_TRY(cudaMemcpyAsync(res, scr + kResZ, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaStreamSynchronize(st));
    alpha->push_back(res[0]);
    const double nw2 = res[2];
    if (nw2 < 1e-24) break;
    const double b_k = std::sqrt(nw2);
    beta->push_back(b_k);
    // rotate: W_{k-1} <- W_k, W_k <- w (unnormalised, scale 1/b_k), the old W_{k-1} buffer is next Y
    double2* t = Wkm1;
    Wkm1 = Wk;
    Wk = Y;
    Y = t;
    skm1 = sk;
    sk = 1.0 / b_k;
    bprev = b_k;
  }
  return FTLM_OK;
}

}  // namespace

extern "C" {

int ftlm_gpu_lanczos(ftlm_sector* s, int max_steps, unsigned seed, int start_mode, double* alpha, double* beta,
                     int* n_beta, int* used) {
  int rc = need_device(s);
  if (rc) return rc;
  std::vector<double> a, b;
  if (s->effective_path() >= 2)
    rc = run_lanczos_fused(s, max_steps, seed, start_mode, &a, &b);
  else
    rc = run_lanczos(
        s->plan.dim, [s](const double2* x, double2* y, cudaStream_t st) { return s->apply(x, y, st); }, s->ws,
        max_steps, seed, start_mode, s->stream, &a, &b);
  if (rc) return rc;
  if (alpha) std::copy(a.begin(), a.end(), alpha);
  if (beta) std::copy(b.begin(), b.end(), beta);
  if (n_beta) *n_beta = static_cast<int>(b.size());
  if (used) *used = static_cast<int>(a.size());
  return FTLM_OK;
}

int ftlm_gpu_lanczos_op(long long dim, ftlm_apply_fn fn, void* ctx, int max_steps, unsigned seed, int start_mode,
                        double* alpha, double* beta, int* n_beta, int* used) {
  if (!fn) return fail(FTLM_ERR_INVALID, "null operator");
  LanczosWs ws;
  std::vector<double> a, b;
  const int rc = run_lanczos(
      dim,
      [fn, ctx](const double2* x, double2* y, cudaStream_t st) {
        if (cudaStreamSynchronize(st) != cudaSuccess) return fail(FTLM_ERR_CUDA, "stream sync before operator");
        fn(reinterpret_cast<const double*>(x), reinterpret_cast<double*>(y), ctx);
        if (cudaDeviceSynchronize() != cudaSuccess) return fail(FTLM_ERR_CUDA, "operator callback failed");
        return FTLM_OK;
      },
      ws, max_steps, seed, start_mode, nullptr, &a, &b);
  if (rc) return rc;
  if (alpha) std::copy(a.begin(), a.end(), alpha);
  if (beta) std::copy(b.begin(), b.end(), beta);
  if (n_beta) *n_beta = static_cast<int>(b.size());
  if (used) *used = static_cast<int>(a.size());
  return FTLM_OK;
}

int ftlm_gpu_lanczos_host_op(long long dim, ftlm_host_apply_fn fn, void* ctx, int max_steps, unsigned seed,
                             int start_mode, double* alpha, double* beta, int* n_beta, int* used) {
  if (!fn) return fail(FTLM_ERR_INVALID, "null operator");
  LanczosWs ws;
  std::vector<double> a, b, hx, hy;
  try {
    hx.resize(static_cast<size_t>(std::max(0LL, dim)) * 2);
    hy.resize(static_cast<size_t>(std::max(0LL, dim)) * 2);
  } catch (const std::bad_alloc&) {
    return fail(FTLM_ERR_NOMEM, "host staging buffers");
  }
  const int rc = run_lanczos(
      dim,
      [&](const double2* x, double2* y, cudaStream_t st) {
        CU_TRY(cudaMemcpyAsync(hx.data(), x, dim * sizeof(double2), cudaMemcpyDeviceToHost, st));
        CU_TRY(cudaStreamSynchronize(st));
        fn(hx.data(), hy.data(), ctx);
        CU_TRY(cudaMemcpyAsync(y, hy.data(), dim * sizeof(double2), cudaMemcpyHostToDevice, st));
        CU_TRY(cudaStreamSynchronize(st));
        return FTLM_OK;
      },
      ws, max_steps, seed, start_mode, nullptr, &a, &b);
  if (rc) return rc;
  if (alpha) std::copy(a.begin(), a.end(), alpha);
  if (beta) std::copy(b.begin(), b.end(), beta);
  if (n_beta) *n_beta = static_cast<int>(b.size());
  if (used) *used = static_cast<int>(a.size());
  return FTLM_OK;
}

int ftlm_gpu_ftlm_combine(const double* logq, const double* energy_r, const int* used, int R, int n_bt, double log_dim,
                          double* lnz, double* energy) {
  if (R <= 0 || n_bt < 0 || !logq || !energy_r || !used || !lnz || !energy) return fail(FTLM_ERR_INVALID, "bad arguments");
  if (n_bt == 0) return FTLM_OK;
  const size_t qb = static_cast<size_t>(R) * n_bt * sizeof(double);
  DevBuf dq, de, dn, dz, den;
  CU_TRY(dq.alloc(qb));
  CU_TRY(de.alloc(qb));
  CU_TRY(dn.alloc(R * sizeof(int)));
  CU_TRY(dz.alloc(n_bt * sizeof(double)));
  CU_TRY(den.alloc(n_bt * sizeof(double)));
  CU_TRY(cudaMemcpy(dq.p, logq, qb, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(de.p, energy_r, qb, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(dn.p, used, R * sizeof(int), cudaMemcpyHostToDevice));
  CU_TRY(quad_sector(dq.as<double>(), de.as<double>(), dn.as<int>(), R, n_bt, log_dim, dz.as<double>(),
                     den.as<double>(), nullptr));
  CU_TRY(cudaMemcpy(lnz, dz.p, n_bt * sizeof(double), cudaMemcpyDeviceToHost));
  CU_TRY(cudaMemcpy(energy, den.p, n_bt * sizeof(double), cudaMemcpyDeviceToHost));
  return FTLM_OK;
}

int ftlm_gpu_tridiag_eig(const double* alpha, const double* beta, const int* n, int nc, int ld, int max_rot, double tol,
                         double* lam, double* w0) {
  if (nc < 0 || ld <= 0 || !alpha || !beta || !n || !lam || !w0) return fail(FTLM_ERR_INVALID, "bad arguments");
  if (ld > 160) return fail(FTLM_ERR_UNSUPPORTED, "tridiagonal size > 160 is not supported by the on-chip Jacobi");
  for (int c = 0; c < nc; ++c)
    if (n[c] < 0 || n[c] > ld) return fail(FTLM_ERR_INVALID, "chain length outside [0, ld]");
  if (nc == 0) return FTLM_OK;
  const size_t mat = static_cast<size_t>(nc) * ld * sizeof(double);
  DevBuf da, db, dn, dl, dw;
  CU_TRY(da.alloc(mat));
  CU_TRY(db.alloc(mat));
  CU_TRY(dn.alloc(nc * sizeof(int)));
  CU_TRY(dl.alloc(mat));
  CU_TRY(dw.alloc(mat));
  CU_TRY(cudaMemcpy(da.p, alpha, mat, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(db.p, beta, mat, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(dn.p, n, nc * sizeof(int), cudaMemcpyHostToDevice));
  CU_TRY(quad_jacobi(da.as<double>(), db.as<double>(), dn.as<int>(), nc, ld, max_rot, tol, dl.as<double>(),
                     dw.as<double>(), nullptr));
  CU_TRY(cudaMemcpy(lam, dl.p, mat, cudaMemcpyDeviceToHost));
  CU_TRY(cudaMemcpy(w0, dw.p, mat, cudaMemcpyDeviceToHost));
  return FTLM_OK;
}

int ftlm_gpu_tridiag_quadrature(const double* alpha, const double* beta, const int* n, int nc, int ld,
                                const double* bts, int n_bt, double* logq, double* energy) {
  if (nc < 0 || ld <= 0 || n_bt < 0 || !alpha || !beta || !n || !bts || !logq || !energy)
    return fail(FTLM_ERR_INVALID, "bad arguments");
  if (ld > 160) return fail(FTLM_ERR_UNSUPPORTED, "tridiagonal size > 160 is not supported by the on-chip Jacobi");
  for (int c = 0; c < nc; ++c)
    if (n[c] < 0 || n[c] > ld) return fail(FTLM_ERR_INVALID, "chain length outside [0, ld]");
  if (static_cast<long long>(nc) * n_bt > 0x7fffffffLL) return fail(FTLM_ERR_INVALID, "n_chains * n_bt exceeds 2^31 - 1");
  if (nc == 0 || n_bt == 0) return FTLM_OK;
  const size_t mat = static_cast<size_t>(nc) * ld * sizeof(double);
  const size_t outb = static_cast<size_t>(nc) * n_bt * sizeof(double);
  DevBuf da, db, dn, dl, dw, dbt, dq, de;
  CU_TRY(da.alloc(mat));
  CU_TRY(db.alloc(mat));
  CU_TRY(dn.alloc(nc * sizeof(int)));
  CU_TRY(dl.alloc(mat));
  CU_TRY(dw.alloc(mat));
  CU_TRY(dbt.alloc(n_bt * sizeof(double)));
  CU_TRY(dq.alloc(outb));
  CU_TRY(de.alloc(outb));
  CU_TRY(cudaMemcpy(da.p, alpha, mat, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(db.p, beta, mat, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(dn.p, n, nc * sizeof(int), cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(dbt.p, bts, n_bt * sizeof(double), cudaMemcpyHostToDevice));
  CU_TRY(quad_jacobi(da.as<double>(), db.as<double>(), dn.as<int>(), nc, ld, 0, 1e-14, dl.as<double>(), dw.as<double>(),
                     nullptr));
  CU_TRY(quad_eval(dl.as<double>(), dw.as<double>(), dn.as<int>(), nc, ld, dbt.as<double>(), n_bt, dq.as<double>(),
                   de.as<double>(), nullptr));
  CU_TRY(cudaMemcpy(logq, dq.p, outb, cudaMemcpyDeviceToHost));
  CU_TRY(cudaMemcpy(energy, de.p, outb, cudaMemcpyDeviceToHost));
  return FTLM_OK;
}

int ftlm_gpu_ritz_values(const double* alpha, const double* beta, int n, int k, double* ritz) {
  if (n <= 0 || k <= 0 || !alpha || !ritz || (n > 1 && !beta)) return fail(FTLM_ERR_INVALID, "bad arguments");
  k = std::min(k, n);
  DevBuf da, db, dr;
  CU_TRY(da.alloc(n * sizeof(double)));
  CU_TRY(db.alloc(n * sizeof(double)));
  CU_TRY(dr.alloc(k * sizeof(double)));
  CU_TRY(cudaMemcpy(da.p, alpha, n * sizeof(double), cudaMemcpyHostToDevice));
  if (n > 1) CU_TRY(cudaMemcpy(db.p, beta, (n - 1) * sizeof(double), cudaMemcpyHostToDevice));
  CU_TRY(ritz_bisect(da.as<double>(), db.as<double>(), n, k, dr.as<double>(), nullptr));
  CU_TRY(cudaMemcpy(ritz, dr.p, k * sizeof(double), cudaMemcpyDeviceToHost));
  return FTLM_OK;
}

int ftlm_gpu_lanczos_extrema(ftlm_sector* s, int max_steps, unsigned seed, int start_mode, double* mn, double* mx,
                             int* steps_used) {
  if (!mn || !mx) return fail(FTLM_ERR_INVALID, "null output");
  *mn = 0.0;
  *mx = 0.0;
  if (steps_used) *steps_used = 0;
  std::vector<double> a(std::max(1, max_steps)), b(std::max(1, max_steps));
  int nb = 0, used = 0;
  int rc = ftlm_gpu_lanczos(s, max_steps, seed, start_mode, a.data(), b.data(), &nb, &used);
  if (rc) return rc;
  if (steps_used) *steps_used = used;
  if (used == 0) return FTLM_OK;
  // src/lanczos.cpp:106-123, 211-231: 120 Jacobi rotations, tol 1e-15, on beta[0..used-2].
  if (used > 160) return fail(FTLM_ERR_UNSUPPORTED, "more than 160 Lanczos steps for the on-chip Jacobi");
  std::vector<double> lam(static_cast<size_t>(used)), w(static_cast<size_t>(used));
  std::vector<double> bt(static_cast<size_t>(used), 0.0);
  for (int i = 0; i + 1 < used && i < nb; ++i) bt[static_cast<size_t>(i)] = b[static_cast<size_t>(i)];
  int n1 = used;
  if (used == 1) {
    *mn = a[0];
    *mx = a[0];
    return FTLM_OK;
  }
  rc = ftlm_gpu_tridiag_eig(a.data(), bt.data(), &n1, 1, used, 120, 1e-15, lam.data(), w.data());
  if (rc) return rc;
  *mn = *std::min_element(lam.begin(), lam.end());
  *mx = *std::max_element(lam.begin(), lam.end());
  return FTLM_OK;
}

int ftlm_gpu_set_quadrature(int mode) {
  if (mode != FTLM_QUAD_REFERENCE && mode != FTLM_QUAD_CONVERGED) return fail(FTLM_ERR_INVALID, "unknown quadrature");
  g_quad_converged.store(mode == FTLM_QUAD_CONVERGED);
  return FTLM_OK;
}

int ftlm_gpu_ftlm_sector(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed, int start_mode,
                         double* lnz, double* energy) {
  return plain_sector_ftlm(s, bts, n_bt, R, M, seed, start_mode, plain_quadrature_converged(), lnz, energy);
}

}  // extern "C"

namespace ftlm_b200 {
namespace capi {

int plain_sector_ftlm(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed, int start_mode,
                      bool converged, double* lnz, double* energy) {
  int rc = need_device(s);
  if (rc) return rc;
  if (n_bt < 0 || (n_bt > 0 && (!bts || !lnz || !energy))) return fail(FTLM_ERR_INVALID, "bad arguments");
  const int64_t dim = s->plan.dim;
  R = std::max(1, R);
  M = std::max(1, M);
  if (M > 160) return fail(FTLM_ERR_UNSUPPORTED, "more than 160 Lanczos steps for the on-chip Jacobi");
  if (dim == 1) {  // src/ftlm_thermo.cpp:219-223: apply H to e_0.
    const double one[2] = {1.0, 0.0};
    double h00[2] = {0.0, 0.0};
    rc = ftlm_gpu_apply_host(s, one, h00);
    if (rc) return rc;
    for (int b = 0; b < n_bt; ++b) {
      lnz[b] = -bts[b] * h00[0];
      energy[b] = h00[0];
    }
    return FTLM_OK;
  }
  std::vector<double> A(static_cast<size_t>(R) * M, 0.0), B(static_cast<size_t>(R) * M, 0.0);
  std::vector<int> nv(static_cast<size_t>(R), 0);
  for (int r = 0; r < R; ++r) {
    const unsigned seed_r = seed + static_cast<unsigned>(r) * 100003u;
    int nb = 0, used = 0;
    rc = ftlm_gpu_lanczos(s, M, seed_r, start_mode, &A[static_cast<size_t>(r) * M], &B[static_cast<size_t>(r) * M], &nb,
                          &used);
    if (rc) return rc;
    nv[static_cast<size_t>(r)] = used;
  }
  std::vector<double> lq(static_cast<size_t>(R) * n_bt), eq(static_cast<size_t>(R) * n_bt);
  rc = chain_quadrature(A.data(), B.data(), nv.data(), R, M, bts, n_bt, lq.data(), eq.data(), converged);
  if (rc) return rc;
  DevBuf dq, de, dn, dz, den;
  CU_TRY(dq.alloc(lq.size() * sizeof(double)));
  CU_TRY(de.alloc(eq.size() * sizeof(double)));
  CU_TRY(dn.alloc(nv.size() * sizeof(int)));
  CU_TRY(dz.alloc(n_bt * sizeof(double)));
  CU_TRY(den.alloc(n_bt * sizeof(double)));
  CU_TRY(cudaMemcpy(dq.p, lq.data(), lq.size() * sizeof(double), cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(de.p, eq.data(), eq.size() * sizeof(double), cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(dn.p, nv.data(), nv.size() * sizeof(int), cudaMemcpyHostToDevice));
  CU_TRY(quad_sector(dq.as<double>(), de.as<double>(), dn.as<int>(), R, n_bt, std::log(static_cast<double>(dim)),
                     dz.as<double>(), den.as<double>(), nullptr));
  CU_TRY(cudaMemcpy(lnz, dz.p, n_bt * sizeof(double), cudaMemcpyDeviceToHost));
  CU_TRY(cudaMemcpy(energy, den.p, n_bt * sizeof(double), cudaMemcpyDeviceToHost));
  return FTLM_OK;
}

int chain_quadrature(const double* A, const double* B, const int* n, int nc, int ld, const double* bts, int n_bt,
                     double* lq, double* eq, bool converged) {
  return converged ? ftlm_gpu_tridiag_quadrature_exact(A, B, n, nc, ld, bts, n_bt, lq, eq)
                   : ftlm_gpu_tridiag_quadrature(A, B, n, nc, ld, bts, n_bt, lq, eq);
}

bool plain_quadrature_converged() { return g_quad_converged.load(); }

}  // namespace capi
}  // namespace ftlm_b200

extern "C" {

int ftlm_gpu_gc_reduce(const double* lnz_s, const double* e_s, const int* N_s, int n_sec, const double* bts, int n_bt,
                       const double* mus, int n_mu, int n_sites, double* lnz_gc, double* n_avg, double* e_avg) {
  if (n_sec < 0 || n_bt < 0 || n_mu < 0 || !lnz_s || !e_s || !N_s || !bts || !mus || !lnz_gc || !n_avg || !e_avg)
    return fail(FTLM_ERR_INVALID, "bad arguments");
  if (n_bt == 0 || n_mu == 0) return FTLM_OK;
  const size_t sb = static_cast<size_t>(std::max(n_sec, 1)) * n_bt * sizeof(double);
  const size_t gb = static_cast<size_t>(n_bt) * n_mu * sizeof(double);
  DevBuf dl, de, dN, db, dm, o1, o2, o3;
  CU_TRY(dl.alloc(sb));
  CU_TRY(de.alloc(sb));
  CU_TRY(dN.alloc(std::max(n_sec, 1) * sizeof(int)));
  CU_TRY(db.alloc(n_bt * sizeof(double)));
  CU_TRY(dm.alloc(n_mu * sizeof(double)));
  CU_TRY(o1.alloc(gb));
  CU_TRY(o2.alloc(gb));
  CU_TRY(o3.alloc(gb));
  if (n_sec > 0) {
    CU_TRY(cudaMemcpy(dl.p, lnz_s, static_cast<size_t>(n_sec) * n_bt * sizeof(double), cudaMemcpyHostToDevice));
    CU_TRY(cudaMemcpy(de.p, e_s, static_cast<size_t>(n_sec) * n_bt * sizeof(double), cudaMemcpyHostToDevice));
    CU_TRY(cudaMemcpy(dN.p, N_s, n_sec * sizeof(int), cudaMemcpyHostToDevice));
  }
  CU_TRY(cudaMemcpy(db.p, bts, n_bt * sizeof(double), cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(dm.p, mus, n_mu * sizeof(double), cudaMemcpyHostToDevice));
  CU_TRY(gc_reduce_dev(dl.as<double>(), de.as<double>(), dN.as<int>(), n_sec, db.as<double>(), n_bt, dm.as<double>(),
                       n_mu, n_sites, o1.as<double>(), o2.as<double>(), o3.as<double>(), nullptr));
  CU_TRY(cudaMemcpy(lnz_gc, o1.p, gb, cudaMemcpyDeviceToHost));
  CU_TRY(cudaMemcpy(n_avg, o2.p, gb, cudaMemcpyDeviceToHost));
  CU_TRY(cudaMemcpy(e_avg, o3.p, gb, cudaMemcpyDeviceToHost));
  return FTLM_OK;
}

}  // extern "C"

namespace ftlm_b200 {
namespace capi {

int64_t g_fused_max_dim = int64_t(1) << 17;

// ftlm_gpu_ftlm_sector for many small sectors at once: every chain of every sector in one
// chains_lanczos launch (one CTA per chain), then one batched quadrature; per-sector results in
// lnz_s/e_s rows out_idx[i].  Same start vectors and seeds as the per-sector path.
int fused_sectors_lanczos(const std::vector<ftlm_sector*>& secs, int R, int M, unsigned seed, int start_mode,
                          std::vector<double>* Aout, std::vector<double>* Bout, std::vector<int>* Uout) {
  if (secs.empty()) return FTLM_OK;
  if (start_mode != FTLM_START_REFERENCE && start_mode != FTLM_START_PHILOX)
    return fail(FTLM_ERR_INVALID, "unknown start_mode");
  const int ns = static_cast<int>(secs.size());
  const int nc = ns * R;
  std::vector<DevSector> devs(static_cast<size_t>(ns));
  std::vector<ChainDesc> cds(static_cast<size_t>(nc));
  int64_t total = 0;
  for (int i = 0; i < ns; ++i) {
    devs[static_cast<size_t>(i)] = secs[static_cast<size_t>(i)]->dev;
    for (int r = 0; r < R; ++r) {
      cds[static_cast<size_t>(i) * R + r] = ChainDesc{i, i * R + r, total};
      total += 3 * secs[static_cast<size_t>(i)]->plan.dim;
    }
  }
  cudaStream_t st = secs[0]->stream;
  DevBuf d_sec, d_cd, d_scr, d_a, d_b, d_u, d_red;
  CU_TRY(d_sec.alloc(devs.size() * sizeof(DevSector)));
  CU_TRY(d_cd.alloc(cds.size() * sizeof(ChainDesc)));
  CU_TRY(d_scr.alloc(static_cast<size_t>(total) * sizeof(double2)));
  CU_TRY(d_a.alloc(static_cast<size_t>(nc) * M * sizeof(double)));
  CU_TRY(d_b.alloc(static_cast<size_t>(nc) * M * sizeof(double)));
  CU_TRY(d_u.alloc(static_cast<size_t>(nc) * sizeof(int)));
  CU_TRY(cudaMemcpyAsync(d_sec.p, devs.data(), devs.size() * sizeof(DevSector), cudaMemcpyHostToDevice, st));
  // chains of larger sectors first, 1024 threads each; the rest 256 threads each
  std::vector<ChainDesc> ordered;
  ordered.reserve(cds.size());
  for (const auto& c : cds)
    if (secs[static_cast<size_t>(c.sector)]->plan.dim > 8192) ordered.push_back(c);
  const int n_wide = static_cast<int>(ordered.size());
  for (const auto& c : cds)
    if (secs[static_cast<size_t>(c.sector)]->plan.dim <= 8192) ordered.push_back(c);
  CU_TRY(cudaMemcpyAsync(d_cd.p, ordered.data(), ordered.size() * sizeof(ChainDesc), cudaMemcpyHostToDevice, st));
  CU_TRY(cudaMemsetAsync(d_a.p, 0, static_cast<size_t>(nc) * M * sizeof(double), st));
  CU_TRY(cudaMemsetAsync(d_b.p, 0, static_cast<size_t>(nc) * M * sizeof(double), st));
  double2* scr = d_scr.as<double2>();
  if (start_mode == FTLM_START_REFERENCE) {
    // host RNG (libstdc++ mt19937 + normal_distribution, as the reference), chains in parallel
    std::vector<std::complex<double>> host(static_cast<size_t>(total));
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < hw; ++w)
      pool.emplace_back([&, w]() {
        std::vector<std::complex<double>> q;
        for (int c = static_cast<int>(w); c < nc; c += static_cast<int>(hw)) {
          const int i = c / R, r = c % R;
          reference_start(secs[static_cast<size_t>(i)]->plan.dim, seed + static_cast<unsigned>(r) * 100003u, &q);
          std::copy(q.begin(), q.end(), host.begin() + cds[static_cast<size_t>(c)].off);
        }
      });
    for (auto& th : pool) th.join();
    CU_TRY(cudaMemcpyAsync(scr, host.data(), host.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
    CU_TRY(cudaStreamSynchronize(st));
  } else {
    CU_TRY(d_red.alloc(kScratchDoubles * sizeof(double)));
    for (int c = 0; c < nc; ++c) {
      const int i = c / R, r = c % R;
      const int64_t dim = secs[static_cast<size_t>(i)]->plan.dim;
      double2* q = scr + cds[static_cast<size_t>(c)].off;
      CU_TRY(lz_philox_start(q, dim, seed + static_cast<unsigned>(r) * 100003u, d_red.as<double>(), st));
      CU_TRY(lz_normalise_start(q, dim, d_red.as<double>(), st));
    }
  }
  // the two launches run concurrently: the small chains on a second stream ordered after the copies
  cudaStream_t st2 = nullptr;
  cudaEvent_t ready = nullptr, done = nullptr;
  CU_TRY(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
  cudaError_t ce = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaEventRecord(ready, st);
  if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st2, ready, 0);
  if (ce == cudaSuccess)
    ce = chains_lanczos(d_sec.as<DevSector>(), d_cd.as<ChainDesc>(), n_wide, M, scr, d_a.as<double>(),
                        d_b.as<double>(), d_u.as<int>(), true, st);
  if (ce == cudaSuccess)
    ce = chains_lanczos(d_sec.as<DevSector>(), d_cd.as<ChainDesc>() + n_wide, nc - n_wide, M, scr, d_a.as<double>(),
                        d_b.as<double>(), d_u.as<int>(), false, st2);
  if (ce == cudaSuccess) ce = cudaEventRecord(done, st2);
  if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st, done, 0);
  const cudaError_t se = cudaStreamSynchronize(st);
  if (ready) cudaEventDestroy(ready);
  if (done) cudaEventDestroy(done);
  cudaStreamDestroy(st2);
  CU_TRY(ce);
  CU_TRY(se);
  std::vector<double>& A = *Aout;
  std::vector<double>& B = *Bout;
  std::vector<int>& used = *Uout;
  A.assign(static_cast<size_t>(nc) * M, 0.0);
  B.assign(static_cast<size_t>(nc) * M, 0.0);
  used.assign(static_cast<size_t>(nc), 0);
  CU_TRY(cudaMemcpyAsync(A.data(), d_a.p, A.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaMemcpyAsync(B.data(), d_b.p, B.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaMemcpyAsync(used.data(), d_u.p, used.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  return FTLM_OK;
}

int fused_sectors_ftlm(const std::vector<ftlm_sector*>& secs, const std::vector<int>& out_idx, int R, int M,
                       unsigned seed, int start_mode, const double* bts, int n_bt, double* lnz_s, double* e_s,
                       bool converged) {
  if (secs.empty()) return FTLM_OK;
  const int ns = static_cast<int>(secs.size());
  const int nc = ns * R;
  std::vector<double> A, B;
  std::vector<int> used;
  int rc0 = fused_sectors_lanczos(secs, R, M, seed, start_mode, &A, &B, &used);
  if (rc0) return rc0;
  std::vector<double> lq(static_cast<size_t>(nc) * n_bt), eq(static_cast<size_t>(nc) * n_bt);
  int rc = chain_quadrature(A.data(), B.data(), used.data(), nc, M, bts, n_bt, lq.data(), eq.data(), converged);
  if (rc) return rc;
  for (int i = 0; i < ns; ++i) {
    const size_t o = static_cast<size_t>(i) * R;
    const size_t dst = static_cast<size_t>(out_idx[static_cast<size_t>(i)]) * n_bt;
    rc = ftlm_gpu_ftlm_combine(lq.data() + o * n_bt, eq.data() + o * n_bt, used.data() + o, R, n_bt,
                               std::log(static_cast<double>(secs[static_cast<size_t>(i)]->plan.dim)), lnz_s + dst,
                               e_s + dst);
    if (rc) return rc;
  }
  return FTLM_OK;
}

}  // namespace capi
}  // namespace ftlm_b200

extern "C" {

int ftlm_gpu_lanczos_sectors(ftlm_sector* const* secs, int n_sectors, int R, int M, unsigned seed, int start_mode,
                             double* alpha, double* beta, int* used) {
  if (!secs || n_sectors < 0 || R <= 0 || M <= 0 || !alpha || !beta || !used) return fail(FTLM_ERR_INVALID, "bad arguments");
  std::vector<ftlm_sector*> v(secs, secs + n_sectors);
  for (ftlm_sector* s : v) {
    const int rc = need_device(s);
    if (rc) return rc;
  }
  std::vector<double> A, B;
  std::vector<int> u;
  const int rc = fused_sectors_lanczos(v, R, M, seed, start_mode, &A, &B, &u);
  if (rc) return rc;
  std::copy(A.begin(), A.end(), alpha);
  std::copy(B.begin(), B.end(), beta);
  std::copy(u.begin(), u.end(), used);
  return FTLM_OK;
}

int ftlm_gpu_set_cols_variant(ftlm_sector* s, int variant) {
  if (!s || variant < 0 || variant > 5) return fail(FTLM_ERR_INVALID, "cols variant must be in [0, 6)");
  s->cols_variant = variant;
  return FTLM_OK;
}

int ftlm_gpu_autotune_apply(ftlm_sector* s, int reps, int* path, int* cols_variant, float* ms) {
  int rc = need_device(s);
  if (rc) return rc;
  reps = std::max(1, reps);
  const SectorPlan& P = s->plan;
  // one timing per sector shape and process
  static std::mutex mu;
  static std::map<std::string, std::pair<int, int>> cache;
  char key[160];
  std::snprintf(key, sizeof(key), "%d/%d/%d/%zu/%zu/%d/%d", P.n, P.nu, P.nd, P.hu.size(), P.hd.size(), P.max_up_deg,
                P.max_dn_deg);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      s->apply_path = it->second.first;
      s->cols_variant = it->second.second;
      if (path) *path = s->apply_path;
      if (cols_variant) *cols_variant = s->cols_variant;
      if (ms) *ms = -1.0f;
      return FTLM_OK;
    }
  }
  const int64_t dim = P.dim;
  DevBuf x, y;
  CU_TRY(x.alloc(static_cast<size_t>(dim) * sizeof(double2)));
  CU_TRY(y.alloc(static_cast<size_t>(dim) * sizeof(double2)));
  cudaStream_t st = s->stream;
  CU_TRY(cudaMemsetAsync(x.p, 0, static_cast<size_t>(dim) * sizeof(double2), st));
  const double one[2] = {1.0, 0.0};
  CU_TRY(cudaMemcpyAsync(x.p, one, sizeof(double2), cudaMemcpyHostToDevice, st));
  cudaEvent_t e0, e1;
  CU_TRY(cudaEventCreate(&e0));
  CU_TRY(cudaEventCreate(&e1));
  int best_p = 1, best_v = 0;
  float best = 3.4e38f;
  const bool fast = hv_fast_path_ok(s->dev_for(2), P.max_up_deg);
  const int variants[10][2] = {{1, 0}, {2, 0}, {2, 1}, {2, 2}, {3, 0}, {3, 1}, {3, 2}, {3, 3}, {3, 4}, {3, 5}};
  cudaError_t ce = cudaSuccess;
  for (const auto& v : variants) {
    if (v[0] >= 2 && !fast) continue;
    if (v[0] == 3 && !s->path_available(3)) continue;
    if (v[1] >= 3 && !s->dev.up_pk) continue;
    const DevSector d = s->dev_for(v[0], v[1]);
    const int lp = v[0] == 3 ? 2 : v[0];
    ce = hv_launch(d, x.as<double2>(), y.as<double2>(), lp, st, v[1]);  // warm-up
    if (ce == cudaSuccess) ce = cudaEventRecord(e0, st);
    for (int r = 0; r < reps && ce == cudaSuccess; ++r) ce = hv_launch(d, x.as<double2>(), y.as<double2>(), lp, st, v[1]);
    if (ce == cudaSuccess) ce = cudaEventRecord(e1, st);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    float t = 0.0f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&t, e0, e1);
    if (ce != cudaSuccess) break;
    if (t < best) {
      best = t;
      best_p = v[0];
      best_v = v[1];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CU_TRY(ce);
  s->apply_path = best_p;
  s->cols_variant = best_v;
  {
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = {best_p, best_v};
  }
  if (path) *path = best_p;
  if (cols_variant) *cols_variant = best_v;
  if (ms) *ms = best / static_cast<float>(reps);
  return FTLM_OK;
}

int ftlm_gpu_set_fused_max_dim(long long max_dim) {
  if (max_dim < 0) return fail(FTLM_ERR_INVALID, "max_dim must be >= 0");
  g_fused_max_dim = max_dim;
  return FTLM_OK;
}

int ftlm_gpu_gc_sweep(const ftlm_params* p, int R, int M, unsigned seed, int start_mode, const double* bts, int n_bt,
                      const double* mus, int n_mu, double* lnz_s, double* e_s, double* lnz_gc, double* n_avg,
                      double* e_avg) {
  if (!p || !lnz_s || !e_s) return fail(FTLM_ERR_INVALID, "null argument");
  const int n = p->Lx * p->Ly;
  if (n <= 0 || n > 32) return fail(FTLM_ERR_INVALID, "FockBasis: require 1 <= n_sites <= 32 (bit packing)");
  const int nsec = (n + 1) * (n + 1);
  std::vector<int> N(static_cast<size_t>(nsec));
  std::vector<ftlm_sector*> small;  // sectors for the fused small-sector launch
  std::vector<int> small_idx;
  auto clear_and = [](std::vector<ftlm_sector*>& v, int rc) {
    for (ftlm_sector* x : v) ftlm_gpu_sector_destroy(x);
    v.clear();
    return rc;
  };
  for (int nu = 0; nu <= n; ++nu)
    for (int nd = 0; nd <= n; ++nd) {
      const int idx = nu * (n + 1) + nd;  // benchmarks/bench_ftlm_nmu_rect.cpp:62
      N[static_cast<size_t>(idx)] = nu + nd;
      ftlm_sector* s = nullptr;
      int rc = ftlm_gpu_sector_create(p, nu, nd, &s);
      if (rc) return clear_and(small, rc);
      if (s->plan.dim >= 2 && s->plan.dim <= g_fused_max_dim && M <= 160) {  // fused below
        small.push_back(s);
        small_idx.push_back(idx);
        continue;
      }
      rc = ftlm_gpu_ftlm_sector(s, bts, n_bt, R, M, seed, start_mode, lnz_s + static_cast<size_t>(idx) * n_bt,
                                e_s + static_cast<size_t>(idx) * n_bt);
      ftlm_gpu_sector_destroy(s);
      if (rc) return clear_and(small, rc);
    }
  const int rcf = fused_sectors_ftlm(small, small_idx, std::max(1, R), std::max(1, M), seed, start_mode, bts, n_bt,
                                     lnz_s, e_s, plain_quadrature_converged());
  clear_and(small, FTLM_OK);
  if (rcf) return rcf;
  if (lnz_gc && n_avg && e_avg)
    return ftlm_gpu_gc_reduce(lnz_s, e_s, N.data(), nsec, bts, n_bt, mus, n_mu, n, lnz_gc, n_avg, e_avg);
  return FTLM_OK;
}

}  // extern "C"

