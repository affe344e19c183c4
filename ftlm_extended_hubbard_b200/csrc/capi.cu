// C ABI (include/ftlm_gpu.h): sector handles, H·v, Lanczos, quadrature, grand-canonical sweep.
// Host orchestration only; every floating-point operation on sector vectors runs in the
// kernels of hv.cu / lanczos.cu / quad.cu.  No exception crosses the ABI.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "../../include/ftlm_gpu.h"
#include "batched.cuh"
#include "grad.cuh"
#include "hv.cuh"
#include "orbit.cuh"
#include "plan.hpp"
#include "tridiag.hpp"

using namespace ftlm_b200;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

}  // namespace

int ftlm_b200::set_error(int code, const char* msg) { return fail(code, msg); }

namespace {

#define CU_TRY(expr)                                                                                     \
  do {                                                                                                   \
    cudaError_t e_ = (expr);                                                                             \
    if (e_ != cudaSuccess)                                                                               \
      return fail(e_ == cudaErrorMemoryAllocation ? FTLM_ERR_NOMEM : FTLM_ERR_CUDA,                      \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));                                   \
  } while (0)

template <class T>
cudaError_t upload(const std::vector<T>& v, T** out, std::vector<void*>* owned) {
  *out = nullptr;
  const size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(T);
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return e;
  owned->push_back(p);
  if (!v.empty()) e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  *out = static_cast<T*>(p);
  return e;
}

// Device buffer that frees itself.
struct DevBuf {
  void* p = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t bytes) {
    if (p) cudaFree(p);
    p = nullptr;
    return cudaMalloc(&p, std::max<size_t>(bytes, 16));
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Reference start vector (src/lanczos.cpp:140-175): re, im from std::normal_distribution<double>
// over std::mt19937(seed), normalised with a serial sum; falls back to e_0 when ||q|| < 1e-18.
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
struct LanczosWs {
  int64_t n = 0;
  DevBuf q, qp, w, scratch;
  cudaError_t ensure(int64_t dim) {
    if (n == dim && q.p) return cudaSuccess;
    n = dim;
    cudaError_t e;
    if ((e = q.alloc(dim * sizeof(double2))) != cudaSuccess) return e;
    if ((e = qp.alloc(dim * sizeof(double2))) != cudaSuccess) return e;
    if ((e = w.alloc(dim * sizeof(double2))) != cudaSuccess) return e;
    return scratch.alloc(kScratchDoubles * sizeof(double));
  }
};

// Generic Lanczos loop around an operator on device vectors; the recurrence of
// src/lanczos.cpp:180-205 with alpha, ||w||^2 read back once per step for the breakdown test.
template <class Apply>
int run_lanczos(int64_t dim, Apply&& apply, LanczosWs& ws, int max_steps, unsigned seed, int start_mode,
                cudaStream_t st, std::vector<double>* alpha, std::vector<double>* beta, double2* store = nullptr) {
  alpha->clear();
  beta->clear();
  if (dim <= 0 || max_steps <= 0) return FTLM_OK;
  CU_TRY(ws.ensure(dim));
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
  double2* q = ws.q.as<double2>();
  double2* qp = ws.qp.as<double2>();
  double2* w = ws.w.as<double2>();
  double bprev = 0.0;
  double res[4];
  for (int k = 0; k < max_steps; ++k) {
    if (store)  // keep q_k (gradient replay)
      CU_TRY(cudaMemcpyAsync(store + static_cast<int64_t>(k) * dim, q, dim * sizeof(double2), cudaMemcpyDeviceToDevice,
                             st));
    const int rc = apply(q, w, st);
    if (rc != FTLM_OK) return rc;
    CU_TRY(lz_dotc(q, w, dim, scr, st));
    CU_TRY(lz_update(w, q, qp, bprev, k > 0, dim, scr, st));
    // Next q into the old q_prev buffer (harmless if this step turns out to be the last).
    CU_TRY(lz_scale_by_norm(qp, w, dim, scr, st));
    CU_TRY(cudaMemcpyAsync(res, scr + kResZ, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaStreamSynchronize(st));
    const double a_k = res[0];
    const double nw2 = res[2];
    alpha->push_back(a_k);
    if (nw2 < 1e-24) break;
    const double b_k = std::sqrt(nw2);
    beta->push_back(b_k);
    std::swap(q, qp);  // q_prev <- q ; q <- w / b_k (already written)
    bprev = b_k;
  }
  return FTLM_OK;
}

}  // namespace

struct OrbitSectorData;

struct ftlm_sector {
  SectorPlan plan;
  int Lx = 0, Ly = 0;  // lattice (sectors built from ftlm_params); 0 when built from hop lists
  std::shared_ptr<OrbitSectorData> orbit_data;
  bool on_device = false;
  int device = -1;
  DevSector dev{};
  std::vector<void*> owned;
  int apply_path = 0;  // 0 auto, 1 generic, 2 rows+cols
  LanczosWs ws;
  DevBuf hx, hy;  // staging for the host-buffer apply
  cudaStream_t stream = nullptr;
  ~ftlm_sector() {
    for (void* p : owned) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
  int effective_path() const {
    if (apply_path == 1 || apply_path == 2) return apply_path;
    return hv_fast_path_ok(dev, plan.max_up_deg) ? 2 : 1;
  }
  int apply(const double2* x, double2* y, cudaStream_t st) {
    const int path = effective_path();
    if (path == 2 && hv_rows_smem_bytes(dev) > 227 * 1024)
      return fail(FTLM_ERR_UNSUPPORTED, "row pass does not fit in shared memory for this sector");
    CU_TRY(hv_launch(dev, x, y, path, st));
    return FTLM_OK;
  }
};

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
  float2 *ucf32, *dcf32;
  CU_TRY(upload(upc32, &ucf32, &s->owned));
  CU_TRY(upload(dnc32, &dcf32, &s->owned));
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

int need_device(const ftlm_sector* s) {
  if (!s) return fail(FTLM_ERR_INVALID, "null sector");
  if (!s->on_device) return fail(FTLM_ERR_INVALID, "sector was created host-only");
  return FTLM_OK;
}

}  // namespace

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
  if (!s || path < 0 || path > 2) return fail(FTLM_ERR_INVALID, "bad path");
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
  cudaEvent_t ev[3];
  for (auto& e : ev) CU_TRY(cudaEventCreate(&e));
  CU_TRY(cudaEventRecord(ev[0], st));
  if (path == 2) {
    CU_TRY(hv_launch_pass(s->dev, reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y), 0, st));
    CU_TRY(cudaEventRecord(ev[1], st));
    CU_TRY(hv_launch_pass(s->dev, reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y), 1, st));
  } else {
    CU_TRY(hv_launch(s->dev, reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y), path, st));
    CU_TRY(cudaEventRecord(ev[1], st));
  }
  CU_TRY(cudaEventRecord(ev[2], st));
  CU_TRY(cudaEventSynchronize(ev[2]));
  CU_TRY(cudaEventElapsedTime(&ms_passes[0], ev[0], ev[1]));
  *n_passes = 1;
  if (path == 2) {
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

int ftlm_gpu_lanczos(ftlm_sector* s, int max_steps, unsigned seed, int start_mode, double* alpha, double* beta,
                     int* n_beta, int* used) {
  int rc = need_device(s);
  if (rc) return rc;
  std::vector<double> a, b;
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
    if (n[c] > ld) return fail(FTLM_ERR_INVALID, "chain length exceeds ld");
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

int ftlm_gpu_ftlm_sector(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed, int start_mode,
                         double* lnz, double* energy) {
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
  rc = ftlm_gpu_tridiag_quadrature(A.data(), B.data(), nv.data(), R, M, bts, n_bt, lq.data(), eq.data());
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

int ftlm_gpu_gc_sweep(const ftlm_params* p, int R, int M, unsigned seed, int start_mode, const double* bts, int n_bt,
                      const double* mus, int n_mu, double* lnz_s, double* e_s, double* lnz_gc, double* n_avg,
                      double* e_avg) {
  if (!p || !lnz_s || !e_s) return fail(FTLM_ERR_INVALID, "null argument");
  const int n = p->Lx * p->Ly;
  if (n <= 0 || n > 32) return fail(FTLM_ERR_INVALID, "FockBasis: require 1 <= n_sites <= 32 (bit packing)");
  const int nsec = (n + 1) * (n + 1);
  std::vector<int> N(static_cast<size_t>(nsec));
  for (int nu = 0; nu <= n; ++nu)
    for (int nd = 0; nd <= n; ++nd) {
      const int idx = nu * (n + 1) + nd;  // benchmarks/bench_ftlm_nmu_rect.cpp:62
      N[static_cast<size_t>(idx)] = nu + nd;
      ftlm_sector* s = nullptr;
      int rc = ftlm_gpu_sector_create(p, nu, nd, &s);
      if (rc) return rc;
      rc = ftlm_gpu_ftlm_sector(s, bts, n_bt, R, M, seed, start_mode, lnz_s + static_cast<size_t>(idx) * n_bt,
                                e_s + static_cast<size_t>(idx) * n_bt);
      ftlm_gpu_sector_destroy(s);
      if (rc) return rc;
    }
  if (lnz_gc && n_avg && e_avg)
    return ftlm_gpu_gc_reduce(lnz_s, e_s, N.data(), nsec, bts, n_bt, mus, n_mu, n, lnz_gc, n_avg, e_avg);
  return FTLM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Batched complex64 FTLM (batched.cu): 32 chains per block vector, the M Lanczos steps of a block
// captured once into a CUDA graph and launched without host synchronisation.
namespace {

struct BtWs {
  int64_t cap = 0;
  int mcap = 0;
  DevBuf buf[3], st, partial, alpha, beta, used, flags;
  cudaError_t ensure(int64_t dim, int M) {
    cudaError_t e = cudaSuccess;
    if (dim > cap) {
      for (auto& b : buf) b.alloc(0);  // release before growing
      for (auto& b : buf)
        if ((e = b.alloc(static_cast<size_t>(dim) * kBtChains * sizeof(float2))) != cudaSuccess) return e;
      cap = dim;
    }
    if (!st.p) {
      if ((e = st.alloc(kBtFields * kBtChains * sizeof(double))) != cudaSuccess) return e;
      if ((e = partial.alloc(kBtPartialDoubles * sizeof(double))) != cudaSuccess) return e;
      if ((e = used.alloc(kBtChains * sizeof(int))) != cudaSuccess) return e;
      if ((e = flags.alloc(2 * sizeof(int))) != cudaSuccess) return e;
    }
    if (M > mcap) {
      if ((e = alpha.alloc(static_cast<size_t>(M) * kBtChains * sizeof(double))) != cudaSuccess) return e;
      if ((e = beta.alloc(static_cast<size_t>(M) * kBtChains * sizeof(double))) != cudaSuccess) return e;
      mcap = M;
    }
    return e;
  }
  void release() {
    for (auto& b : buf) b.alloc(0);
    cap = 0;
  }
};

BtWs g_bt;
std::mutex g_bt_mu;

// Krylov vector store of the gradient replay (grows to the largest sector seen).
struct GradWs {
  DevBuf Q, AQ, Kp, part, stunit, zflag;
  size_t qcap = 0, acap = 0, kcap = 0, pcap = 0;
  cudaError_t grow(DevBuf& b, size_t& cap, size_t bytes) {
    if (bytes <= cap && b.p) return cudaSuccess;
    cap = bytes;
    return b.alloc(bytes);
  }
  void release() {
    Q.alloc(0);
    AQ.alloc(0);
    qcap = acap = 0;
  }
};
GradWs g_grad;


// Runs ceil(R/32) blocks of 32 chains on sector s; A/B [R][M] (beta zero-padded), used [R].
template <class Step>
int bt_run_chains_impl(int64_t dim, cudaStream_t st, Step&& step, int R, int M, unsigned seed, std::vector<double>* A,
                       std::vector<double>* B, std::vector<int>* used) {
  A->assign(static_cast<size_t>(R) * M, 0.0);
  B->assign(static_cast<size_t>(R) * M, 0.0);
  used->assign(static_cast<size_t>(R), 0);
  std::lock_guard<std::mutex> lock(g_bt_mu);
  CU_TRY(g_bt.ensure(dim, M));
  float2* bufs[3] = {g_bt.buf[0].as<float2>(), g_bt.buf[1].as<float2>(), g_bt.buf[2].as<float2>()};
  double* sd = g_bt.st.as<double>();
  double* part = g_bt.partial.as<double>();
  double* al = g_bt.alpha.as<double>();
  double* be = g_bt.beta.as<double>();
  int* us = g_bt.used.as<int>();
  int* fl = g_bt.flags.as<int>();
  std::vector<double> ha(static_cast<size_t>(M) * kBtChains), hb(static_cast<size_t>(M) * kBtChains);
  std::vector<int> hu(kBtChains);
  for (int blk = 0; blk * kBtChains < R; ++blk) {
    const unsigned seed_b = seed + static_cast<unsigned>(blk * kBtChains) * 100003u;
    CU_TRY(cudaMemsetAsync(al, 0, static_cast<size_t>(M) * kBtChains * sizeof(double), st));
    CU_TRY(cudaMemsetAsync(be, 0, static_cast<size_t>(M) * kBtChains * sizeof(double), st));
    CU_TRY(bt_start(bufs[0], dim, seed_b, sd, part, us, fl, st));
    cudaGraph_t graph = nullptr;
    CU_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    float2 *wk = bufs[0], *y = bufs[1], *wkm1 = bufs[2];
    cudaError_t ce = cudaSuccess;
    for (int k = 0; k < M && ce == cudaSuccess; ++k) {
      ce = step(wk, wkm1, y, k, sd, part, al, be, us, fl);
      float2* t = wkm1;
      wkm1 = wk;
      wk = y;
      y = t;
    }
    const cudaError_t ee = cudaStreamEndCapture(st, &graph);
    if (ce != cudaSuccess || ee != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return fail(FTLM_ERR_CUDA, std::string("batched step capture: ") +
                                     cudaGetErrorString(ce != cudaSuccess ? ce : ee));
    }
    cudaGraphExec_t exec = nullptr;
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return fail(FTLM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    ce = cudaGraphLaunch(exec, st);
    const cudaError_t se = cudaStreamSynchronize(st);
    cudaGraphExecDestroy(exec);
    if (ce != cudaSuccess || se != cudaSuccess)
      return fail(FTLM_ERR_CUDA, std::string("batched steps: ") + cudaGetErrorString(ce != cudaSuccess ? ce : se));
    CU_TRY(cudaMemcpy(ha.data(), al, ha.size() * sizeof(double), cudaMemcpyDeviceToHost));
    CU_TRY(cudaMemcpy(hb.data(), be, hb.size() * sizeof(double), cudaMemcpyDeviceToHost));
    CU_TRY(cudaMemcpy(hu.data(), us, hu.size() * sizeof(int), cudaMemcpyDeviceToHost));
    for (int r = 0; r < kBtChains; ++r) {
      const int ch = blk * kBtChains + r;
      if (ch >= R) break;
      (*used)[static_cast<size_t>(ch)] = hu[static_cast<size_t>(r)];
      for (int k = 0; k < M; ++k) {
        (*A)[static_cast<size_t>(ch) * M + k] = ha[static_cast<size_t>(k) * kBtChains + r];
        (*B)[static_cast<size_t>(ch) * M + k] = hb[static_cast<size_t>(k) * kBtChains + r];
      }
    }
  }
  return FTLM_OK;
}

int bt_run_chains(ftlm_sector* s, int R, int M, unsigned seed, std::vector<double>* A, std::vector<double>* B,
                  std::vector<int>* used) {
  cudaStream_t st = s->stream;
  const DevSector& S = s->dev;
  return bt_run_chains_impl(
      s->plan.dim, st,
      [&S, st](const float2* wk, const float2* wkm1, float2* y, int k, double* sd, double* part, double* al, double* be,
               int* us, int* fl) { return bt_step(S, wk, wkm1, y, k, sd, part, al, be, us, fl, st); },
      R, M, seed, A, B, used);
}

}  // namespace

extern "C" {

int ftlm_gpu_batched_lanczos(ftlm_sector* s, int R, int M, unsigned seed, double* alpha, double* beta, int* used) {
  int rc = need_device(s);
  if (rc) return rc;
  if (s->plan.max_up_deg > 120)
    return fail(FTLM_ERR_UNSUPPORTED, "batched path: more than 120 up-hop sources per string");
  if (R <= 0 || M <= 0 || !alpha || !beta || !used) return fail(FTLM_ERR_INVALID, "bad arguments");
  std::vector<double> A, B;
  std::vector<int> u;
  rc = bt_run_chains(s, R, M, seed, &A, &B, &u);
  if (rc) return rc;
  std::copy(A.begin(), A.end(), alpha);
  std::copy(B.begin(), B.end(), beta);
  std::copy(u.begin(), u.end(), used);
  return FTLM_OK;
}

int ftlm_gpu_batched_ftlm_sector(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed, double* lnz,
                                 double* energy) {
  int rc = need_device(s);
  if (rc) return rc;
  if (n_bt < 0 || (n_bt > 0 && (!bts || !lnz || !energy))) return fail(FTLM_ERR_INVALID, "bad arguments");
  R = std::max(1, R);
  M = std::max(1, M);
  if (M > 160) return fail(FTLM_ERR_UNSUPPORTED, "more than 160 Lanczos steps for the on-chip Jacobi");
  const int64_t dim = s->plan.dim;
  // Sectors whose Krylov space the chain can exhaust stay on the complex128 path (same Philox
  // start vectors), where the reference's breakdown test is meaningful.
  if (dim <= 2 * static_cast<int64_t>(M)) return ftlm_gpu_ftlm_sector(s, bts, n_bt, R, M, seed, FTLM_START_PHILOX, lnz, energy);
  if (s->plan.max_up_deg > 120)
    return fail(FTLM_ERR_UNSUPPORTED, "batched path: more than 120 up-hop sources per string");
  std::vector<double> A, B;
  std::vector<int> used;
  rc = bt_run_chains(s, R, M, seed, &A, &B, &used);
  if (rc) return rc;
  std::vector<double> lq(static_cast<size_t>(R) * n_bt), eq(static_cast<size_t>(R) * n_bt);
  rc = ftlm_gpu_tridiag_quadrature(A.data(), B.data(), used.data(), R, M, bts, n_bt, lq.data(), eq.data());
  if (rc) return rc;
  return ftlm_gpu_ftlm_combine(lq.data(), eq.data(), used.data(), R, n_bt, std::log(static_cast<double>(dim)), lnz, energy);
}

int ftlm_gpu_batched_sweep(const ftlm_params* p, int R, int M, unsigned seed, const double* bts, int n_bt,
                           const double* mus, int n_mu, double* lnz_s, double* e_s, double* lnz_gc, double* n_avg,
                           double* e_avg) {
  if (!p || !lnz_s || !e_s) return fail(FTLM_ERR_INVALID, "null argument");
  const int n = p->Lx * p->Ly;
  if (n <= 0 || n > 32) return fail(FTLM_ERR_INVALID, "FockBasis: require 1 <= n_sites <= 32 (bit packing)");
  const int nsec = (n + 1) * (n + 1);
  std::vector<int> N(static_cast<size_t>(nsec));
  for (int nu = 0; nu <= n; ++nu)
    for (int nd = 0; nd <= n; ++nd) {
      const int idx = nu * (n + 1) + nd;
      N[static_cast<size_t>(idx)] = nu + nd;
      ftlm_sector* s = nullptr;
      int rc = ftlm_gpu_sector_create(p, nu, nd, &s);
      if (rc) return rc;
      rc = ftlm_gpu_batched_ftlm_sector(s, bts, n_bt, R, M, seed, lnz_s + static_cast<size_t>(idx) * n_bt,
                                        e_s + static_cast<size_t>(idx) * n_bt);
      ftlm_gpu_sector_destroy(s);
      if (rc) return rc;
    }
  if (lnz_gc && n_avg && e_avg)
    return ftlm_gpu_gc_reduce(lnz_s, e_s, N.data(), nsec, bts, n_bt, mus, n_mu, n, lnz_gc, n_avg, e_avg);
  return FTLM_OK;
}

int ftlm_gpu_batched_release(void) {
  std::lock_guard<std::mutex> lock(g_bt_mu);
  g_bt.release();
  g_grad.release();
  return FTLM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Parameter gradient of the sector FTLM estimate (no reference counterpart).
//
// For one chain with normalised start vector r, Lanczos vectors q_i and tridiagonal T, the
// estimator term is g = e_1^T e^{-bT T} e_1 and, with r fixed, its exact derivative in the Krylov
// space is dg/dtheta = -sum_il K_il <q_i| dH/dtheta |q_l> (Duhamel; K from duhamel_weights).  The
// chains are replayed from their seed with the forward's kernels (bit-identical alpha/beta), the
// vectors kept on the device, and the three moments of dH/dU (double occupancy), dH/dV (neighbour
// pair density) and dH/dt' (the t' hopping operator) reduced by grad.cu.
namespace {

struct ChainGrad {
  bool ok = false;
  double lmin = 0.0, g = 0.0, m[3] = {0.0, 0.0, 0.0};
};

// Weight matrices of up to nc chains, layout [i][ld][nc] (chain fastest), scales 1/(b_i b_l).
int fill_weights(int nc, int ld, double bT, const std::vector<int>& n, const std::vector<double>& A,
                 const std::vector<double>& B, const std::vector<std::vector<double>>& scale, std::vector<double>* Kp,
                 std::vector<ChainGrad>* out) {
  Kp->assign(static_cast<size_t>(ld) * ld * nc, 0.0);
  std::vector<double> K;
  for (int c = 0; c < nc; ++c) {
    const int nn = n[static_cast<size_t>(c)];
    ChainGrad& cg = (*out)[static_cast<size_t>(c)];
    cg = ChainGrad{};
    if (nn <= 0) continue;
    K.assign(static_cast<size_t>(nn) * nn, 0.0);
    const std::string err = duhamel_weights(nn, A.data() + static_cast<size_t>(c) * ld, B.data() + static_cast<size_t>(c) * ld,
                                            bT, K.data(), &cg.g, &cg.lmin);
    if (!err.empty()) return fail(FTLM_ERR_NUMERIC, err);
    cg.ok = true;
    const std::vector<double>& sc = scale[static_cast<size_t>(c)];
    for (int i = 0; i < nn; ++i)
      for (int l = 0; l < nn; ++l)
        (*Kp)[(static_cast<size_t>(i) * ld + l) * nc + c] =
            K[static_cast<size_t>(i) * nn + l] / (sc[static_cast<size_t>(i)] * sc[static_cast<size_t>(l)]);
  }
  return FTLM_OK;
}

// Moments of one batch of chains: Q [n][vstride], AQ likewise (or null), Kp [n][ld][nc].
template <class T>
int run_moments(ftlm_sector* s, const T* Q, const T* AQ, int64_t vstride, const std::vector<double>& Kp, int n, int ld,
                int nc, std::vector<ChainGrad>* out) {
  cudaStream_t st = s->stream;
  CU_TRY(g_grad.grow(g_grad.Kp, g_grad.kcap, Kp.size() * sizeof(double)));
  CU_TRY(cudaMemcpyAsync(g_grad.Kp.p, Kp.data(), Kp.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  CU_TRY(g_grad.grow(g_grad.part, g_grad.pcap, static_cast<size_t>(2048) * 32 * 3 * sizeof(double)));
  int grid = 0;
  cudaError_t e;
  if constexpr (sizeof(T) == sizeof(float2))
    e = grad_moments_c64(s->dev, Q, AQ ? AQ : Q, vstride, g_grad.Kp.as<double>(), n, ld, g_grad.part.as<double>(), &grid, st);
  else
    e = grad_moments_c128(s->dev, Q, AQ ? AQ : Q, vstride, g_grad.Kp.as<double>(), n, ld, g_grad.part.as<double>(), &grid,
                          st);
  if (e == cudaErrorInvalidValue)
    return fail(FTLM_ERR_UNSUPPORTED, "gradient: Lanczos vectors of one block do not fit in shared memory");
  CU_TRY(e);
  std::vector<double> hp(static_cast<size_t>(grid) * nc * 3);
  CU_TRY(cudaMemcpyAsync(hp.data(), g_grad.part.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  for (int c = 0; c < nc; ++c) {
    ChainGrad& cg = (*out)[static_cast<size_t>(c)];
    for (int q = 0; q < 3; ++q) {
      double sum = 0.0;
      for (int b = 0; b < grid; ++b) sum += hp[(static_cast<size_t>(b) * nc + c) * 3 + q];
      cg.m[q] = sum;
    }
  }
  return FTLM_OK;
}

// Plain path: complex128 chains of ftlm_gpu_ftlm_sector (seed_r = seed + r*100003).
int grad_plain(ftlm_sector* s, ftlm_sector* op, double bT, int R, int M, unsigned seed, int start_mode,
               std::vector<ChainGrad>* out) {
  const int64_t dim = s->plan.dim;
  CU_TRY(g_grad.grow(g_grad.Q, g_grad.qcap, static_cast<size_t>(M) * dim * sizeof(double2)));
  if (op) CU_TRY(g_grad.grow(g_grad.AQ, g_grad.acap, static_cast<size_t>(M) * dim * sizeof(double2)));
  double2* Q = g_grad.Q.as<double2>();
  double2* AQ = op ? g_grad.AQ.as<double2>() : nullptr;
  out->assign(static_cast<size_t>(R), ChainGrad{});
  std::vector<ChainGrad> one(1);
  for (int r = 0; r < R; ++r) {
    std::vector<double> a, b;
    int rc = run_lanczos(
        dim, [s](const double2* x, double2* y, cudaStream_t st) { return s->apply(x, y, st); }, s->ws, M,
        seed + static_cast<unsigned>(r) * 100003u, start_mode, s->stream, &a, &b, Q);
    if (rc) return rc;
    const int n = static_cast<int>(a.size());
    if (n <= 0) continue;
    std::vector<double> A(static_cast<size_t>(M), 0.0), B(static_cast<size_t>(M), 0.0);
    std::copy(a.begin(), a.end(), A.begin());
    std::copy(b.begin(), b.begin() + std::min<size_t>(b.size(), static_cast<size_t>(M)), B.begin());
    if (op)
      for (int i = 0; i < n; ++i) {
        rc = op->apply(Q + static_cast<int64_t>(i) * dim, AQ + static_cast<int64_t>(i) * dim, s->stream);
        if (rc) return rc;
      }
    std::vector<double> Kp;
    std::vector<std::vector<double>> scale(1, std::vector<double>(static_cast<size_t>(n), 1.0));
    rc = fill_weights(1, M, bT, std::vector<int>{n}, A, B, scale, &Kp, &one);
    if (rc) return rc;
    rc = run_moments<double2>(s, Q, AQ, dim, Kp, n, M, 1, &one);
    if (rc) return rc;
    (*out)[static_cast<size_t>(r)] = one[0];
  }
  return FTLM_OK;
}

// Batched path: complex64 32-chain blocks of ftlm_gpu_batched_ftlm_sector, replayed step by step.
int grad_batched(ftlm_sector* s, ftlm_sector* op, double bT, int R, int M, unsigned seed, std::vector<ChainGrad>* out) {
  const int64_t dim = s->plan.dim;
  const int64_t vs = dim * kBtChains;
  std::lock_guard<std::mutex> lock(g_bt_mu);
  CU_TRY(g_bt.ensure(dim, M));
  CU_TRY(g_grad.grow(g_grad.Q, g_grad.qcap, static_cast<size_t>(M + 1) * vs * sizeof(float2)));
  if (op) CU_TRY(g_grad.grow(g_grad.AQ, g_grad.acap, static_cast<size_t>(M) * vs * sizeof(float2)));
  if (!g_grad.stunit.p) {
    std::vector<double> unit(static_cast<size_t>(kBtFields) * kBtChains, 0.0);
    for (int c = 0; c < kBtChains; ++c) unit[static_cast<size_t>(kBtSin) * kBtChains + c] = 1.0;
    CU_TRY(g_grad.stunit.alloc(unit.size() * sizeof(double)));
    CU_TRY(cudaMemcpy(g_grad.stunit.p, unit.data(), unit.size() * sizeof(double), cudaMemcpyHostToDevice));
    CU_TRY(g_grad.zflag.alloc(sizeof(int)));
    CU_TRY(cudaMemset(g_grad.zflag.p, 0, sizeof(int)));
  }
  cudaStream_t st = s->stream;
  float2* Q = g_grad.Q.as<float2>();
  float2* AQ = op ? g_grad.AQ.as<float2>() : nullptr;
  double* sd = g_bt.st.as<double>();
  double* part = g_bt.partial.as<double>();
  double* al = g_bt.alpha.as<double>();
  double* be = g_bt.beta.as<double>();
  int* us = g_bt.used.as<int>();
  int* fl = g_bt.flags.as<int>();
  out->assign(static_cast<size_t>(R), ChainGrad{});
  std::vector<double> ha(static_cast<size_t>(M) * kBtChains), hb(static_cast<size_t>(M) * kBtChains),
      hs(static_cast<size_t>(kBtFields) * kBtChains);
  std::vector<int> hu(kBtChains);
  for (int blk = 0; blk * kBtChains < R; ++blk) {
    const unsigned seed_b = seed + static_cast<unsigned>(blk * kBtChains) * 100003u;
    CU_TRY(cudaMemsetAsync(al, 0, static_cast<size_t>(M) * kBtChains * sizeof(double), st));
    CU_TRY(cudaMemsetAsync(be, 0, static_cast<size_t>(M) * kBtChains * sizeof(double), st));
    CU_TRY(bt_start(Q, dim, seed_b, sd, part, us, fl, st));
    CU_TRY(cudaMemcpyAsync(hs.data(), sd, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    for (int k = 0; k < M; ++k)
      CU_TRY(bt_step(s->dev, Q + static_cast<int64_t>(k) * vs, Q + static_cast<int64_t>(k > 0 ? k - 1 : 0) * vs,
                     Q + static_cast<int64_t>(k + 1) * vs, k, sd, part, al, be, us, fl, st));
    CU_TRY(cudaMemcpyAsync(ha.data(), al, ha.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaMemcpyAsync(hb.data(), be, hb.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaMemcpyAsync(hu.data(), us, hu.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaStreamSynchronize(st));
    const int nc = std::min(kBtChains, R - blk * kBtChains);
    std::vector<int> n(static_cast<size_t>(kBtChains), 0);
    std::vector<double> A(static_cast<size_t>(kBtChains) * M, 0.0), B(static_cast<size_t>(kBtChains) * M, 0.0);
    std::vector<std::vector<double>> scale(static_cast<size_t>(kBtChains));
    int nmax = 0;
    for (int c = 0; c < nc; ++c) {
      const double sin0 = hs[static_cast<size_t>(kBtSin) * kBtChains + c];
      const int nn = (sin0 > 0.0) ? hu[static_cast<size_t>(c)] : 0;
      n[static_cast<size_t>(c)] = nn;
      nmax = std::max(nmax, nn);
      auto& sc = scale[static_cast<size_t>(c)];
      sc.assign(static_cast<size_t>(std::max(nn, 1)), 1.0);
      for (int k = 0; k < M; ++k) {
        A[static_cast<size_t>(c) * M + k] = ha[static_cast<size_t>(k) * kBtChains + c];
        B[static_cast<size_t>(c) * M + k] = hb[static_cast<size_t>(k) * kBtChains + c];
      }
      if (nn > 0) {  // W_0 = ||raw|| q_0, W_i = beta_{i-1} q_i
        sc[0] = 1.0 / sin0;
        for (int i = 1; i < nn; ++i) sc[static_cast<size_t>(i)] = B[static_cast<size_t>(c) * M + i - 1];
      }
    }
    if (nmax == 0) continue;
    if (op)
      for (int i = 0; i < nmax; ++i)
        CU_TRY(bt_apply(op->dev, Q + static_cast<int64_t>(i) * vs, AQ + static_cast<int64_t>(i) * vs,
                        g_grad.stunit.as<double>(), part, g_grad.zflag.as<int>(), st));
    std::vector<double> Kp;
    std::vector<ChainGrad> cg(static_cast<size_t>(kBtChains));
    int rc = fill_weights(kBtChains, M, bT, n, A, B, scale, &Kp, &cg);
    if (rc) return rc;
    rc = run_moments<float2>(s, Q, AQ, vs, Kp, nmax, M, kBtChains, &cg);
    if (rc) return rc;
    for (int c = 0; c < nc; ++c) (*out)[static_cast<size_t>(blk * kBtChains + c)] = cg[static_cast<size_t>(c)];
  }
  return FTLM_OK;
}

}  // namespace

extern "C" {

int ftlm_gpu_grad_sector(ftlm_sector* s, ftlm_sector* op_tp, double bT, int R, int M, unsigned seed, int method,
                         int start_mode, double* lnz, double* dlnz) {
  int rc = need_device(s);
  if (rc) return rc;
  if (op_tp) {
    rc = need_device(op_tp);
    if (rc) return rc;
    if (op_tp->plan.n != s->plan.n || op_tp->plan.nu != s->plan.nu || op_tp->plan.nd != s->plan.nd)
      return fail(FTLM_ERR_INVALID, "gradient operator sector has a different (n_sites, N_up, N_dn)");
  }
  if (!lnz || !dlnz || method < 0 || method > 1) return fail(FTLM_ERR_INVALID, "bad arguments");
  R = std::max(1, R);
  M = std::max(1, M);
  const int64_t dim = s->plan.dim;
  std::vector<ChainGrad> cg;
  if (method == 1 && dim > 2 * static_cast<int64_t>(M)) {
    if (s->plan.max_up_deg > 120 || (op_tp && op_tp->plan.max_up_deg > 120))
      return fail(FTLM_ERR_UNSUPPORTED, "batched path: more than 120 up-hop sources per string");
    rc = grad_batched(s, op_tp, bT, R, M, seed, &cg);
  } else {
    rc = grad_plain(s, op_tp, bT, R, M, seed, method == 1 ? FTLM_START_PHILOX : start_mode, &cg);
  }
  if (rc) return rc;
  // ln Z = ln dim + log mean_r g_r, g_r = e^{-bT lmin_r} ghat_r; d ln Z = -sum_r e^{-bT lmin_r} m_r / sum_r g_r
  double mx = -std::numeric_limits<double>::infinity();
  int used = 0;
  for (const auto& c : cg)
    if (c.ok) {
      mx = std::max(mx, -bT * c.lmin + std::log(c.g));
      ++used;
    }
  if (used == 0) {
    *lnz = -std::numeric_limits<double>::infinity();
    dlnz[0] = dlnz[1] = dlnz[2] = 0.0;
    return FTLM_OK;
  }
  double zs = 0.0, d[3] = {0.0, 0.0, 0.0};
  for (const auto& c : cg) {
    if (!c.ok) continue;
    const double w = std::exp(-bT * c.lmin - mx);
    zs += w * c.g;
    for (int q = 0; q < 3; ++q) d[q] -= w * c.m[q];
  }
  *lnz = std::log(static_cast<double>(dim)) + mx + std::log(zs / static_cast<double>(used));
  for (int q = 0; q < 3; ++q) dlnz[q] = d[q] / zs;
  if (!op_tp) dlnz[2] = 0.0;
  return FTLM_OK;
}

// Per-chain log quadrature and energy ratio with a converged eigen-decomposition (host QL), the
// quadrature the gradient differentiates; same layout as ftlm_gpu_tridiag_quadrature.
int ftlm_gpu_tridiag_quadrature_exact(const double* alpha, const double* beta, const int* n, int nc, int ld,
                                      const double* bts, int n_bt, double* logq, double* energy) {
  if (nc < 0 || ld <= 0 || n_bt < 0 || !alpha || !beta || !n || (n_bt > 0 && (!bts || !logq || !energy)))
    return fail(FTLM_ERR_INVALID, "bad arguments");
  std::vector<double> lam, Z;
  for (int c = 0; c < nc; ++c) {
    const int nn = n[c];
    if (nn > ld) return fail(FTLM_ERR_INVALID, "chain length exceeds ld");
    double* lq = logq + static_cast<size_t>(c) * n_bt;
    double* eq = energy + static_cast<size_t>(c) * n_bt;
    if (nn <= 0) {
      for (int b = 0; b < n_bt; ++b) {
        lq[b] = -std::numeric_limits<double>::infinity();
        eq[b] = 0.0;
      }
      continue;
    }
    lam.assign(static_cast<size_t>(nn), 0.0);
    Z.assign(static_cast<size_t>(nn) * nn, 0.0);
    const std::string err = tridiag_eigvec(nn, alpha + static_cast<size_t>(c) * ld, beta + static_cast<size_t>(c) * ld,
                                           lam.data(), Z.data());
    if (!err.empty()) return fail(FTLM_ERR_NUMERIC, err);
    for (int b = 0; b < n_bt; ++b) {
      const double bT = bts[b];
      double z = 0.0, ze = 0.0;
      for (int j = 0; j < nn; ++j) {
        const double w = Z[static_cast<size_t>(j)] * Z[static_cast<size_t>(j)] * std::exp(-bT * (lam[static_cast<size_t>(j)] - lam[0]));
        z += w;
        ze += w * lam[static_cast<size_t>(j)];
      }
      lq[b] = -bT * lam[0] + std::log(z);
      eq[b] = ze / z;
    }
  }
  return FTLM_OK;
}

// Host-only helper exposed for tests: eigenvalues/eigenvectors of a symmetric tridiagonal.
int ftlm_gpu_tridiag_eigvec(const double* alpha, const double* beta, int n, double* lam, double* Z) {
  if (n < 0 || (n > 0 && (!alpha || !lam || !Z || (n > 1 && !beta)))) return fail(FTLM_ERR_INVALID, "bad arguments");
  const std::string err = tridiag_eigvec(n, alpha, beta, lam, Z);
  if (!err.empty()) return fail(FTLM_ERR_NUMERIC, err);
  return FTLM_OK;
}

// Host-only helper exposed for tests: the Duhamel weight matrix of one tridiagonal.
int ftlm_gpu_duhamel_weights(const double* alpha, const double* beta, int n, double bT, double* K, double* g,
                             double* lam_min) {
  if (n < 0 || (n > 0 && (!alpha || !K || !g || (n > 1 && !beta)))) return fail(FTLM_ERR_INVALID, "bad arguments");
  const std::string err = duhamel_weights(n, alpha, beta, bT, K, g, lam_min);
  if (!err.empty()) return fail(FTLM_ERR_NUMERIC, err);
  return FTLM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Translation-orbit k-blocks (orbit.cu).  Reference: OrbitKBlockBasis::build and
// apply_orbit_k_block (src/orbit_k_block_basis.cpp:70-220), k-bench block loop
// (benchmarks/bench_ftlm_nmu_4x4_k.cpp:801-1081).
struct OrbitSectorData {
  int G = 0;
  DevBuf tlut, tsite, rorder, rank_u, rank_d, rep_full, reta;
  DevBuf uh_from, uh_to, uh_c, uh_own, uh_oth, dh_from, dh_to, dh_c, dh_own, dh_oth;
  int n_uh = 0, n_dh = 0;
  std::vector<uint32_t> reps_packed;  // all orbit representatives, ascending packed (up<<16 | dn)
  std::vector<int64_t> reps_full;     // their full-space indices
  DevBuf reps_dev;                    // reps_packed on the device
  OrbitDev dev{};
};

struct ftlm_orbit {
  ftlm_sector* sector = nullptr;
  std::shared_ptr<OrbitSectorData> data;
  int kx = 0, ky = 0;
  int64_t dk = 0;
  std::vector<uint32_t> reps;  // surviving representatives (ascending packed)
  std::vector<double> absA;
  std::vector<double> Ak;         // A(K), 2 per representative
  std::vector<int> stab;          // stabiliser size
  std::vector<int64_t> orbit_idx; // index among all representatives of the sector (ascending packed)
  DevBuf reps_dev, sqrtA, table, chi, xs;
  OrbitApplyDev app{};
  LanczosWs ws;
  DevBuf hx, hy;
};

namespace {

template <class T>
cudaError_t upload_to(DevBuf& b, const std::vector<T>& v) {
  cudaError_t e = b.alloc(std::max<size_t>(v.size(), 1) * sizeof(T));
  if (e != cudaSuccess || v.empty()) return e;
  return cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

int build_orbit_sector(ftlm_sector* s) {
  if (s->orbit_data) return FTLM_OK;
  const SectorPlan& P = s->plan;
  if (s->Lx <= 0 || s->Ly <= 0) return fail(FTLM_ERR_UNSUPPORTED, "orbit k-blocks need a sector built from lattice parameters");
  if (P.n > 16) return fail(FTLM_ERR_INVALID, "OrbitKBlockBasis::build: n_sites must be <= 16 (RawState bit width)");
  auto D = std::make_shared<OrbitSectorData>();
  const int Lx = s->Lx, Ly = s->Ly, n = P.n, G = Lx * Ly;
  D->G = G;
  std::vector<uint16_t> tl(static_cast<size_t>(G) * 512, 0);
  std::vector<uint8_t> ts(static_cast<size_t>(G) * 16, 0), ro;
  for (int dy = 0; dy < Ly; ++dy)
    for (int dx = 0; dx < Lx; ++dx) {
      const int R = dy * Lx + dx;
      for (int site = 0; site < n; ++site) {
        const int x = site % Lx, y = site / Lx;
        ts[static_cast<size_t>(R) * 16 + site] = static_cast<uint8_t>(((y + dy) % Ly) * Lx + (x + dx) % Lx);
      }
      for (int half = 0; half < 2; ++half)
        for (int m = 0; m < 256; ++m) {
          uint16_t out = 0;
          for (int b = 0; b < 8; ++b) {
            const int site = half * 8 + b;
            if (site < n && ((m >> b) & 1)) out |= static_cast<uint16_t>(1u << ts[static_cast<size_t>(R) * 16 + site]);
          }
          tl[static_cast<size_t>(R) * 512 + half * 256 + m] = out;
        }
    }
  for (int dx = 0; dx < Lx; ++dx)
    for (int dy = 0; dy < Ly; ++dy) ro.push_back(static_cast<uint8_t>(dy * Lx + dx));  // reference search order
  std::vector<int32_t> rku(65536, -1), rkd(65536, -1);
  for (int64_t i = 0; i < P.up.D; ++i) rku[P.up.masks[static_cast<size_t>(i)]] = static_cast<int32_t>(i);
  for (int64_t i = 0; i < P.dn.D; ++i) rkd[P.dn.masks[static_cast<size_t>(i)]] = static_cast<int32_t>(i);
  CU_TRY(upload_to(D->tlut, tl));
  CU_TRY(upload_to(D->tsite, ts));
  CU_TRY(upload_to(D->rorder, ro));
  CU_TRY(upload_to(D->rank_u, rku));
  CU_TRY(upload_to(D->rank_d, rkd));
  OrbitDev& O = D->dev;
  O.n = n;
  O.Lx = Lx;
  O.Ly = Ly;
  O.G = G;
  O.Du = P.up.D;
  O.Dd = P.dn.D;
  O.dim = P.dim;
  O.umask = s->dev.umask;
  O.dmask = s->dev.dmask;
  O.rank_u = D->rank_u.as<int32_t>();
  O.rank_d = D->rank_d.as<int32_t>();
  O.tlut = D->tlut.as<uint16_t>();
  O.tsite = D->tsite.as<uint8_t>();
  O.rorder = D->rorder.as<uint8_t>();
  CU_TRY(D->rep_full.alloc(static_cast<size_t>(P.dim) * sizeof(int32_t)));
  CU_TRY(D->reta.alloc(static_cast<size_t>(P.dim)));
  CU_TRY(orbit_canon(O, D->rep_full.as<int32_t>(), D->reta.as<uint8_t>(), s->stream));
  std::vector<int32_t> rf(static_cast<size_t>(P.dim));
  CU_TRY(cudaMemcpyAsync(rf.data(), D->rep_full.p, rf.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
  CU_TRY(cudaStreamSynchronize(s->stream));
  std::vector<std::pair<uint32_t, int64_t>> reps;
  for (int64_t i = 0; i < P.dim; ++i)
    if (rf[static_cast<size_t>(i)] == i) {
      const uint32_t u = P.up.masks[static_cast<size_t>(i / P.dn.D)], d = P.dn.masks[static_cast<size_t>(i % P.dn.D)];
      reps.emplace_back((u << 16) | d, i);
    }
  std::sort(reps.begin(), reps.end());
  D->reps_packed.resize(reps.size());
  D->reps_full.resize(reps.size());
  for (size_t b = 0; b < reps.size(); ++b) {
    D->reps_packed[b] = reps[b].first;
    D->reps_full[b] = reps[b].second;
  }
  CU_TRY(upload_to(D->reps_dev, D->reps_packed));
  // merged hops with their JW masks (same convention as the sector plan)
  std::vector<int32_t> f, t;
  std::vector<double2> c;
  std::vector<uint32_t> own, oth;
  for (const auto& h : P.hu) {
    f.push_back(h.from);
    t.push_back(h.to);
    c.push_back(make_double2(h.cre, h.cim));
    own.push_back(h.own_mask);
    oth.push_back(h.other_mask);
  }
  D->n_uh = static_cast<int>(f.size());
  CU_TRY(upload_to(D->uh_from, f));
  CU_TRY(upload_to(D->uh_to, t));
  CU_TRY(upload_to(D->uh_c, c));
  CU_TRY(upload_to(D->uh_own, own));
  CU_TRY(upload_to(D->uh_oth, oth));
  f.clear();
  t.clear();
  c.clear();
  own.clear();
  oth.clear();
  for (const auto& h : P.hd) {
    f.push_back(h.from);
    t.push_back(h.to);
    c.push_back(make_double2(h.cre, h.cim));
    own.push_back(h.own_mask);
    oth.push_back(h.other_mask);
  }
  D->n_dh = static_cast<int>(f.size());
  CU_TRY(upload_to(D->dh_from, f));
  CU_TRY(upload_to(D->dh_to, t));
  CU_TRY(upload_to(D->dh_c, c));
  CU_TRY(upload_to(D->dh_own, own));
  CU_TRY(upload_to(D->dh_oth, oth));
  s->orbit_data = D;
  return FTLM_OK;
}

int orbit_apply_dev(ftlm_orbit* o, const double2* x, double2* y, cudaStream_t st) {
  CU_TRY(orbit_apply(o->app, x, y, st));
  return FTLM_OK;
}

}  // namespace

extern "C" {

int ftlm_gpu_orbit_create(ftlm_sector* s, int kx, int ky, ftlm_orbit** out) {
  return ftlm_gpu_orbit_create_ex(s, kx, ky, 1e-12, out);
}

int ftlm_gpu_sector_set_lattice(ftlm_sector* s, int Lx, int Ly) {
  if (!s || Lx <= 0 || Ly <= 0 || Lx * Ly != s->plan.n)
    return fail(FTLM_ERR_INVALID, "lattice Lx*Ly must equal the sector's number of sites");
  if (s->Lx == Lx && s->Ly == Ly) return FTLM_OK;
  s->Lx = Lx;
  s->Ly = Ly;
  s->orbit_data.reset();
  return FTLM_OK;
}

int ftlm_gpu_orbit_create_ex(ftlm_sector* s, int kx, int ky, double survive_tol, ftlm_orbit** out) {
  int rc = need_device(s);
  if (rc) return rc;
  if (!out) return fail(FTLM_ERR_INVALID, "null output");
  *out = nullptr;
  if (s->Lx > 0 && (kx < 0 || ky < 0 || kx >= s->Lx || ky >= s->Ly)) return fail(FTLM_ERR_INVALID, "momentum out of range");
  rc = build_orbit_sector(s);
  if (rc) return rc;
  auto o = std::make_unique<ftlm_orbit>();
  o->sector = s;
  o->data = s->orbit_data;
  o->kx = kx;
  o->ky = ky;
  const OrbitSectorData& D = *o->data;
  // translation_bloch_phase(K, dx, dy) (include/ftlm/symmetry/momentum_sector.hpp:57-63), R = dy*Lx + dx
  std::vector<double2> chi(static_cast<size_t>(D.G));
  const double pi = std::acos(-1.0);
  for (int dy = 0; dy < s->Ly; ++dy)
    for (int dx = 0; dx < s->Lx; ++dx) {
      const double theta = -2.0 * pi *
                           (static_cast<double>(kx * dx) / static_cast<double>(s->Lx) +
                            static_cast<double>(ky * dy) / static_cast<double>(s->Ly));
      chi[static_cast<size_t>(dy * s->Lx + dx)] = make_double2(std::cos(theta), std::sin(theta));
    }
  CU_TRY(upload_to(o->chi, chi));
  const int64_t nreps = static_cast<int64_t>(D.reps_packed.size());
  DevBuf absA, Adev, sdev;
  CU_TRY(absA.alloc(std::max<int64_t>(nreps, 1) * sizeof(double)));
  CU_TRY(Adev.alloc(std::max<int64_t>(nreps, 1) * sizeof(double2)));
  CU_TRY(sdev.alloc(std::max<int64_t>(nreps, 1) * sizeof(int)));
  CU_TRY(orbit_absA(D.dev, D.reps_dev.as<uint32_t>(), nreps, o->chi.as<double2>(), absA.as<double>(),
                    Adev.as<double2>(), sdev.as<int>(), s->stream));
  std::vector<double> aa(static_cast<size_t>(nreps)), AA(static_cast<size_t>(nreps) * 2);
  std::vector<int> ss(static_cast<size_t>(nreps));
  CU_TRY(cudaMemcpyAsync(aa.data(), absA.p, aa.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CU_TRY(cudaMemcpyAsync(AA.data(), Adev.p, AA.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CU_TRY(cudaMemcpyAsync(ss.data(), sdev.p, ss.size() * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  CU_TRY(cudaStreamSynchronize(s->stream));
  std::vector<int64_t> full;
  std::vector<double> sq;
  for (int64_t b = 0; b < nreps; ++b) {
    if (aa[static_cast<size_t>(b)] <= survive_tol) continue;  // survive_tol (orbit_k_block_basis.hpp:53)
    o->reps.push_back(D.reps_packed[static_cast<size_t>(b)]);
    o->absA.push_back(aa[static_cast<size_t>(b)]);
    o->Ak.push_back(AA[2 * static_cast<size_t>(b)]);
    o->Ak.push_back(AA[2 * static_cast<size_t>(b) + 1]);
    o->stab.push_back(ss[static_cast<size_t>(b)]);
    o->orbit_idx.push_back(b);
    full.push_back(D.reps_full[static_cast<size_t>(b)]);
    sq.push_back(std::sqrt(aa[static_cast<size_t>(b)]));
  }
  o->dk = static_cast<int64_t>(o->reps.size());
  if (o->dk >= (1 << 24)) return fail(FTLM_ERR_UNSUPPORTED, "k-block larger than 2^24 states");
  CU_TRY(upload_to(o->reps_dev, o->reps));
  CU_TRY(upload_to(o->sqrtA, sq));
  {
    DevBuf red, fl;
    CU_TRY(red.alloc(static_cast<size_t>(s->plan.dim) * sizeof(int32_t)));
    CU_TRY(cudaMemsetAsync(red.p, 0xFF, static_cast<size_t>(s->plan.dim) * sizeof(int32_t), s->stream));
    CU_TRY(upload_to(fl, full));
    CU_TRY(orbit_scatter_index(fl.as<int64_t>(), o->dk, red.as<int32_t>(), s->stream));
    CU_TRY(o->table.alloc(static_cast<size_t>(s->plan.dim) * sizeof(uint32_t)));
    CU_TRY(orbit_table(D.dev, D.rep_full.as<int32_t>(), D.reta.as<uint8_t>(), red.as<int32_t>(), o->table.as<uint32_t>(),
                       s->stream));
    CU_TRY(cudaStreamSynchronize(s->stream));
  }
  OrbitApplyDev& A = o->app;
  A.O = D.dev;
  A.S = s->dev;
  A.dk = o->dk;
  A.reps = o->reps_dev.as<uint32_t>();
  A.sqrtA = o->sqrtA.as<double>();
  A.table = o->table.as<uint32_t>();
  A.chi_tab = o->chi.as<double2>();
  A.uhop_from = D.uh_from.as<int32_t>();
  A.uhop_to = D.uh_to.as<int32_t>();
  A.uhop_c = D.uh_c.as<double2>();
  A.uhop_own = D.uh_own.as<uint32_t>();
  A.uhop_oth = D.uh_oth.as<uint32_t>();
  A.n_uhops = D.n_uh;
  A.dhop_from = D.dh_from.as<int32_t>();
  A.dhop_to = D.dh_to.as<int32_t>();
  A.dhop_c = D.dh_c.as<double2>();
  A.dhop_own = D.dh_own.as<uint32_t>();
  A.dhop_oth = D.dh_oth.as<uint32_t>();
  A.n_dhops = D.n_dh;
  CU_TRY(o->xs.alloc(static_cast<size_t>(std::max<int64_t>(o->dk, 1)) * sizeof(double2)));
  A.xs = o->xs.as<double2>();
  A.path = 1;
  *out = o.release();
  return FTLM_OK;
}

int ftlm_gpu_orbit_destroy(ftlm_orbit* o) {
  delete o;
  return FTLM_OK;
}

int ftlm_gpu_orbit_set_apply_path(ftlm_orbit* o, int path) {
  if (!o || (path != 0 && path != 1)) return fail(FTLM_ERR_INVALID, "path must be 0 or 1");
  o->app.path = path;
  return FTLM_OK;
}

int ftlm_gpu_orbit_dim(const ftlm_orbit* o, long long* dim) {
  if (!o || !dim) return fail(FTLM_ERR_INVALID, "null argument");
  *dim = o->dk;
  return FTLM_OK;
}

int ftlm_gpu_orbit_entries(const ftlm_orbit* o, uint32_t* rep_packed, double* absA) {
  if (!o) return fail(FTLM_ERR_INVALID, "null orbit");
  if (rep_packed) std::copy(o->reps.begin(), o->reps.end(), rep_packed);
  if (absA) std::copy(o->absA.begin(), o->absA.end(), absA);
  return FTLM_OK;
}

int ftlm_gpu_orbit_entries_ex(const ftlm_orbit* o, uint32_t* rep_packed, double* A, double* absA, int* orbit_size,
                              int* stabilizer_size, long long* orbit_index) {
  if (!o) return fail(FTLM_ERR_INVALID, "null orbit");
  const int G = o->data->G;
  for (size_t i = 0; i < o->reps.size(); ++i) {
    if (rep_packed) rep_packed[i] = o->reps[i];
    if (A) {
      A[2 * i] = o->Ak[2 * i];
      A[2 * i + 1] = o->Ak[2 * i + 1];
    }
    if (absA) absA[i] = o->absA[i];
    if (stabilizer_size) stabilizer_size[i] = o->stab[i];
    if (orbit_size) orbit_size[i] = o->stab[i] > 0 ? G / o->stab[i] : 0;
    if (orbit_index) orbit_index[i] = o->orbit_idx[i];
  }
  return FTLM_OK;
}

int ftlm_gpu_orbit_apply(ftlm_orbit* o, const double* x, double* y, void* stream) {
  if (!o || !x || !y) return fail(FTLM_ERR_INVALID, "null argument");
  if (x == y) return fail(FTLM_ERR_INVALID, "x and y must not alias");
  return orbit_apply_dev(o, reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y),
                         static_cast<cudaStream_t>(stream));
}

int ftlm_gpu_orbit_apply_host(ftlm_orbit* o, const double* x, double* y) {
  if (!o || !x || !y) return fail(FTLM_ERR_INVALID, "null argument");
  const size_t bytes = static_cast<size_t>(std::max<int64_t>(o->dk, 1)) * sizeof(double2);
  if (!o->hx.p) {
    CU_TRY(o->hx.alloc(bytes));
    CU_TRY(o->hy.alloc(bytes));
  }
  cudaStream_t st = o->sector->stream;
  CU_TRY(cudaMemcpyAsync(o->hx.p, x, o->dk * sizeof(double2), cudaMemcpyHostToDevice, st));
  const int rc = orbit_apply_dev(o, o->hx.as<double2>(), o->hy.as<double2>(), st);
  if (rc) return rc;
  CU_TRY(cudaMemcpyAsync(y, o->hy.p, o->dk * sizeof(double2), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  return FTLM_OK;
}

int ftlm_gpu_orbit_ftlm(ftlm_orbit* o, const double* bts, int n_bt, int R, int M, unsigned seed, int start_mode,
                        double* lnz, double* energy) {
  if (!o) return fail(FTLM_ERR_INVALID, "null orbit");
  if (n_bt < 0 || (n_bt > 0 && (!bts || !lnz || !energy))) return fail(FTLM_ERR_INVALID, "bad arguments");
  R = std::max(1, R);
  M = std::max(1, M);
  if (M > 160) return fail(FTLM_ERR_UNSUPPORTED, "more than 160 Lanczos steps for the on-chip Jacobi");
  const int64_t dk = o->dk;
  if (dk <= 0) {
    for (int b = 0; b < n_bt; ++b) {
      lnz[b] = -std::numeric_limits<double>::infinity();
      energy[b] = 0.0;
    }
    return FTLM_OK;
  }
  if (dk == 1) {  // src/ftlm_thermo.cpp:219-223
    const double one[2] = {1.0, 0.0};
    double h00[2] = {0.0, 0.0};
    const int rc = ftlm_gpu_orbit_apply_host(o, one, h00);
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
    std::vector<double> a, b;
    const int rc = run_lanczos(
        dk, [o](const double2* x, double2* y, cudaStream_t st) { return orbit_apply_dev(o, x, y, st); }, o->ws, M,
        seed + static_cast<unsigned>(r) * 100003u, start_mode, o->sector->stream, &a, &b);
    if (rc) return rc;
    std::copy(a.begin(), a.end(), A.begin() + static_cast<long>(r) * M);
    std::copy(b.begin(), b.end(), B.begin() + static_cast<long>(r) * M);
    nv[static_cast<size_t>(r)] = static_cast<int>(a.size());
  }
  std::vector<double> lq(static_cast<size_t>(R) * n_bt), eq(static_cast<size_t>(R) * n_bt);
  int rc = ftlm_gpu_tridiag_quadrature(A.data(), B.data(), nv.data(), R, M, bts, n_bt, lq.data(), eq.data());
  if (rc) return rc;
  return ftlm_gpu_ftlm_combine(lq.data(), eq.data(), nv.data(), R, n_bt, std::log(static_cast<double>(dk)), lnz, energy);
}

// Batched complex64 FTLM of one block: 32-chain blocks of bt_orbit_step (Philox starts, as the
// sector path); blocks with dim <= 2M use the complex128 Philox path.
int ftlm_gpu_orbit_batched_ftlm(ftlm_orbit* o, const double* bts, int n_bt, int R, int M, unsigned seed, double* lnz,
                                double* energy) {
  if (!o) return fail(FTLM_ERR_INVALID, "null orbit");
  if (n_bt < 0 || (n_bt > 0 && (!bts || !lnz || !energy))) return fail(FTLM_ERR_INVALID, "bad arguments");
  R = std::max(1, R);
  M = std::max(1, M);
  if (M > 160) return fail(FTLM_ERR_UNSUPPORTED, "more than 160 Lanczos steps for the on-chip Jacobi");
  const int64_t dk = o->dk;
  if (dk <= 2 * static_cast<int64_t>(M)) return ftlm_gpu_orbit_ftlm(o, bts, n_bt, R, M, seed, FTLM_START_PHILOX, lnz, energy);
  const SectorPlan& P = o->sector->plan;
  if (P.max_up_deg > 120 || P.max_up_deg + ((P.max_dn_deg + 7) / 8) * 8 + 8 > 256)
    return fail(FTLM_ERR_UNSUPPORTED, "batched orbit path: more than 256 sources per representative");
  cudaStream_t st = o->sector->stream;
  const OrbitApplyDev& Adev = o->app;
  std::vector<double> A, B;
  std::vector<int> used;
  int rc = bt_run_chains_impl(
      dk, st,
      [&Adev, st](const float2* wk, const float2* wkm1, float2* y, int k, double* sd, double* part, double* al,
                  double* be, int* us, int* fl) { return bt_orbit_step(Adev, wk, wkm1, y, k, sd, part, al, be, us, fl, st); },
      R, M, seed, &A, &B, &used);
  if (rc) return rc;
  std::vector<double> lq(static_cast<size_t>(R) * n_bt), eq(static_cast<size_t>(R) * n_bt);
  rc = ftlm_gpu_tridiag_quadrature(A.data(), B.data(), used.data(), R, M, bts, n_bt, lq.data(), eq.data());
  if (rc) return rc;
  return ftlm_gpu_ftlm_combine(lq.data(), eq.data(), used.data(), R, n_bt, std::log(static_cast<double>(dk)), lnz, energy);
}

// Exact ln Tr e^{-bT H_K} of a small block (the k-bench's exact_log_partition_small_complex,
// benchmarks/bench_ftlm_nmu_4x4_k.cpp:249-333): H_K built on the GPU column by column, eigenvalues of
// its real 2dk x 2dk embedding [[Re, -Im], [Im, Re]] (each eigenvalue twice) on the host.
static int orbit_block_ed(ftlm_orbit* o, const double* bts, int n_bt, double* lnz, double* energy) {
  const int64_t dk = o->dk;
  const size_t col = static_cast<size_t>(dk) * sizeof(double2);
  DevBuf X, Y;
  CU_TRY(X.alloc(col * dk));
  CU_TRY(Y.alloc(col * dk));
  cudaStream_t st = o->sector->stream;
  CU_TRY(cudaMemsetAsync(X.p, 0, col * dk, st));
  const double one[2] = {1.0, 0.0};
  for (int64_t j = 0; j < dk; ++j)
    CU_TRY(cudaMemcpyAsync(X.as<double2>() + j * dk + j, one, sizeof(double2), cudaMemcpyHostToDevice, st));
  for (int64_t j = 0; j < dk; ++j) {
    const int rc = orbit_apply_dev(o, X.as<double2>() + j * dk, Y.as<double2>() + j * dk, st);
    if (rc) return rc;
  }
  std::vector<double> H(static_cast<size_t>(dk) * dk * 2);  // column j = H_K e_j
  CU_TRY(cudaMemcpyAsync(H.data(), Y.p, col * dk, cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  const int m = static_cast<int>(2 * dk);
  std::vector<double> Rm(static_cast<size_t>(m) * m), lam(static_cast<size_t>(m));
  for (int64_t j = 0; j < dk; ++j)
    for (int64_t i = 0; i < dk; ++i) {
      const double re = H[2 * (static_cast<size_t>(j) * dk + i)], im = H[2 * (static_cast<size_t>(j) * dk + i) + 1];
      Rm[static_cast<size_t>(i) * m + j] = re;
      Rm[static_cast<size_t>(i) * m + j + dk] = -im;
      Rm[static_cast<size_t>(i + dk) * m + j] = im;
      Rm[static_cast<size_t>(i + dk) * m + j + dk] = re;
    }
  const std::string err = sym_eigvals(m, Rm.data(), lam.data());
  if (!err.empty()) return fail(FTLM_ERR_NUMERIC, err);
  for (int b = 0; b < n_bt; ++b) {
    double z = 0.0, ze = 0.0;
    for (int i = 0; i < m; ++i) {
      const double w = std::exp(-bts[b] * (lam[static_cast<size_t>(i)] - lam[0]));
      z += w;
      ze += w * lam[static_cast<size_t>(i)];
    }
    lnz[b] = std::log(0.5) - bts[b] * lam[0] + std::log(z);
    energy[b] = ze / z;
  }
  return FTLM_OK;
}

// All momentum blocks of a sector (ky outer, kx inner): blocks with dim <= ed_cutoff exactly
// (the k-bench's --ed-cutoff, default 64), larger ones by FTLM with seed_k = seed + sector_index*257 +
// ky*17 + kx; ln Z_sector = log-sum-exp over blocks (benchmarks/bench_ftlm_nmu_4x4_k.cpp:801-1081).
static int orbit_sector_impl(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed,
                             int sector_index, int start_mode, int ed_cutoff, bool batched, double* lnz, double* energy,
                             long long* dims_k) {
  int rc = need_device(s);
  if (rc) return rc;
  if (n_bt <= 0 || !bts || !lnz || !energy) return fail(FTLM_ERR_INVALID, "bad arguments");
  rc = build_orbit_sector(s);
  if (rc) return rc;
  std::vector<double> acc(static_cast<size_t>(n_bt), -std::numeric_limits<double>::infinity());
  std::vector<double> eacc(static_cast<size_t>(n_bt), 0.0);
  std::vector<double> lk(static_cast<size_t>(n_bt)), ek(static_cast<size_t>(n_bt));
  for (int ky = 0; ky < s->Ly; ++ky)
    for (int kx = 0; kx < s->Lx; ++kx) {
      ftlm_orbit* o = nullptr;
      rc = ftlm_gpu_orbit_create(s, kx, ky, &o);
      if (rc) return rc;
      if (dims_k) dims_k[ky * s->Lx + kx] = o->dk;
      if (o->dk > 0) {
        const unsigned seed_k = seed + static_cast<unsigned>(sector_index * 257 + ky * 17 + kx);
        if (o->dk <= ed_cutoff)
          rc = o->dk == 1 ? ftlm_gpu_orbit_ftlm(o, bts, n_bt, R, M, seed_k, start_mode, lk.data(), ek.data())
                          : orbit_block_ed(o, bts, n_bt, lk.data(), ek.data());
        else if (batched)
          rc = ftlm_gpu_orbit_batched_ftlm(o, bts, n_bt, R, M, seed_k, lk.data(), ek.data());
        else
          rc = ftlm_gpu_orbit_ftlm(o, bts, n_bt, R, M, seed_k, start_mode, lk.data(), ek.data());
        if (rc) {
          ftlm_gpu_orbit_destroy(o);
          return rc;
        }
        for (int b = 0; b < n_bt; ++b) {  // running log-sum-exp, energy weighted by e^{ln Z_K}
          const double a = acc[static_cast<size_t>(b)], x = lk[static_cast<size_t>(b)];
          if (!std::isfinite(x)) continue;
          if (!std::isfinite(a)) {
            acc[static_cast<size_t>(b)] = x;
            eacc[static_cast<size_t>(b)] = ek[static_cast<size_t>(b)];
            continue;
          }
          const double m = std::max(a, x);
          const double wa = std::exp(a - m), wx = std::exp(x - m);
          acc[static_cast<size_t>(b)] = m + std::log(wa + wx);
          eacc[static_cast<size_t>(b)] = (wa * eacc[static_cast<size_t>(b)] + wx * ek[static_cast<size_t>(b)]) / (wa + wx);
        }
      }
      ftlm_gpu_orbit_destroy(o);
    }
  std::copy(acc.begin(), acc.end(), lnz);
  std::copy(eacc.begin(), eacc.end(), energy);
  return FTLM_OK;
}

int ftlm_gpu_orbit_sector_ftlm(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed,
                               int sector_index, int start_mode, int ed_cutoff, double* lnz, double* energy,
                               long long* dims_k) {
  return orbit_sector_impl(s, bts, n_bt, R, M, seed, sector_index, start_mode, ed_cutoff, false, lnz, energy, dims_k);
}

int ftlm_gpu_orbit_sector_batched_ftlm(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed,
                                       int sector_index, int ed_cutoff, double* lnz, double* energy, long long* dims_k) {
  return orbit_sector_impl(s, bts, n_bt, R, M, seed, sector_index, FTLM_START_PHILOX, ed_cutoff, true, lnz, energy,
                           dims_k);
}

}  // extern "C"
