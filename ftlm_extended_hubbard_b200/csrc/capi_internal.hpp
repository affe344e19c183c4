// Shared host-side state of the C ABI (capi*.cu): error reporting, device buffers, the Lanczos
// driver, the sector handle and the batched-path workspaces.  Internal; not installed.
#pragma once

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
#include "symeig.cuh"
#include "tridiag.hpp"

namespace ftlm_b200 {
namespace capi {

// Records msg for ftlm_gpu_last_error() (per host thread) and returns code.
int fail(int code, const std::string& msg);

#define CU_TRY(expr)                                                                                     \
  do {                                                                                                   \
    cudaError_t e_ = (expr);                                                                             \
    if (e_ != cudaSuccess)                                                                               \
      return ::ftlm_b200::capi::fail(e_ == cudaErrorMemoryAllocation ? FTLM_ERR_NOMEM : FTLM_ERR_CUDA,   \
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
void reference_start(int64_t dim, unsigned seed, std::vector<std::complex<double>>* q);

struct LanczosWs {
  int64_t n = 0;
  DevBuf q, qp, w, scratch;
  DevBuf dotp;  // column-pass partials of the fused sector recurrence
  int64_t dotp_n = 0;
  cudaError_t ensure_dotp(int64_t nblocks) {
    if (nblocks <= dotp_n && dotp.p) return cudaSuccess;
    dotp_n = nblocks;
    return dotp.alloc(static_cast<size_t>(nblocks) * 2 * sizeof(double));
  }
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

}  // namespace capi
}  // namespace ftlm_b200

struct OrbitSectorData;

// The opaque C handle: a sector plan, its device tables and per-sector workspaces.
struct ftlm_sector {
  ftlm_b200::SectorPlan plan;
  int Lx = 0, Ly = 0;  // lattice (sectors built from ftlm_params); 0 when built from hop lists
  std::shared_ptr<OrbitSectorData> orbit_data;
  bool on_device = false;
  int device = -1;
  ftlm_b200::DevSector dev{};
  std::vector<void*> owned;
  int apply_path = 0;    // 0 auto, 1 generic, 2 rows+cols, 3 rows (register coefficient classes)+cols
  int cols_variant = 0;  // column slab 256/128/512 (0/1/2); 3/4/5: the same over the packed up list (path 3)
  ftlm_b200::capi::LanczosWs ws;
  ftlm_b200::capi::DevBuf hx, hy;  // staging for the host-buffer apply
  cudaStream_t stream = nullptr;
  ~ftlm_sector() {
    for (void* p : owned) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
  // Kernel choice for H·v: 1 = generic gather; 2 = row pass with the per-row coefficient table +
  // column-slab pass over the CSR up list; 3 = row pass in the gauge basis (register-held real
  // coefficients) + column-slab pass, over the packed up list when cols_variant >= 3 and the sector
  // has one.  Automatic: 3, else 2, else 1.
  bool path_available(int path) const {
    if (path == 1) return true;
    if (path == 3 && !dev.dn_g.ent) return false;
    return (path == 2 || path == 3) && ftlm_b200::hv_fast_path_ok(dev_for(path), plan.max_up_deg);
  }
  int effective_path() const {
    if (apply_path >= 1 && apply_path <= 3) return (apply_path == 3 && !dev.dn_g.ent) ? 2 : apply_path;
    if (path_available(3)) return 3;
    return path_available(2) ? 2 : 1;
  }
  // The device view a launch of `path` with column variant cv uses (the row pass reads dn_g on path
  // 3 only, the column pass up_pk on path 3 with cv >= 3 only).
  ftlm_b200::DevSector dev_for(int path, int cv = -1) const {
    ftlm_b200::DevSector d = dev;
    if (cv < 0) cv = cols_variant;
    if (path != 3) d.dn_g.ent = nullptr;
    if (path != 3 || cv < 3) d.up_pk = nullptr;
    return d;
  }
  int apply(const double2* x, double2* y, cudaStream_t st) {
    const int path = effective_path();
    const ftlm_b200::DevSector d = dev_for(path);
    if (path >= 2 && ftlm_b200::hv_rows_smem_bytes(d) > 227 * 1024)
      return ftlm_b200::capi::fail(FTLM_ERR_UNSUPPORTED, "row pass does not fit in shared memory for this sector");
    CU_TRY(ftlm_b200::hv_launch(d, x, y, path == 3 ? 2 : path, st, cols_variant));
    return FTLM_OK;
  }
};

namespace ftlm_b200 {
namespace capi {

int need_device(const ftlm_sector* s);

// ---- batched complex64 path (capi_batched.cu) ------------------------------------------------
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

extern BtWs g_bt;
extern std::mutex g_bt_mu;

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
extern GradWs g_grad;


// Runs ceil(R/32) blocks of 32 chains on sector s; A/B [R][M] (beta zero-padded), used [R].
template <class Step>
int bt_run_chains_impl(int64_t dim, cudaStream_t st, Step&& step, int R, int M, unsigned seed, std::vector<double>* A,
                       std::vector<double>* B, std::vector<int>* used, const DevSector* gauge) {
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
    CU_TRY(bt_start(bufs[0], dim, seed_b, sd, part, us, fl, st, gauge));
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

// Per-chain log quadrature and energy (layout of ftlm_gpu_tridiag_quadrature) with the reference's
// rotation-capped Jacobi (converged == false) or the converged GPU eigen-decomposition.
int chain_quadrature(const double* A, const double* B, const int* n, int nc, int ld, const double* bts, int n_bt,
                     double* lq, double* eq, bool converged);
// The quadrature of the complex128 sector path (ftlm_gpu_set_quadrature; the reference's Jacobi by default).
bool plain_quadrature_converged();
// ftlm_gpu_ftlm_sector with an explicit quadrature choice.
int plain_sector_ftlm(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed, int start_mode,
                      bool converged, double* lnz, double* energy);

// ftlm_gpu_ftlm_sector for many small sectors in one chains_lanczos launch (capi.cu); results in
// rows out_idx[i] of lnz_s / e_s.
int fused_sectors_ftlm(const std::vector<ftlm_sector*>& secs, const std::vector<int>& out_idx, int R, int M,
                       unsigned seed, int start_mode, const double* bts, int n_bt, double* lnz_s, double* e_s,
                       bool converged);

// 32-chain blocks of one sector (bt_step), alpha/beta [R][M], steps used [R].
int bt_run_chains(ftlm_sector* s, int R, int M, unsigned seed, std::vector<double>* A, std::vector<double>* B,
                  std::vector<int>* used);

}  // namespace capi
}  // namespace ftlm_b200
