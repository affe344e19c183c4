// Launchers for the sector H·v kernels (hv.cu) and the Lanczos / quadrature kernels.
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

namespace ftlm_b200 {

// path: 1 = generic gather kernel, 2 = row pass + column-slab pass.  The row pass reads the gauge
// table when S.dn_g.ent is set (else the per-row coefficient table), the column pass the packed up
// list when S.up_pk is set (else the CSR list).  cols_variant: column slab of 256 (0 or 3), 128 (1
// or 4) or 512 (2 or 5) columns.
cudaError_t hv_launch(const DevSector& S, const double2* x, double2* y, int path, cudaStream_t st,
                      int cols_variant = 0);
// One pass of the fast path: 0 = row pass (diag + down hops), 1 = column-slab pass (up hops).
// sx: the passes compute H (sx x) (sx = 1: plain H x, unchanged arithmetic); dotp (column pass,
// may be null): one (re, im) partial of <sx x, y> per column-pass block, hv_cols_blocks() of them.
cudaError_t hv_launch_pass(const DevSector& S, const double2* x, double2* y, int pass, cudaStream_t st,
                           int cols_variant = 0, double sx = 1.0, double* dotp = nullptr);
int64_t hv_cols_blocks(const DevSector& S, int cols_variant);
bool hv_fast_path_ok(const DevSector& S, int max_up_deg);
size_t hv_rows_smem_bytes(const DevSector& S);

// ---- Lanczos BLAS-1 (lanczos.cu); all reductions deterministic (fixed grid, fixed tree) ----
constexpr int kRedBlocks = 1184;  // 8 x 148 SMs
constexpr int kRedThreads = 256;
// Scratch layout (doubles): [0, 2*kRedBlocks) partials; then results.
constexpr int kScratchDoubles = 2 * kRedBlocks + 64;
constexpr int kResZ = 2 * kRedBlocks;       // complex <q, w>
constexpr int kResNw2 = 2 * kRedBlocks + 2; // ||w||^2
constexpr int kResN0 = 2 * kRedBlocks + 3;  // ||q||^2 (start vector)

cudaError_t lz_dotc(const double2* q, const double2* w, int64_t n, double* scratch, cudaStream_t st);
// Sum of nb (re, im) partials (fixed two-level tree) into scratch[kResZ..kResZ+1].
cudaError_t lz_reduce_pairs(const double* partial, int64_t nb, double* scratch, cudaStream_t st);
// Lanczos update on unnormalised vectors q_k = sk Wk, q_{k-1} = skm1 Wkm1:
// w = w - z q_k - bprev q_{k-1} (z from scratch[kResZ]); ||w||^2 -> scratch[kResNw2].
cudaError_t lz_update_scaled(double2* w, const double2* Wk, double sk, const double2* Wkm1, double skm1, double bprev,
                             int use_prev, int64_t n, double* scratch, cudaStream_t st);
// w = w - z q - bprev * qp (bprev from host; use_prev selects the second term); ||w||^2 -> scratch.
cudaError_t lz_update(double2* w, const double2* q, const double2* qp, double bprev, int use_prev, int64_t n,
                      double* scratch, cudaStream_t st);
// dst = src / sqrt(scratch[kResNw2])
cudaError_t lz_scale_by_norm(double2* dst, const double2* src, int64_t n, const double* scratch, cudaStream_t st);
// q <- Philox complex Gaussian (key = seed), then ||q||^2 -> scratch[kResN0].
cudaError_t lz_philox_start(double2* q, int64_t n, unsigned seed, double* scratch, cudaStream_t st);
// q <- q / sqrt(scratch[kResN0]) (or e_0 if the norm is < 1e-18)
cudaError_t lz_normalise_start(double2* q, int64_t n, const double* scratch, cudaStream_t st);

// ---- quadrature (quad.cu) ----
// Batched classical Jacobi, one CTA per chain: alpha/beta [nc][ld], n[nc]; outputs lam/w0 [nc][ld].
// A chain with n outside [0, ld] is skipped and sets *bad (when bad is given).
cudaError_t quad_jacobi(const double* alpha, const double* beta, const int* n, int nc, int ld, int max_rot,
                        double tol, double* lam, double* w0, cudaStream_t st, int* bad = nullptr);
// logq/energy [nc][nbt] from lam/w0; a chain with n outside [0, ld] gets NaN and sets *bad.
cudaError_t quad_eval(const double* lam, const double* w0, const int* n, int nc, int ld, const double* bts, int nbt,
                      double* logq, double* energy, cudaStream_t st, int* bad = nullptr);
// Sector ln Z from R chain values: lnz[b] = ln(dim) + log mean_r exp(logq[r][b]); energy weighted.
cudaError_t quad_sector(const double* logq, const double* eq, const int* n, int R, int nbt, double log_dim,
                        double* lnz, double* energy, cudaStream_t st);
cudaError_t gc_reduce_dev(const double* lnz_s, const double* e_s, const int* N_s, int n_sec, const double* bts,
                          int n_bt, const double* mus, int n_mu, int n_sites, double* lnz_gc, double* n_avg,
                          double* e_avg, cudaStream_t st);
cudaError_t ritz_bisect(const double* alpha, const double* beta, int n, int k, double* ritz, cudaStream_t st);

// Records an error message for ftlm_gpu_last_error() (capi.cu) and returns `code`.
int set_error(int code, const char* msg);

}  // namespace ftlm_b200
