/* ftlm_gpu.h — C ABI of the B200 FTLM hot path for the 2D extended Hubbard model.
 *
 * Every entry point returns an int status (FTLM_OK == 0).  No exception crosses this
 * boundary; on failure ftlm_gpu_last_error() returns a message for the calling thread.
 * Complex vectors are interleaved (re, im) doubles ("complex128") or floats
 * ("complex64").  Functions taking *_dev pointers expect device memory on the current
 * CUDA device; *_host pointers are ordinary host memory.  A `stream` argument is a
 * cudaStream_t passed as void* (NULL = the legacy default stream).  Sector handles are
 * not thread-safe: use one host thread per handle.
 *
 * Reference interfaces replaced (paths inside PeizhiMai/FTLM_extended_Hubbard):
 *   ftlm_gpu_sector_create        FockBasis(n_sites,n_up,n_down)      include/ftlm/fock_basis.hpp:13
 *                                 + build_hubbard_geometry            include/ftlm/lattice.hpp:38-40
 *   ftlm_gpu_sector_create_hops   FockBasis + caller-supplied hoppings/nn_pairs
 *                                 (the vectors apply_extended_hubbard takes)  include/ftlm/hubbard_hamiltonian.hpp:13-16
 *   ftlm_gpu_sector_dim/masks/index_of   FockBasis::dim/up_mask/down_mask/index_of  include/ftlm/fock_basis.hpp:18-24
 *   ftlm_gpu_apply / _apply_host  apply_extended_hubbard               include/ftlm/hubbard_hamiltonian.hpp:13-16
 *   ftlm_gpu_lanczos              lanczos_tridiagonal                  include/ftlm/lanczos.hpp:55-59
 *   ftlm_gpu_lanczos_extrema      lanczos_extrema                      include/ftlm/lanczos.hpp:45-48
 *   ftlm_gpu_lanczos_op           lanczos_tridiagonal with a caller operator (std::function apply_h)
 *   ftlm_gpu_tridiag_quadrature   log_lanczos_tridiagonal_quadrature_exp  src/ftlm_thermo.cpp:83-146
 *   ftlm_gpu_ftlm_sector          ftlm_log_partition_complex/_real     include/ftlm/ftlm_thermo.hpp:41-50
 *   ftlm_gpu_gc_reduce            grand-canonical mu loop              benchmarks/bench_ftlm_nmu_rect.cpp:186-219
 *   ftlm_gpu_gc_sweep             sector loop + mu loop                benchmarks/bench_ftlm_nmu_rect.cpp:138-219
 */
#ifndef FTLM_GPU_H_
#define FTLM_GPU_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FTLM_OK 0
#define FTLM_ERR_INVALID 1     /* bad argument: the reference throws std::invalid_argument */
#define FTLM_ERR_CUDA 2        /* CUDA runtime error (including "no device") */
#define FTLM_ERR_NOMEM 3       /* device or host allocation failed */
#define FTLM_ERR_TIMEOUT 4     /* a bounded device-side wait ran out */
#define FTLM_ERR_UNSUPPORTED 5 /* outside the sizes this build supports */
#define FTLM_ERR_NUMERIC 6     /* a dense eigen-solver did not converge */

/* Mirrors ftlm::HubbardParams (include/ftlm/hubbard_params.hpp:6-15). */
typedef struct ftlm_params {
  int Lx, Ly;
  double t, tp, U, V, phi_x, phi_y;
} ftlm_params;

/* Mirrors ftlm::SpinfulHopping (include/ftlm/lattice.hpp:11-16): H += coeff c^dag_to c_from. */
typedef struct ftlm_hop {
  int from, to, spin; /* spin 0 = up, 1 = down */
  double coeff_re, coeff_im;
} ftlm_hop;

/* Mirrors ftlm::NearestPair (include/ftlm/lattice.hpp:19-22). */
typedef struct ftlm_pair {
  int i, j;
} ftlm_pair;

typedef struct ftlm_sector ftlm_sector;

/* Start vectors of Lanczos chains. */
#define FTLM_START_REFERENCE 0 /* std::mt19937(seed)+std::normal_distribution, host-made (src/lanczos.cpp:140-175) */
#define FTLM_START_PHILOX 1    /* Philox4x32-10 + Box-Muller on the device (counter = element, key = seed) */

const char* ftlm_gpu_last_error(void);
const char* ftlm_gpu_version_string(void);
int ftlm_gpu_device_count(int* n);

/* Geometry exactly as build_hubbard_geometry (src/lattice.cpp:38-110); host-only, no GPU needed.
 * Returns the hop count in *n_hops and pair count in *n_pairs; writes at most max_* entries. */
int ftlm_gpu_build_geometry(const ftlm_params* p, ftlm_hop* hops, int max_hops, int* n_hops, ftlm_pair* pairs,
                            int max_pairs, int* n_pairs);

/* Sector = FockBasis(Lx*Ly, n_up, n_dn) + its device tables.  n_sites <= 32, each spin
 * space <= 2^22 strings, dim = C(n,n_up)*C(n,n_dn) < 2^31 (the reference's int index). */
int ftlm_gpu_sector_create(const ftlm_params* p, int n_up, int n_dn, ftlm_sector** out);
int ftlm_gpu_sector_create_hops(int n_sites, int n_up, int n_dn, double U, double V, const ftlm_hop* hops, int n_hops,
                                const ftlm_pair* pairs, int n_pairs, ftlm_sector** out);
/* Host-only variant (no device tables): basis, tables and plan statistics for CPU checks. */
int ftlm_gpu_sector_create_host(int n_sites, int n_up, int n_dn, double U, double V, const ftlm_hop* hops, int n_hops,
                                const ftlm_pair* pairs, int n_pairs, ftlm_sector** out);
int ftlm_gpu_sector_destroy(ftlm_sector* s);
int ftlm_gpu_sector_dim(const ftlm_sector* s, long long* dim);
int ftlm_gpu_sector_masks(const ftlm_sector* s, uint64_t* up_host, uint64_t* dn_host);
int ftlm_gpu_sector_index_of(const ftlm_sector* s, uint64_t up, uint64_t dn, long long* index);
/* (up, down) strings of one state (FockBasis::up_mask/down_mask, include/ftlm/fock_basis.hpp:20-21). */
int ftlm_gpu_sector_state(const ftlm_sector* s, long long index, uint64_t* up, uint64_t* dn);
/* Mean number of distinct up-hop source rows per up string (the row-gather traffic model). */
int ftlm_gpu_sector_stats(const ftlm_sector* s, double* mean_up_sources, double* mean_dn_sources, long long* du,
                          long long* dd);
/* Host copy of the down-hop gather table (for inspection/tests): n_groups+1 group offsets and the
 * entries (src_rank<<10 | hop_id<<1 | sign), 32 lanes interleaved per group.  Pass NULL buffers to
 * query the sizes. */
int ftlm_gpu_sector_down_table(const ftlm_sector* s, long long* n_groups, long long* n_entries, long long* gptr,
                               uint32_t* entries, int* pad_hop);
/* Host copy of the gauge-basis row-pass table (inspection and tests; no reference counterpart):
 * *available = 0 when the sector has none (Dd + 8 > 16384, more than 32 sites or more than 512 table
 * coefficients).  In the basis g(u,d) = (-1)^popc(u & prefix_parity_shifted(d)) a down hop's
 * coefficient is (-1)^s c_h, s the down-string sign alone.  groups: 4 ints per group of 32 output
 * down strings (entry offset, real-section rounds KR, table-section rounds KT, 0); round k of lane l
 * at offset + ((k / 4) * 32 + l) * 4 + k % 4, KR and KT each a multiple of 4.  Real section (k <
 * KR): src<<4 | cls<<30 | s<<31 with c_h = real2[cls] (or the XOR form, ftlm_gpu_sector_down_table_form);
 * table section (KR <= k < KR + KT):
 * src<<4 | t<<18 | s<<31 with c_h = table[2t] + i table[2t+1].  src >= Dd is a zero sentinel
 * (padding).  NULL buffers query the sizes. */
int ftlm_gpu_sector_down_table_gauge(const ftlm_sector* s, int* available, long long* n_groups, long long* n_entries,
                                     int* n_table, int* groups, uint32_t* entries, double* table, double* real2);
/* Encoding forms of the gauge table (no counterpart in the reference; they say how the row pass
 * forms each coefficient).  *phase = 1: every table value equals real2[cls] * (pc, +-ps) bit for bit,
 * with cls = entry bit 30 and the sign of ps from entry bit 27 (set = conjugate), pc_ps[0..1] =
 * (pc, ps); *phase = 0: the row pass loads table[t] (entry bits 18..26).  *xor_real = 1: a
 * real-section entry's bits 18..31 are the bits by which the high word of its signed coefficient
 * (-1)^s real2[cls] differs from that of real2[0] (same low word); *xor_real = 0: cls<<30 | s<<31.
 * Each section (KR, KT rounds) is padded to a multiple of 4 rounds.  lane_perm (n_groups * 32 bytes):
 * lane L of group g holds the entries of output string g*32 + lane_perm[g*32 + L] (strings are
 * moved between quarter-warps to balance their bank-group loads; the last, partial group is in
 * order).  Outputs other than phase may be NULL. */
int ftlm_gpu_sector_down_table_form(const ftlm_sector* s, int* phase, double* pc_ps, int* xor_real,
                                    unsigned char* lane_perm);
/* Host copy of the packed up-hop list of the column pass (inspection and tests; no reference
 * counterpart): *available = 0 when the sector has none (Du > 16384, more than 32 sites, or a
 * coefficient outside the form below; the column pass then reads the CSR list).  ptr: Du + 1
 * offsets; entry = src | lo<<14 | hi<<19 | conj<<28 | phase<<29 | cls<<30 | s<<31: output up string
 * r gathers x[src, c] with coefficient (-1)^s real2[cls] (times (pc, +-ps), minus sign when conj,
 * for a phase hop) and the column sign (-1)^(number of down sites of column c in [lo, hi)).  NULL
 * buffers query the size. */
int ftlm_gpu_sector_up_table_packed(const ftlm_sector* s, int* available, long long* n_entries, int32_t* ptr,
                                    uint32_t* entries, double* real2, double* pc_ps);
/* Diagonal entry H[i,i] (host computation from the sector tables). */
int ftlm_gpu_sector_diag(const ftlm_sector* s, long long index, double* value);

/* y = H x on device complex128 vectors of length dim (apply_extended_hubbard; y overwritten). */
int ftlm_gpu_apply(ftlm_sector* s, const double* x_dev, double* y_dev, void* stream);
/* Same with host buffers (copies in and out; the drop-in for apply_extended_hubbard). */
int ftlm_gpu_apply_host(ftlm_sector* s, const double* x_host, double* y_host);
/* ftlm_gpu_apply with CUDA-event timing of each kernel pass on `stream` (synchronises): ms_passes[0..1]
 * = row pass, column-slab pass (one entry for the generic path); *n_passes = entries written. */
int ftlm_gpu_apply_profiled(ftlm_sector* s, const double* x_dev, double* y_dev, void* stream, float* ms_passes,
                            int* n_passes);
/* Kernel selection for ftlm_gpu_apply: 0 = automatic, 1 = generic gather, 2 = row pass (per-row
 * coefficient table in shared memory) + column-slab pass, 3 = row pass in the gauge basis
 * (ftlm_gpu_sector_down_table_gauge: register-held real coefficients, one shared-memory load per
 * hop) + column-slab pass (where the sector has no gauge table, as 2).  Automatic picks 3, else 2,
 * else 1; ftlm_gpu_autotune_apply times them all.  All paths give the same matrix elements (sums may
 * differ in the last bits). */
int ftlm_gpu_set_apply_path(ftlm_sector* s, int path);

/* lanczos_tridiagonal on the sector operator.  alpha/beta: host arrays of max_steps entries;
 * *n_beta = number of beta entries written (steps used, or used-1 after a breakdown), *used =
 * steps used.  start_mode: FTLM_START_REFERENCE or FTLM_START_PHILOX. */
int ftlm_gpu_lanczos(ftlm_sector* s, int max_steps, unsigned seed, int start_mode, double* alpha, double* beta,
                     int* n_beta, int* used);
/* lanczos_extrema (min/max Ritz values with the reference's 120-rotation Jacobi). */
int ftlm_gpu_lanczos_extrema(ftlm_sector* s, int max_steps, unsigned seed, int start_mode, double* min_eval,
                             double* max_eval, int* steps_used);

/* Lanczos with a caller operator on device buffers: apply(x_dev, y_dev, ctx) computes y = H x. */
typedef void (*ftlm_apply_fn)(const double* x_dev, double* y_dev, void* ctx);
int ftlm_gpu_lanczos_op(long long dim, ftlm_apply_fn apply, void* ctx, int max_steps, unsigned seed, int start_mode,
                        double* alpha, double* beta, int* n_beta, int* used);

/* Lanczos with a caller operator on HOST buffers, the std::function apply_h of lanczos_tridiagonal
 * (include/ftlm/lanczos.hpp:55-59): vectors stay on the device; each step copies q to a host
 * buffer, calls apply(x_host, y_host, ctx) and copies y back. */
typedef void (*ftlm_host_apply_fn)(const double* x_host, double* y_host, void* ctx);
int ftlm_gpu_lanczos_host_op(long long dim, ftlm_host_apply_fn apply, void* ctx, int max_steps, unsigned seed,
                             int start_mode, double* alpha, double* beta, int* n_beta, int* used);

/* Ritz values and first-row weights of n_chains tridiagonals (alpha/beta: [n_chains][ld]),
 * by the reference's classical Jacobi with max_rot rotations (<=0: max(3000,120n)) and tol.
 * lam/w0 outputs [n_chains][ld]; n[c] = size of chain c.  Host buffers. */
int ftlm_gpu_tridiag_eig(const double* alpha, const double* beta, const int* n, int n_chains, int ld, int max_rot,
                         double tol, double* lam, double* w0);
/* log sum_k w_k exp(-bT lam_k) per chain and temperature: out [n_chains][n_bt]. */
int ftlm_gpu_tridiag_quadrature(const double* alpha, const double* beta, const int* n, int n_chains, int ld,
                                const double* bts, int n_bt, double* logq, double* energy);
/* ftlm_gpu_tridiag_quadrature on caller-owned DEVICE buffers that allocates nothing (no counterpart in
 * the reference).  For callers that must not call cudaMalloc/cudaFree here: device memory owned by
 * another allocator (e.g. a framework pool that has reserved most of HBM) or latency-critical loops
 * where allocation would implicitly synchronise the device.  Intermediate Ritz pairs live in a
 * library-owned 1 MiB __device__ array on every GPU that loads the library: n_chains*ld <= 65536,
 * larger requests fail with FTLM_ERR_UNSUPPORTED.  Requires 0 <= n_dev[c] <= ld: a chain outside
 * that range is skipped (its outputs become NaN) and the call returns FTLM_ERR_INVALID.  Calls that
 * overlap on the GPU race on that array (serialise them on one stream).  The first call on each
 * device (and the first after that device's context is recreated, e.g. by cudaDeviceReset) looks
 * the array up with cudaGetSymbolAddress; make it before any stream capture on that device.  Work
 * is enqueued on `stream`, and the call waits for that stream only, to read back the chain-length
 * check (no device-wide synchronisation). */
int ftlm_gpu_tridiag_quadrature_noalloc(const double* alpha_dev, const double* beta_dev, const int* n_dev, int n_chains,
                                        int ld, const double* bts_dev, int n_bt, double* logq_dev, double* energy_dev,
                                        void* stream);
/* Exact Ritz values (Sturm bisection, ascending) of one tridiagonal: lowest k into ritz[k]. */
int ftlm_gpu_ritz_values(const double* alpha, const double* beta, int n, int k, double* ritz);

/* ln Tr_s e^{-bT H} of one sector at n_bt temperatures from R chains of M steps
 * (seed_r = seed + r*100003, src/ftlm_thermo.cpp:234), plus the FTLM energy <H>_s. */
int ftlm_gpu_ftlm_sector(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed, int start_mode,
                         double* lnz, double* energy);

/* Quadrature of the complex128 sector path (ftlm_gpu_ftlm_sector, ftlm_gpu_gc_sweep, orbit blocks):
 * FTLM_QUAD_REFERENCE (default) = the reference's classical Jacobi with max(3000, 120 n) rotations
 * (src/ftlm_thermo.cpp:83-146; for n ~ 100 at low temperature it stops unconverged, so its ln Z moves
 * by up to ~1e-5 under 1e-7 changes of alpha/beta); FTLM_QUAD_CONVERGED = the converged GPU Jacobi.
 * The batched complex64 path always uses the converged quadrature.  Process-wide setting. */
#define FTLM_QUAD_REFERENCE 0
#define FTLM_QUAD_CONVERGED 1
int ftlm_gpu_set_quadrature(int mode);
/* Sector ln Z from R chain quadratures (src/ftlm_thermo.cpp:246-256): lnz[b] = log_dim +
 * log mean_{r: used[r] > 0} e^{logq[r][b]}; energy = e^{logq}-weighted chain energies.  Host arrays. */
int ftlm_gpu_ftlm_combine(const double* logq, const double* energy_r, const int* used, int R, int n_bt, double log_dim,
                          double* lnz, double* energy);

/* Grand-canonical combination over sectors (host arrays): lnz_s/e_s [n_sec][n_bt], N_s [n_sec];
 * outputs [n_bt][n_mu]: ln Z_GC, <n> per site, <E>. */
int ftlm_gpu_gc_reduce(const double* lnz_s, const double* e_s, const int* N_s, int n_sec, const double* bts, int n_bt,
                       const double* mus, int n_mu, int n_sites, double* lnz_gc, double* n_avg, double* e_avg);

/* Full plain sweep over all (N_up, N_dn) sectors of p: per-sector ln Z_s/E_s [n_sec][n_bt]
 * with sector order nu*(n+1)+nd (bench_ftlm_nmu_rect.cpp:62), then the GC grid. */
int ftlm_gpu_gc_sweep(const ftlm_params* p, int R, int M, unsigned seed, int start_mode, const double* bts, int n_bt,
                      const double* mus, int n_mu, double* lnz_s, double* e_s, double* lnz_gc, double* n_avg,
                      double* e_avg);

/* ---- batched complex64 FTLM (32 chains of a sector per block vector, FP64 scalars) ----
 * Chain r of a sector uses the Philox start vector of FTLM_START_PHILOX with seed + r*100003 (the
 * same vectors the complex128 path draws), rounded to complex64; H·v in FP32, dot products and
 * norms in compensated FP64; the M steps of each 32-chain block run as one CUDA graph.  Device
 * memory: 3 block vectors of dim*32 complex64 (127 GB at 4x4 (8,8)), kept between calls until
 * ftlm_gpu_batched_release(). */
/* Column-pass variant of the batched H·v on this sector: 0/1/2 = 16/8/4-column chunks (the slab of
 * Du x chunk x 256 bytes that L2 keeps resident while every output row reads it).  Same terms in the
 * same order per element: the variants give the same block vector. */
int ftlm_gpu_batched_set_cols_variant(ftlm_sector* s, int variant);
/* Times the batched H·v with each column-pass variant (CUDA events, reps launches after one warm-up,
 * on the batched workspace) and keeps the fastest on the sector; the choice is cached per sector shape
 * for the process (a cached answer returns *ms = -1).  Outputs may be NULL. */
int ftlm_gpu_batched_autotune(ftlm_sector* s, int reps, int* variant, float* ms);
/* alpha/beta [R][M] (beta zero-padded after a breakdown), used [R]. */
int ftlm_gpu_batched_lanczos(ftlm_sector* s, int R, int M, unsigned seed, double* alpha, double* beta, int* used);
/* ftlm_gpu_ftlm_sector on the batched path; sectors with dim <= 2M use the complex128 path with
 * FTLM_START_PHILOX (their Krylov space can be exhausted, where FP64 breakdown detection matters).
 * Chains are evaluated with the converged quadrature (FTLM_QUAD_CONVERGED). */
int ftlm_gpu_batched_ftlm_sector(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed, double* lnz,
                                 double* energy);
/* ftlm_gpu_batched_ftlm_sector with its rounding-error estimate against the complex128 path (the
 * per-result error statement of the complex64 method; no reference counterpart): chains r < n_check
 * (n_check >= 1) are rerun with complex128 vectors from the same Philox start and
 * lnz_err[b] = max_r |L_r(complex64) - L_r(complex128)|, L_r the chain's log quadrature at bts[b];
 * it bounds |d ln Z| for a common per-chain error.  Sectors on the complex128 path report 0. */
int ftlm_gpu_batched_ftlm_sector_checked(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed,
                                         int n_check, double* lnz, double* energy, double* lnz_err);
/* ftlm_gpu_gc_sweep on the batched path (config: all sectors, R chains, M steps). */
int ftlm_gpu_batched_sweep(const ftlm_params* p, int R, int M, unsigned seed, const double* bts, int n_bt,
                           const double* mus, int n_mu, double* lnz_s, double* e_s, double* lnz_gc, double* n_avg,
                           double* e_avg);
/* ftlm_gpu_batched_sweep with per-result error estimates against the complex128 path: lnz_s_err
 * [n_sec][n_bt] as ftlm_gpu_batched_ftlm_sector_checked, and their first-order propagation through
 * the grand-canonical combination, lnz_gc_err = sum_s w_s lnz_s_err and n_err = sum_s w_s
 * |N_s/n - <n>| lnz_s_err ([n_bt][n_mu], w_s the sector weights).  n_check >= 1 complex128 chains
 * per sector (about n_check/R of the plain path's cost). */
int ftlm_gpu_batched_sweep_checked(const ftlm_params* p, int R, int M, unsigned seed, const double* bts, int n_bt,
                                   const double* mus, int n_mu, int n_check, double* lnz_s, double* e_s, double* lnz_gc,
                                   double* n_avg, double* e_avg, double* lnz_s_err, double* lnz_gc_err, double* n_err);
int ftlm_gpu_batched_release(void);

/* Sectors with 2 <= dim <= max_dim in ftlm_gpu_gc_sweep run as one fused launch (one CTA per chain,
 * all M steps on the device; same start vectors and recurrence); default 131072, 0 disables.
 * No reference counterpart (scheduling only). */
int ftlm_gpu_set_fused_max_dim(long long max_dim);
/* Autotuner (no reference counterpart): times the sector's H·v variants — the generic gather kernel
 * and, where it fits, both row passes with 256-, 128- and 512-column slabs (the gauge row pass also
 * with the packed up list) — `reps` times
 * each on a device vector and keeps the fastest for this handle (later ftlm_gpu_apply calls use it).
 * The choice is cached per sector shape (sites, particle numbers, hop counts) for the process; a
 * cached answer returns *ms = -1.  Outputs may be NULL.  Replaces ftlm_gpu_set_apply_path's choice. */
int ftlm_gpu_autotune_apply(ftlm_sector* s, int reps, int* path, int* cols_variant, float* ms);
/* Column-slab width of the row + column pair: 0 = 256, 1 = 128, 2 = 512 columns over the CSR up list;
 * 3 / 4 / 5 = the same widths over the packed up list (ftlm_gpu_sector_up_table_packed; path 3 only,
 * else as 0 / 1 / 2). */
int ftlm_gpu_set_cols_variant(ftlm_sector* s, int variant);
/* The Lanczos chains of several sectors in one launch (one CTA per chain, all M steps on the device):
 * chain r of sector i uses seed + r*100003 and start_mode as ftlm_gpu_lanczos; alpha/beta
 * [n_sectors*R][M] (zero-padded), used [n_sectors*R].  Meant for small sectors (one SM per chain). */
int ftlm_gpu_lanczos_sectors(ftlm_sector* const* secs, int n_sectors, int R, int M, unsigned seed, int start_mode,
                             double* alpha, double* beta, int* used);

/* ---- translation-orbit momentum blocks (sectors built from lattice parameters, n_sites <= 16) ----
 * Basis: canonical orbit representatives (smallest packed up<<16|dn) whose fermionic stabiliser sum
 * |A(K)| > 1e-12, ascending packed order (OrbitKBlockBasis::build, src/orbit_k_block_basis.cpp:70-117).
 * Apply: apply_orbit_k_block (src/orbit_k_block_basis.cpp:151-220) on reduced complex128 vectors. */
typedef struct ftlm_orbit ftlm_orbit;
int ftlm_gpu_orbit_create(ftlm_sector* s, int kx, int ky, ftlm_orbit** out);
/* Same with the survival threshold of OrbitKBlockBasis::build(fb, K, survive_tol)
 * (include/ftlm/symmetry/orbit_k_block_basis.hpp:53, default 1e-12). */
int ftlm_gpu_orbit_create_ex(ftlm_sector* s, int kx, int ky, double survive_tol, ftlm_orbit** out);
/* Tag a sector built from hop lists with its Lx x Ly rectangle (site = y*Lx + x), so that orbit
 * blocks can be built on it (MomentumSector K carries lx, ly in the reference). */
int ftlm_gpu_sector_set_lattice(ftlm_sector* s, int Lx, int Ly);
int ftlm_gpu_orbit_destroy(ftlm_orbit* o);
int ftlm_gpu_orbit_dim(const ftlm_orbit* o, long long* dim);
/* Host copies of the reduced basis: packed representatives and |A(K)| (OrbitKRepEntry rep / abs_A). */
int ftlm_gpu_orbit_entries(const ftlm_orbit* o, uint32_t* rep_packed, double* absA);
/* All OrbitKRepEntry fields (orbit_k_block_basis.hpp:35-42): rep, A_k (2 doubles each), abs_A,
 * orbit_size, stabilizer_size, orbit_index (index into the sector's orbit list, which the reference
 * builds in ascending packed order of the representatives).  Any pointer may be NULL. */
int ftlm_gpu_orbit_entries_ex(const ftlm_orbit* o, uint32_t* rep_packed, double* A, double* absA, int* orbit_size,
                              int* stabilizer_size, long long* orbit_index);
int ftlm_gpu_orbit_apply(ftlm_orbit* o, const double* x_dev, double* y_dev, void* stream);
/* 0: hop list scan per representative; 1 (default): the sector's gather tables, batched gathers.
 * No reference counterpart (both compute apply_orbit_k_block). */
int ftlm_gpu_orbit_set_apply_path(ftlm_orbit* o, int path);
int ftlm_gpu_orbit_apply_host(ftlm_orbit* o, const double* x_host, double* y_host);
/* ftlm_log_partition_complex on one block (seed_r = seed + r*100003). */
int ftlm_gpu_orbit_ftlm(ftlm_orbit* o, const double* bts, int n_bt, int R, int M, unsigned seed, int start_mode,
                        double* lnz, double* energy);
/* All Lx*Ly momentum blocks of a sector (ky outer, kx inner): blocks of dim <= ed_cutoff exactly (dense
 * H_K, eigenvalues of its real embedding; the k-bench's --ed-cutoff, default 64), larger blocks by FTLM
 * with seed_k = seed + sector_index*257 + ky*17 + kx; ln Z_sector = log-sum-exp over blocks
 * (benchmarks/bench_ftlm_nmu_4x4_k.cpp:249-333, 801-1081).  dims_k [Lx*Ly] (may be NULL) receives the
 * block dimensions. */
int ftlm_gpu_orbit_sector_ftlm(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed,
                               int sector_index, int start_mode, int ed_cutoff, double* lnz, double* energy,
                               long long* dims_k);
/* The same with complex64 32-chain blocks (FP64 scalars, Philox starts, the batched sector path's
 * rules; blocks with dim <= 2M on the complex128 Philox path).  ftlm_gpu_orbit_batched_ftlm: one block. */
int ftlm_gpu_orbit_batched_ftlm(ftlm_orbit* o, const double* bts, int n_bt, int R, int M, unsigned seed, double* lnz,
                                double* energy);
int ftlm_gpu_orbit_sector_batched_ftlm(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed,
                                       int sector_index, int ed_cutoff, double* lnz, double* energy, long long* dims_k);

/* ---- parameter gradient of the sector FTLM estimate (no counterpart in the reference) ----
 * Replays the chains of ftlm_gpu_ftlm_sector (method 0, start_mode as there) or of
 * ftlm_gpu_batched_ftlm_sector (method 1; complex64 32-chain blocks, sectors with
 * dim <= 2M on the complex128 Philox path as there) from their seed, keeps their Lanczos vectors
 * on the device and returns
 *   lnz      the sector ln Z estimate at inverse temperature bT (the forward call's value),
 *   dlnz[3]  d lnZ/dU, d lnZ/dV, d lnZ/dt' of that estimate with the start vectors fixed: per
 *            chain the Duhamel derivative -sum_il K_il <q_i|dH/dtheta|q_l> of e_1^T e^{-bT T} e_1.
 * op_tp is a sector of the same (n_sites, N_up, N_dn) built with t = 0, t' = 1, U = V = 0 (the
 * operator dH/dt'), or NULL (dlnz[2] = 0).  Device memory: M (M+1 for method 1) vectors of the
 * sector, twice with op_tp; released by ftlm_gpu_batched_release. */
int ftlm_gpu_grad_sector(ftlm_sector* s, ftlm_sector* op_tp, double bT, int R, int M, unsigned seed, int method,
                         int start_mode, double* lnz, double* dlnz);
/* Differentiable grand-canonical ln Z at one point (no reference counterpart; the combination is the
 * grand-canonical reduction of benchmarks/bench_ftlm_nmu_rect.cpp:186-219 at a single (T, mu)).
 * p gives the lattice and (t, t', U, V, phi_x, phi_y); every (N_up, N_dn) sector's FTLM ln Z_s and
 * energy E_s at inverse temperature bT (method 0: complex128 chains with start_mode; method 1: the
 * batched complex64 chains; converged tridiagonal quadrature; the small sectors' chains in one fused
 * launch) go to lnz_s/e_s [(n+1)^2] in sector order nu*(n+1)+nd, and
 * lnz_gc = log sum_s exp(ln Z_s + bT mu (N_up + N_dn)). */
int ftlm_gpu_gc_logz(const ftlm_params* p, double mu, double bT, int R, int M, unsigned seed, int method,
                     int start_mode, double* lnz_s, double* e_s, double* lnz_gc);
/* Its gradient grad[5] = d lnz_gc / d(U, V, t', mu, bT) from the forward's sector table, the chains
 * replayed from their seeds (ftlm_gpu_grad_sector; sectors of weight < 1e-13 skipped).  Fails with
 * FTLM_ERR_NUMERIC if a replay does not reproduce the forward's ln Z_s. */
int ftlm_gpu_gc_logz_grad(const ftlm_params* p, double mu, double bT, int R, int M, unsigned seed, int method,
                          int start_mode, const double* lnz_s, const double* e_s, double* grad);
/* Host-only dense helpers behind the gradient (no reference counterpart): eigen-decomposition of
 * a symmetric tridiagonal (implicit QL; lam ascending, Z row-major with eigenvectors in columns),
 * and the Duhamel weight matrix K (n x n) with g = e_1^T e^{-bT (T - lam_min)} e_1. */
int ftlm_gpu_tridiag_eigvec(const double* alpha, const double* beta, int n, double* lam, double* Z);
/* Per-chain log e_1^T e^{-bT T} e_1 and energy ratio from that converged decomposition (layout of
 * ftlm_gpu_tridiag_quadrature).  The reference's Jacobi stops after max(3000, 120 n) rotations; for
 * n ~ 80 at low temperature the two differ by up to ~1e-7 in a chain's log quadrature, and the
 * differentiable path uses this one in forward and backward. */
int ftlm_gpu_tridiag_quadrature_exact(const double* alpha, const double* beta, const int* n, int nc, int ld,
                                      const double* bts, int n_bt, double* logq, double* energy);
int ftlm_gpu_duhamel_weights(const double* alpha, const double* beta, int n, double bT, double* K, double* g,
                             double* lam_min);

#ifdef __cplusplus
}
#endif
#endif /* FTLM_GPU_H_ */
