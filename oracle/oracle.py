"""ORACLE (test infrastructure only): ctypes access to the CPU checkers.

  Oracle     oracle/libftlm_oracle.so — the in-repo C++ restatement (ftlm_oracle.cpp)
  Reference  oracle/_ref/libftlm_ref.so — the reference's own hot-path sources + ref_shim.cpp

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use this module, as the checker or
as the timed CPU baseline; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libftlm_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libftlm_ref.so")
# Where the reference checkout lives: $FTLM_REFERENCE_SRC, else a sibling checkout named "reference"
# next to this repository.  Only building the checker reads it; the built libraries travel.
REFERENCE_SRC = os.environ.get("FTLM_REFERENCE_SRC") or os.path.normpath(
    os.path.join(HERE, os.pardir, os.pardir, "reference"))

_d, _i, _vp, _ll = C.c_double, C.c_int, C.c_void_p, C.c_longlong


def build(ref: bool = True) -> None:
    """Builds the oracle (always) and the reference library (when its sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref and os.path.isdir(os.path.join(REFERENCE_SRC, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REFERENCE_SRC}"], check=True)
        # the reference's own test/driver programs compiled against the C++ drop-in (needs libftlm_dropin.so)
        if os.path.exists(os.path.join(os.path.dirname(HERE), "ftlm_extended_hubbard_b200", "libftlm_dropin.so")):
            subprocess.run(["make", "-s", "-C", HERE, "dropin", f"REF={REFERENCE_SRC}"], check=True)


def P(a: np.ndarray) -> C.c_void_p:
    return a.ctypes.data_as(C.c_void_p)


def _load_oracle() -> C.CDLL:
    if not os.path.exists(ORACLE_SO):
        build(ref=False)
    L = C.CDLL(ORACLE_SO)
    L.or_sector_create.restype = _vp
    L.or_sector_create.argtypes = [_i, _i, _d, _d, _d, _d, _d, _d, _i, _i]
    L.or_sector_destroy.argtypes = [_vp]
    L.or_sector_dim.restype = _ll
    L.or_sector_dim.argtypes = [_vp]
    L.or_sector_masks.argtypes = [_vp, _vp, _vp]
    L.or_sector_index_of.restype = _ll
    L.or_sector_index_of.argtypes = [_vp, C.c_uint64, C.c_uint64]
    L.or_sector_diag.restype = _d
    L.or_sector_diag.argtypes = [_vp, C.c_uint64, C.c_uint64]
    L.or_sector_apply.argtypes = [_vp, _vp, _vp, _i, _i]
    L.or_sector_apply_rows.argtypes = [_vp, _vp, _vp, _ll, _ll, _i]
    L.or_sector_lanczos.restype = _i
    L.or_sector_lanczos.argtypes = [_vp, _i, C.c_uint, _vp, _vp, C.POINTER(_i), _i, _i]
    L.or_sector_lanczos_extrema.restype = _i
    L.or_sector_lanczos_extrema.argtypes = [_vp, _i, C.c_uint, C.POINTER(_d), C.POINTER(_d), _i, _i]
    L.or_start_vector.argtypes = [_ll, C.c_uint, _vp]
    L.or_tridiag_eig.restype = _i
    L.or_tridiag_eig.argtypes = [_vp, _i, _vp, _i, _vp, _vp, C.POINTER(_d)]
    L.or_log_quadrature.restype = _d
    L.or_log_quadrature.argtypes = [_vp, _vp, _i, _d]
    L.or_quad_energy.restype = _d
    L.or_quad_energy.argtypes = [_vp, _vp, _i, _d]
    L.or_sector_ftlm.argtypes = [_vp, _vp, _i, _i, _i, C.c_uint, _i, _i, _vp, _vp, _vp, _vp, _vp]
    L.or_gc_reduce.argtypes = [_vp, _vp, _vp, _i, _vp, _i, _vp, _i, _i, _vp, _vp, _vp]
    L.or_geometry.restype = _i
    L.or_geometry.argtypes = [_i, _i, _d, _d, _d, _d, _i, _vp, _vp, _vp, _vp, _i, _vp, _vp, C.POINTER(_i)]
    L.or_enumerate.restype = _ll
    L.or_enumerate.argtypes = [_i, _i, _vp]
    L.or_orbit_create.restype = _vp
    L.or_orbit_create.argtypes = [_vp, _i, _i]
    L.or_orbit_destroy.argtypes = [_vp]
    L.or_orbit_dim.restype = _ll
    L.or_orbit_dim.argtypes = [_vp]
    L.or_orbit_entries.argtypes = [_vp, _vp, _vp, _vp]
    L.or_orbit_apply.argtypes = [_vp, _vp, _vp]
    L.or_orbit_ftlm.argtypes = [_vp, _vp, _i, _i, _i, C.c_uint, _vp, _vp]
    return L


def _load_ref() -> C.CDLL | None:
    if not os.path.exists(REF_SO):
        if os.path.isdir(os.path.join(REFERENCE_SRC, "src")):
            build(ref=True)
        else:
            return None
    L = C.CDLL(REF_SO)
    L.ref_sector_create.restype = _vp
    L.ref_sector_create.argtypes = [_i, _i, _d, _d, _d, _d, _d, _d, _i, _i]
    L.ref_sector_destroy.argtypes = [_vp]
    L.ref_sector_dim.restype = _ll
    L.ref_sector_dim.argtypes = [_vp]
    L.ref_sector_masks.argtypes = [_vp, _vp, _vp]
    L.ref_sector_index_of.restype = _i
    L.ref_sector_index_of.argtypes = [_vp, C.c_uint64, C.c_uint64]
    L.ref_sector_apply.argtypes = [_vp, _vp, _vp]
    L.ref_sample_create.restype = _vp
    L.ref_sample_create.argtypes = [_vp, _i]
    L.ref_sample_destroy.argtypes = [_vp]
    L.ref_sample_run.restype = _d
    L.ref_sample_run.argtypes = [_vp, _ll, _ll, C.POINTER(_ll)]
    L.ref_sector_lanczos.restype = _i
    L.ref_sector_lanczos.argtypes = [_vp, _i, C.c_uint, _vp, _vp, C.POINTER(_i)]
    L.ref_sector_lanczos_extrema.restype = _i
    L.ref_sector_lanczos_extrema.argtypes = [_vp, _i, C.c_uint, C.POINTER(_d), C.POINTER(_d)]
    L.ref_sector_ftlm_complex.restype = _d
    L.ref_sector_ftlm_complex.argtypes = [_vp, _d, _i, _i, C.c_uint]
    L.ref_sector_ftlm_real.restype = _d
    L.ref_sector_ftlm_real.argtypes = [_vp, _d, _i, _i, C.c_uint]
    L.ref_ftlm_diag_real.restype = _d
    L.ref_ftlm_diag_real.argtypes = [_vp, _i, _d, _i, _i, C.c_uint]
    L.ref_geometry.restype = _i
    L.ref_geometry.argtypes = [_i, _i, _d, _d, _d, _d, _d, _d, _i, _vp, _vp, _vp, _vp, _i, _vp, _vp, C.POINTER(_i)]
    L.ref_orbit_create.restype = _vp
    L.ref_orbit_create.argtypes = [_vp, _i, _i]
    L.ref_orbit_destroy.argtypes = [_vp]
    L.ref_orbit_dim.restype = _i
    L.ref_orbit_dim.argtypes = [_vp]
    L.ref_orbit_entries.argtypes = [_vp, _vp, _vp, _vp]
    L.ref_orbit_apply.argtypes = [_vp, _vp, _vp]
    L.ref_orbit_ftlm_complex.restype = _d
    L.ref_orbit_ftlm_complex.argtypes = [_vp, _d, _i, _i, C.c_uint]
    return L


_ORACLE = None
_REF = None


def oracle() -> C.CDLL:
    global _ORACLE
    if _ORACLE is None:
        _ORACLE = _load_oracle()
    return _ORACLE


def reference() -> C.CDLL | None:
    global _REF
    if _REF is None:
        _REF = _load_ref()
    return _REF


def have_reference() -> bool:
    return os.path.exists(REF_SO) or os.path.isdir(os.path.join(REFERENCE_SRC, "src"))


class OracleSector:
    """In-repo restatement for one sector (mode 0 = reference scatter order, 1 = threaded gather)."""

    def __init__(self, Lx, Ly, t, tp, U, V, phix, phiy, nu, nd):
        self.L = oracle()
        self.h = self.L.or_sector_create(Lx, Ly, t, tp, U, V, phix, phiy, nu, nd)
        if not self.h:
            raise ValueError("invalid sector")
        self.dim = self.L.or_sector_dim(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_sector_destroy(self.h)
            self.h = None

    def masks(self):
        up = np.zeros(self.dim, np.uint64)
        dn = np.zeros(self.dim, np.uint64)
        self.L.or_sector_masks(self.h, P(up), P(dn))
        return up, dn

    def apply(self, x, mode=0, nthreads=1):
        x = np.ascontiguousarray(x, np.complex128)
        y = np.zeros_like(x)
        self.L.or_sector_apply(self.h, P(x), P(y), mode, nthreads)
        return y

    def lanczos(self, M, seed, mode=0, nthreads=1):
        a = np.zeros(M)
        b = np.zeros(M)
        nb = _i()
        used = self.L.or_sector_lanczos(self.h, M, seed, P(a), P(b), C.byref(nb), mode, nthreads)
        return a[:used].copy(), b[:nb.value].copy(), used

    def lanczos_extrema(self, M, seed, mode=0, nthreads=1):
        mn, mx = _d(), _d()
        used = self.L.or_sector_lanczos_extrema(self.h, M, seed, C.byref(mn), C.byref(mx), mode, nthreads)
        return mn.value, mx.value, used

    def ftlm(self, betas, R, M, seed, mode=0, nthreads=1, want_chains=False):
        bt = np.ascontiguousarray(np.atleast_1d(betas), np.float64)
        lnz = np.zeros(bt.size)
        en = np.zeros(bt.size)
        if want_chains:
            lam = np.zeros(R * M)
            w = np.zeros(R * M)
            used = np.zeros(R, np.int32)
            self.L.or_sector_ftlm(self.h, P(bt), bt.size, R, M, seed, mode, nthreads, P(lnz), P(en), P(lam), P(w),
                                  P(used))
            return lnz, en, lam.reshape(R, M), w.reshape(R, M), used
        self.L.or_sector_ftlm(self.h, P(bt), bt.size, R, M, seed, mode, nthreads, P(lnz), P(en), None, None, None)
        return lnz, en


class OracleOrbit:
    """In-repo restatement of one translation-orbit momentum block (OrbitKBlockBasis + apply)."""

    def __init__(self, sector: OracleSector, kx: int, ky: int):
        self.L = sector.L
        self.sector = sector  # keeps the sector alive
        self.h = self.L.or_orbit_create(sector.h, kx, ky)
        if not self.h:
            raise ValueError("orbit blocks need n_sites <= 16")
        self.dim = self.L.or_orbit_dim(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_orbit_destroy(self.h)
            self.h = None

    def entries(self):
        rep = np.zeros(self.dim, np.uint32)
        absA = np.zeros(self.dim)
        size = np.zeros(self.dim, np.int32)
        self.L.or_orbit_entries(self.h, P(rep), P(absA), P(size))
        return rep, absA, size

    def apply(self, x):
        x = np.ascontiguousarray(x, np.complex128)
        y = np.zeros_like(x)
        self.L.or_orbit_apply(self.h, P(x), P(y))
        return y

    def ftlm(self, betas, R, M, seed):
        bt = np.ascontiguousarray(np.atleast_1d(betas), np.float64)
        lnz = np.zeros(bt.size)
        en = np.zeros(bt.size)
        self.L.or_orbit_ftlm(self.h, P(bt), bt.size, R, M, seed, P(lnz), P(en))
        return lnz, en


def start_vector(dim: int, seed: int) -> np.ndarray:
    q = np.zeros(dim, np.complex128)
    oracle().or_start_vector(dim, seed, P(q))
    return q


def tridiag_eig(alpha, beta):
    n = len(alpha)
    a = np.ascontiguousarray(alpha, np.float64)
    b = np.ascontiguousarray(beta if len(beta) else np.zeros(1), np.float64)
    lam = np.zeros(max(n, 1))
    w = np.zeros(max(n, 1))
    off = _d()
    rot = oracle().or_tridiag_eig(P(a), n, P(b), len(beta), P(lam), P(w), C.byref(off))
    return lam[:n], w[:n], rot, off.value


def gc_reduce(lnz_s, e_s, N_s, betas, mus, n_sites):
    lnz_s = np.ascontiguousarray(lnz_s, np.float64)
    e_s = np.ascontiguousarray(e_s, np.float64)
    N = np.ascontiguousarray(N_s, np.int32)
    bt = np.ascontiguousarray(betas, np.float64)
    mu = np.ascontiguousarray(mus, np.float64)
    o1 = np.zeros((bt.size, mu.size))
    o2 = np.zeros_like(o1)
    o3 = np.zeros_like(o1)
    oracle().or_gc_reduce(P(lnz_s), P(e_s), P(N), N.size, P(bt), bt.size, P(mu), mu.size, n_sites, P(o1), P(o2),
                          P(o3))
    return o1, o2, o3


def oracle_sweep(Lx, Ly, t, tp, U, V, phix, phiy, R, M, seed, betas, mus, mode=0, nthreads=1):
    """Plain FTLM over all sectors + the GC grid (restated bench_ftlm_nmu_rect.cpp:138-219)."""
    n = Lx * Ly
    bt = np.atleast_1d(betas).astype(np.float64)
    nsec = (n + 1) ** 2
    lz = np.zeros((nsec, bt.size))
    es = np.zeros((nsec, bt.size))
    N = np.zeros(nsec, np.int32)
    dims = np.zeros(nsec, np.int64)
    for nu in range(n + 1):
        for nd in range(n + 1):
            idx = nu * (n + 1) + nd
            s = OracleSector(Lx, Ly, t, tp, U, V, phix, phiy, nu, nd)
            N[idx] = nu + nd
            dims[idx] = s.dim
            lz[idx], es[idx] = s.ftlm(bt, R, M, seed, mode, nthreads)
    g = gc_reduce(lz, es, N, bt, mus, n)
    return lz, es, N, dims, g
