"""Python host API mirroring the reference's C++ interface for the FTLM hot path.

Reference (PeizhiMai/FTLM_extended_Hubbard) names kept:
  HubbardParams, nsites            include/ftlm/hubbard_params.hpp:6-17
  SpinfulHopping, NearestPair,
  RectLattice, build_hubbard_geometry   include/ftlm/lattice.hpp:11-40
  FockBasis                        include/ftlm/fock_basis.hpp:11-35
  apply_extended_hubbard           include/ftlm/hubbard_hamiltonian.hpp:13-16
  lanczos_tridiagonal, lanczos_extrema, LanczosExtrema   include/ftlm/lanczos.hpp:39-59
  FtlmParams, ftlm_log_partition_complex/_real           include/ftlm/ftlm_thermo.hpp:22-50
Errors follow the reference: invalid sectors raise ValueError (std::invalid_argument);
sentinels (-inf ln Z for empty input, index_of == -1) are kept.  Every compute call goes to
the native library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np

from ._lib import APPLY_FN, FTLM_ERR_INVALID, FTLM_START_PHILOX, FTLM_START_REFERENCE, FtlmError, FtlmHop, FtlmPair
from ._lib import FtlmParams as _CParams
from ._lib import call, lib

START_MODES = {"reference": FTLM_START_REFERENCE, "philox": FTLM_START_PHILOX}


@dataclass
class HubbardParams:
    Lx: int = 2
    Ly: int = 2
    t: float = 1.0
    tp: float = 0.0
    U: float = 0.0
    V: float = 0.0
    phi_x: float = 0.0
    phi_y: float = 0.0

    def _c(self) -> _CParams:
        return _CParams(self.Lx, self.Ly, self.t, self.tp, self.U, self.V, self.phi_x, self.phi_y)


def nsites(p: HubbardParams) -> int:
    return p.Lx * p.Ly


def version_string() -> str:
    return lib().ftlm_gpu_version_string().decode()


@dataclass(frozen=True)
class SpinfulHopping:
    """H += coeff c^dag_to c_from for one spin (0 = up, 1 = down)."""
    from_: int
    to: int
    spin: int
    coeff: complex


@dataclass(frozen=True)
class NearestPair:
    i: int
    j: int


@dataclass
class RectLattice:
    Lx: int = 1
    Ly: int = 1

    def n_sites(self) -> int:
        return self.Lx * self.Ly

    def site_index(self, x: int, y: int) -> int:
        return y * self.Lx + x


def build_hubbard_geometry(p: HubbardParams, lat: Optional[RectLattice] = None):
    """Directed hoppings and NN pairs exactly as the reference's build_hubbard_geometry."""
    q = HubbardParams(**{**p.__dict__})
    if lat is not None:
        q.Lx, q.Ly = lat.Lx, lat.Ly
    nh, npair = C.c_int(), C.c_int()
    call("ftlm_gpu_build_geometry", C.byref(q._c()), None, 0, C.byref(nh), None, 0, C.byref(npair))
    hops = (FtlmHop * max(1, nh.value))()
    pairs = (FtlmPair * max(1, npair.value))()
    call("ftlm_gpu_build_geometry", C.byref(q._c()), hops, nh.value, C.byref(nh), pairs, npair.value,
         C.byref(npair))
    H = [SpinfulHopping(h.frm, h.to, h.spin, complex(h.coeff_re, h.coeff_im)) for h in hops[:nh.value]]
    P = [NearestPair(x.i, x.j) for x in pairs[:npair.value]]
    return H, P


def _c_hops(hops: Sequence[SpinfulHopping]):
    arr = (FtlmHop * max(1, len(hops)))()
    for k, h in enumerate(hops):
        arr[k] = FtlmHop(h.from_, h.to, h.spin, complex(h.coeff).real, complex(h.coeff).imag)
    return arr


def _c_pairs(pairs: Sequence[NearestPair]):
    arr = (FtlmPair * max(1, len(pairs)))()
    for k, pr in enumerate(pairs):
        arr[k] = FtlmPair(pr.i, pr.j)
    return arr


def _raise_value(e: FtlmError):
    if e.code == FTLM_ERR_INVALID:
        raise ValueError(str(e)) from None
    raise e


class _Handle:
    _destroy = "ftlm_gpu_sector_destroy"

    def __init__(self):
        self._h = C.c_void_p()

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().ftlm_gpu_sector_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def dim(self) -> int:
        d = C.c_longlong()
        call("ftlm_gpu_sector_dim", self._h, C.byref(d))
        return d.value

    def index_of(self, up: int, down: int) -> int:
        r = C.c_longlong()
        call("ftlm_gpu_sector_index_of", self._h, C.c_uint64(up), C.c_uint64(down), C.byref(r))
        return r.value

    def masks(self):
        n = self.dim()
        up = np.zeros(n, np.uint64)
        dn = np.zeros(n, np.uint64)
        call("ftlm_gpu_sector_masks", self._h, up.ctypes.data_as(C.c_void_p), dn.ctypes.data_as(C.c_void_p))
        return up, dn

    def stats(self):
        mu, md = C.c_double(), C.c_double()
        du, dd = C.c_longlong(), C.c_longlong()
        call("ftlm_gpu_sector_stats", self._h, C.byref(mu), C.byref(md), C.byref(du), C.byref(dd))
        return {"mean_up_sources": mu.value, "mean_dn_sources": md.value, "Du": du.value, "Dd": dd.value}


class FockBasis(_Handle):
    """Fixed (N_up, N_down) sector basis; host tables only (no GPU needed)."""

    def __init__(self, n_sites: int, n_up: int, n_down: int):
        super().__init__()
        self._n, self._nu, self._nd = n_sites, n_up, n_down
        try:
            call("ftlm_gpu_sector_create_host", n_sites, n_up, n_down, 0.0, 0.0, None, 0, None, 0,
                 C.byref(self._h))
        except FtlmError as e:
            _raise_value(e)
        self._up, self._dn = None, None

    def n_sites(self):
        return self._n

    def n_up(self):
        return self._nu

    def n_down(self):
        return self._nd

    def _ensure_masks(self):
        if self._up is None:
            self._up, self._dn = self.masks()

    def up_mask(self, idx: int) -> int:
        self._ensure_masks()
        return int(self._up[idx])

    def down_mask(self, idx: int) -> int:
        self._ensure_masks()
        return int(self._dn[idx])


def _ptr(x) -> int:
    """Device pointer of a torch tensor (complex128/float64, contiguous) or an int."""
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return x.data_ptr()
    raise TypeError("expected a torch tensor or a device pointer")


class Sector(_Handle):
    """One (N_up, N_dn) sector of the extended Hubbard Hamiltonian with its device tables."""

    def __init__(self, p: Optional[HubbardParams], n_up: int, n_down: int, *, hops=None, pairs=None,
                 n_sites: Optional[int] = None, U: Optional[float] = None, V: Optional[float] = None):
        super().__init__()
        self.params = p
        try:
            if hops is None:
                call("ftlm_gpu_sector_create", C.byref(p._c()), n_up, n_down, C.byref(self._h))
            else:
                ns = n_sites if n_sites is not None else nsites(p)
                uu = U if U is not None else p.U
                vv = V if V is not None else p.V
                call("ftlm_gpu_sector_create_hops", ns, n_up, n_down, uu, vv, _c_hops(hops), len(hops),
                     _c_pairs(pairs or []), len(pairs or []), C.byref(self._h))
        except FtlmError as e:
            _raise_value(e)
        self.n_up, self.n_down = n_up, n_down

    def set_apply_path(self, path: int):
        call("ftlm_gpu_set_apply_path", self._h, path)

    def autotune(self, reps: int = 3):
        """Time the H·v variants of this sector shape and keep the fastest: (path, cols_variant, ms per
        H·v; -1 when the shape's answer was cached)."""
        pth, var, ms = C.c_int(), C.c_int(), C.c_float()
        call("ftlm_gpu_autotune_apply", self._h, reps, C.byref(pth), C.byref(var), C.byref(ms))
        return pth.value, var.value, ms.value

    def apply(self, x, y, stream: int = 0):
        """y = H x on device (torch complex128 tensors or pointers)."""
        call("ftlm_gpu_apply", self._h, C.c_void_p(_ptr(x)), C.c_void_p(_ptr(y)), C.c_void_p(stream))

    def apply_host(self, x: np.ndarray, y: Optional[np.ndarray] = None) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.complex128)
        if y is None:
            y = np.empty_like(x)
        call("ftlm_gpu_apply_host", self._h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p))
        return y

    def lanczos(self, max_steps: int, seed: int, start: str = "reference"):
        a = np.zeros(max(1, max_steps))
        b = np.zeros(max(1, max_steps))
        nb, used = C.c_int(), C.c_int()
        call("ftlm_gpu_lanczos", self._h, max_steps, C.c_uint(seed & 0xFFFFFFFF), START_MODES[start],
             a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), C.byref(nb), C.byref(used))
        return a[:used.value].copy(), b[:nb.value].copy(), used.value

    def lanczos_extrema(self, max_steps: int, seed: int = 1, start: str = "reference"):
        mn, mx, used = C.c_double(), C.c_double(), C.c_int()
        call("ftlm_gpu_lanczos_extrema", self._h, max_steps, C.c_uint(seed & 0xFFFFFFFF), START_MODES[start],
             C.byref(mn), C.byref(mx), C.byref(used))
        return LanczosExtrema(mn.value, mx.value, used.value)

    def ftlm(self, betas, n_random: int, lanczos_steps: int, seed: int, start: str = "reference"):
        bt = np.ascontiguousarray(np.atleast_1d(np.asarray(betas, dtype=np.float64)))
        lnz = np.zeros(bt.size)
        en = np.zeros(bt.size)
        call("ftlm_gpu_ftlm_sector", self._h, bt.ctypes.data_as(C.c_void_p), bt.size, n_random, lanczos_steps,
             C.c_uint(seed & 0xFFFFFFFF), START_MODES[start], lnz.ctypes.data_as(C.c_void_p),
             en.ctypes.data_as(C.c_void_p))
        return lnz, en


    def batched_set_cols_variant(self, variant: int):
        """Column-pass variant of the batched H·v: 0/1/2 = 16/8/4-column chunks."""
        call("ftlm_gpu_batched_set_cols_variant", self._h, variant)

    def batched_autotune(self, reps: int = 2):
        """Time the batched column-pass variants and keep the fastest: (variant, ms per block H·v;
        -1 when the shape's answer was cached)."""
        var, ms = C.c_int(), C.c_float()
        call("ftlm_gpu_batched_autotune", self._h, reps, C.byref(var), C.byref(ms))
        return var.value, ms.value

    def batched_lanczos(self, n_random: int, lanczos_steps: int, seed: int):
        """32-chain complex64 Lanczos: alpha/beta [R][M] (beta zero-padded), used [R]."""
        R, M = n_random, lanczos_steps
        a = np.zeros((R, M))
        b = np.zeros((R, M))
        u = np.zeros(R, np.int32)
        call("ftlm_gpu_batched_lanczos", self._h, R, M, C.c_uint(seed & 0xFFFFFFFF), a.ctypes.data_as(C.c_void_p),
             b.ctypes.data_as(C.c_void_p), u.ctypes.data_as(C.c_void_p))
        return a, b, u

    def batched_ftlm(self, betas, n_random: int, lanczos_steps: int, seed: int, check: int = 0):
        """Batched complex64 sector FTLM: (ln Z, E); with check > 0 also the estimated rounding error
        of ln Z against complex128 (chains r < check rerun in complex128): (ln Z, E, err)."""
        bt = np.ascontiguousarray(np.atleast_1d(np.asarray(betas, dtype=np.float64)))
        lnz = np.zeros(bt.size)
        en = np.zeros(bt.size)
        if check > 0:
            err = np.zeros(bt.size)
            call("ftlm_gpu_batched_ftlm_sector_checked", self._h, bt.ctypes.data_as(C.c_void_p), bt.size, n_random,
                 lanczos_steps, C.c_uint(seed & 0xFFFFFFFF), int(check), lnz.ctypes.data_as(C.c_void_p),
                 en.ctypes.data_as(C.c_void_p), err.ctypes.data_as(C.c_void_p))
            return lnz, en, err
        call("ftlm_gpu_batched_ftlm_sector", self._h, bt.ctypes.data_as(C.c_void_p), bt.size, n_random,
             lanczos_steps, C.c_uint(seed & 0xFFFFFFFF), lnz.ctypes.data_as(C.c_void_p), en.ctypes.data_as(C.c_void_p))
        return lnz, en


    def ftlm_grad(self, beta: float, n_random: int, lanczos_steps: int, seed: int, op_tp: Optional["Sector"] = None,
                  method: str = "plain", start: str = "reference"):
        """Sector ln Z estimate at inverse temperature beta and its derivatives with respect to
        (U, V, t') with the start vectors held fixed, from a replay of the forward's chains
        (method "plain" = ftlm(start=...), "batched" = batched_ftlm).  op_tp: the same sector built
        with t=0, t'=1, U=V=0 (dH/dt'); without it the t' derivative is 0."""
        lnz = C.c_double()
        d = np.zeros(3)
        call("ftlm_gpu_grad_sector", self._h, op_tp.handle if op_tp is not None else None, float(beta), n_random,
             lanczos_steps, C.c_uint(seed & 0xFFFFFFFF), {"plain": 0, "batched": 1}[method], START_MODES[start],
             C.byref(lnz), d.ctypes.data_as(C.c_void_p))
        return lnz.value, d

    def orbit_block(self, kx: int, ky: int) -> "OrbitKBlock":
        return OrbitKBlock(self, kx, ky)

    def orbit_ftlm(self, betas, n_random: int, lanczos_steps: int, seed: int, sector_index: int = 0,
                   start: str = "reference", ed_cutoff: int = 64, method: str = "plain"):
        """k-resolved sector ln Z: blocks of dim <= ed_cutoff exactly, larger ones by FTLM with
        seed + sector_index*257 + ky*17 + kx, log-sum-exp over blocks (the k-bench's rule; its
        --ed-cutoff defaults to 64).  method "batched": complex64 32-chain blocks (Philox starts).
        Returns (lnz, energy, block dims [Ly][Lx])."""
        bt = np.ascontiguousarray(np.atleast_1d(np.asarray(betas, dtype=np.float64)))
        lnz = np.zeros(bt.size)
        en = np.zeros(bt.size)
        Lx, Ly = (self.params.Lx, self.params.Ly) if self.params is not None else (0, 0)
        dims = np.zeros(max(1, Lx * Ly), np.int64)
        if method == "batched":
            call("ftlm_gpu_orbit_sector_batched_ftlm", self._h, bt.ctypes.data_as(C.c_void_p), bt.size, n_random,
                 lanczos_steps, C.c_uint(seed & 0xFFFFFFFF), sector_index, ed_cutoff, lnz.ctypes.data_as(C.c_void_p),
                 en.ctypes.data_as(C.c_void_p), dims.ctypes.data_as(C.c_void_p))
        else:
            call("ftlm_gpu_orbit_sector_ftlm", self._h, bt.ctypes.data_as(C.c_void_p), bt.size, n_random,
                 lanczos_steps, C.c_uint(seed & 0xFFFFFFFF), sector_index, START_MODES[start], ed_cutoff,
                 lnz.ctypes.data_as(C.c_void_p), en.ctypes.data_as(C.c_void_p), dims.ctypes.data_as(C.c_void_p))
        return lnz, en, dims[:Lx * Ly].reshape(Ly, Lx)


class OrbitKBlock:
    """Translation-orbit momentum block K = (kx, ky) of a sector (OrbitKBlockBasis + apply_orbit_k_block)."""

    def __init__(self, sector: Sector, kx: int, ky: int):
        self.sector = sector  # the block's device tables reference the sector's
        self._h = C.c_void_p()
        try:
            call("ftlm_gpu_orbit_create", sector.handle, kx, ky, C.byref(self._h))
        except FtlmError as e:
            _raise_value(e)
        d = C.c_longlong()
        call("ftlm_gpu_orbit_dim", self._h, C.byref(d))
        self.dim = d.value
        self.kx, self.ky = kx, ky

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().ftlm_gpu_orbit_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_apply_path(self, path: int):
        call("ftlm_gpu_orbit_set_apply_path", self._h, path)

    def entries(self):
        """Packed representatives (up<<16 | dn) and |A(K)|, ascending packed order."""
        rep = np.zeros(max(1, self.dim), np.uint32)
        absA = np.zeros(max(1, self.dim))
        call("ftlm_gpu_orbit_entries", self._h, rep.ctypes.data_as(C.c_void_p), absA.ctypes.data_as(C.c_void_p))
        return rep[:self.dim], absA[:self.dim]

    def apply(self, x, y, stream: int = 0):
        call("ftlm_gpu_orbit_apply", self._h, C.c_void_p(_ptr(x)), C.c_void_p(_ptr(y)), C.c_void_p(stream))

    def apply_host(self, x: np.ndarray, y: Optional[np.ndarray] = None) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.complex128)
        if y is None:
            y = np.empty_like(x)
        call("ftlm_gpu_orbit_apply_host", self._h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p))
        return y

    def batched_ftlm(self, betas, n_random: int, lanczos_steps: int, seed: int):
        bt = np.ascontiguousarray(np.atleast_1d(np.asarray(betas, dtype=np.float64)))
        lnz = np.zeros(bt.size)
        en = np.zeros(bt.size)
        call("ftlm_gpu_orbit_batched_ftlm", self._h, bt.ctypes.data_as(C.c_void_p), bt.size, n_random, lanczos_steps,
             C.c_uint(seed & 0xFFFFFFFF), lnz.ctypes.data_as(C.c_void_p), en.ctypes.data_as(C.c_void_p))
        return lnz, en

    def ftlm(self, betas, n_random: int, lanczos_steps: int, seed: int, start: str = "reference"):
        bt = np.ascontiguousarray(np.atleast_1d(np.asarray(betas, dtype=np.float64)))
        lnz = np.zeros(bt.size)
        en = np.zeros(bt.size)
        call("ftlm_gpu_orbit_ftlm", self._h, bt.ctypes.data_as(C.c_void_p), bt.size, n_random, lanczos_steps,
             C.c_uint(seed & 0xFFFFFFFF), START_MODES[start], lnz.ctypes.data_as(C.c_void_p),
             en.ctypes.data_as(C.c_void_p))
        return lnz, en


def lanczos_sectors(sectors, n_random: int, lanczos_steps: int, seed: int, start: str = "reference"):
    """The Lanczos chains of several sectors in one launch (one CTA per chain; for small sectors):
    alpha/beta [len(sectors)*R][M] (zero-padded), used [len(sectors)*R]; chain r of a sector uses
    seed + r*100003 as Sector.lanczos."""
    R, M = n_random, lanczos_steps
    hs = (C.c_void_p * max(1, len(sectors)))(*[sec.handle.value for sec in sectors])
    A = np.zeros((len(sectors) * R, M))
    B = np.zeros((len(sectors) * R, M))
    u = np.zeros(len(sectors) * R, np.int32)
    if sectors:
        call("ftlm_gpu_lanczos_sectors", hs, len(sectors), R, M, C.c_uint(seed & 0xFFFFFFFF), START_MODES[start],
             A.ctypes.data_as(C.c_void_p), B.ctypes.data_as(C.c_void_p), u.ctypes.data_as(C.c_void_p))
    return A, B, u


@dataclass
class LanczosExtrema:
    min_eval: float = 0.0
    max_eval: float = 0.0
    steps_used: int = 0


@dataclass
class FtlmParams:
    n_random: int = 16
    lanczos_steps: int = 96
    seed: int = 1
    start: str = "reference"


_SECTOR_CACHE: dict = {}


def _sector_for(p: HubbardParams, basis: FockBasis, hops, pairs) -> Sector:
    key = (basis.n_sites(), basis.n_up(), basis.n_down(), p.U, p.V,
           tuple((h.from_, h.to, h.spin, complex(h.coeff)) for h in hops), tuple((q.i, q.j) for q in pairs))
    s = _SECTOR_CACHE.get(key)
    if s is None:
        if len(_SECTOR_CACHE) > 8:
            _SECTOR_CACHE.clear()
        s = Sector(p, basis.n_up(), basis.n_down(), hops=list(hops), pairs=list(pairs), n_sites=basis.n_sites())
        _SECTOR_CACHE[key] = s
    return s


def apply_extended_hubbard(p: HubbardParams, basis: FockBasis, hops, pairs, x, y) -> None:
    """y = H x with host (numpy complex128) buffers; y is overwritten (reference semantics)."""
    s = _sector_for(p, basis, hops, pairs)
    if isinstance(x, np.ndarray):
        out = s.apply_host(x)
        y[...] = out
    else:
        s.apply(x, y)


def _op_lanczos(dim: int, apply_h: Callable, max_steps: int, seed: int, start: str):
    """Lanczos with a caller operator on device buffers: apply_h(x_ptr, y_ptr)."""
    def cb(x, y, ctx):
        apply_h(int(x), int(y))

    fn = APPLY_FN(cb)
    a = np.zeros(max(1, max_steps))
    b = np.zeros(max(1, max_steps))
    nb, used = C.c_int(), C.c_int()
    call("ftlm_gpu_lanczos_op", C.c_longlong(dim), fn, None, max_steps, C.c_uint(seed & 0xFFFFFFFF),
         START_MODES[start], a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), C.byref(nb),
         C.byref(used))
    return a[:used.value].copy(), b[:nb.value].copy(), used.value


def lanczos_tridiagonal(dim_or_sector, apply_h=None, max_steps: int = 0, seed: int = 1, start: str = "reference"):
    """(alpha, beta, steps_used); beta keeps the last entry as the reference does."""
    if isinstance(dim_or_sector, Sector):
        return dim_or_sector.lanczos(max_steps, seed, start)
    if int(dim_or_sector) <= 0 or max_steps <= 0:
        return np.zeros(0), np.zeros(0), 0
    return _op_lanczos(int(dim_or_sector), apply_h, max_steps, seed, start)


def batched_release():
    """Frees the batched path's block vectors (kept between calls otherwise)."""
    call("ftlm_gpu_batched_release")


QUADRATURES = {"reference": 0, "converged": 1}


def set_quadrature(mode: str) -> None:
    """Quadrature of the complex128 sector path: "reference" (default; the reference's rotation-capped
    Jacobi, src/ftlm_thermo.cpp:83-146) or "converged" (the converged GPU Jacobi, which the batched
    complex64 path always uses).  Process-wide."""
    call("ftlm_gpu_set_quadrature", QUADRATURES[mode])


class quadrature:
    """Context manager: `with quadrature("converged"): ...` sets the complex128 path's quadrature and
    restores the reference quadrature on exit."""

    def __init__(self, mode: str):
        self.mode = mode

    def __enter__(self):
        set_quadrature(self.mode)
        return self

    def __exit__(self, *exc):
        set_quadrature("reference")
        return False


def tridiag_eig(alpha: np.ndarray, beta: np.ndarray, n: np.ndarray, max_rot: int = 0, tol: float = 1e-14):
    """Batched reference Jacobi: alpha/beta [chains][ld] -> (lam, w0) [chains][ld]."""
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    b = np.ascontiguousarray(beta, dtype=np.float64)
    nn = np.ascontiguousarray(n, dtype=np.int32)
    lam = np.zeros_like(a)
    w0 = np.zeros_like(a)
    call("ftlm_gpu_tridiag_eig", a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p),
         nn.ctypes.data_as(C.c_void_p), a.shape[0], a.shape[1], max_rot, tol, lam.ctypes.data_as(C.c_void_p),
         w0.ctypes.data_as(C.c_void_p))
    return lam, w0


def tridiag_quadrature(alpha, beta, n, betas):
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    b = np.ascontiguousarray(beta, dtype=np.float64)
    nn = np.ascontiguousarray(n, dtype=np.int32)
    bt = np.ascontiguousarray(np.atleast_1d(betas), dtype=np.float64)
    lq = np.zeros((a.shape[0], bt.size))
    eq = np.zeros((a.shape[0], bt.size))
    call("ftlm_gpu_tridiag_quadrature", a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p),
         nn.ctypes.data_as(C.c_void_p), a.shape[0], a.shape[1], bt.ctypes.data_as(C.c_void_p), bt.size,
         lq.ctypes.data_as(C.c_void_p), eq.ctypes.data_as(C.c_void_p))
    return lq, eq


def ritz_values(alpha, beta, k: int):
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    b = np.ascontiguousarray(beta, dtype=np.float64)
    k = min(k, a.size)
    out = np.zeros(k)
    call("ftlm_gpu_ritz_values", a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), a.size, k,
         out.ctypes.data_as(C.c_void_p))
    return out


def lanczos_extrema(dim_or_sector, apply_h=None, max_steps: int = 0, seed: int = 1, start: str = "reference"):
    if isinstance(dim_or_sector, Sector):
        return dim_or_sector.lanczos_extrema(max_steps, seed, start)
    a, b, used = lanczos_tridiagonal(dim_or_sector, apply_h, max_steps, seed, start)
    if used == 0:
        return LanczosExtrema(0.0, 0.0, 0)
    if used == 1:
        return LanczosExtrema(a[0], a[0], 1)
    bt = np.zeros(used)
    bt[:used - 1] = b[:used - 1]
    lam, _ = tridiag_eig(a[None, :], bt[None, :], np.array([used]), max_rot=120, tol=1e-15)
    return LanczosExtrema(float(lam.min()), float(lam.max()), used)


def ftlm_log_partition_complex(dim_or_sector, apply_h=None, beta: float = 1.0, par: FtlmParams = FtlmParams()):
    """ln Tr e^{-beta H} (scalar beta or array of betas)."""
    scalar = np.ndim(beta) == 0
    if isinstance(dim_or_sector, Sector):
        lnz, _ = dim_or_sector.ftlm(beta, par.n_random, par.lanczos_steps, par.seed, par.start)
        return float(lnz[0]) if scalar else lnz
    dim = int(dim_or_sector)
    bts = np.atleast_1d(np.asarray(beta, dtype=np.float64))
    if dim <= 0:
        out = np.full(bts.size, -np.inf)
        return float(out[0]) if scalar else out
    if dim == 1:
        import torch
        x = torch.tensor([1.0 + 0j], dtype=torch.complex128, device="cuda")
        y = torch.zeros_like(x)
        apply_h(x.data_ptr(), y.data_ptr())
        out = -bts * float(y[0].real)
        return float(out[0]) if scalar else out
    R, M = max(1, par.n_random), max(1, par.lanczos_steps)
    A = np.zeros((R, M))
    B = np.zeros((R, M))
    n = np.zeros(R, np.int32)
    for r in range(R):
        a, b, used = _op_lanczos(dim, apply_h, M, (par.seed + r * 100003) & 0xFFFFFFFF, par.start)
        A[r, :used] = a
        B[r, :len(b)] = b
        n[r] = used
    lq, _ = tridiag_quadrature(A, B, n, bts)
    ok = n > 0
    if not ok.any():
        out = np.full(bts.size, -np.inf)
    else:
        L = lq[ok]
        mx = L.max(axis=0)
        out = math.log(dim) + mx + np.log(np.exp(L - mx).sum(axis=0) / ok.sum())
    return float(out[0]) if scalar else out


ftlm_log_partition_real = ftlm_log_partition_complex


@dataclass
class SweepResult:
    temperatures: np.ndarray
    betas: np.ndarray
    mus: np.ndarray
    lnz_sector: np.ndarray  # [n_sec][n_T]
    e_sector: np.ndarray
    lnz_gc: np.ndarray  # [n_T][n_mu]
    n_avg: np.ndarray
    e_avg: np.ndarray
    N_sector: np.ndarray = field(default_factory=lambda: np.zeros(0))
    # batched method with check > 0: estimated rounding errors against the complex128 path
    lnz_sector_err: Optional[np.ndarray] = None  # [n_sec][n_T]
    lnz_gc_err: Optional[np.ndarray] = None  # [n_T][n_mu]
    n_err: Optional[np.ndarray] = None


def grand_canonical_sweep(p: HubbardParams, n_random: int, lanczos_steps: int, seed: int, temperatures, mus,
                          start: str = "reference", method: str = "plain", check: int = 0) -> SweepResult:
    """Every (N_up, N_dn) sector, R chains each, then the (T, mu) grid.

    method "plain": complex128, one chain at a time (start "reference" or "philox");
    method "batched": complex64 block vectors of 32 chains, Philox starts (see ftlm_gpu.h); with
    check > 0 the first `check` chains of every sector are rerun in complex128 and the result carries
    the estimated rounding error of each sector ln Z, of ln Z_GC and of <n>."""
    T = np.ascontiguousarray(np.atleast_1d(temperatures), dtype=np.float64)
    bts = np.ascontiguousarray(1.0 / T)
    mu = np.ascontiguousarray(np.atleast_1d(mus), dtype=np.float64)
    n = nsites(p)
    nsec = (n + 1) ** 2
    lz = np.zeros((nsec, bts.size))
    es = np.zeros((nsec, bts.size))
    g1 = np.zeros((bts.size, mu.size))
    g2 = np.zeros_like(g1)
    g3 = np.zeros_like(g1)
    outs = [x.ctypes.data_as(C.c_void_p) for x in (lz, es, g1, g2, g3)]
    errs = None
    if method == "batched" and check > 0:
        errs = (np.zeros((nsec, bts.size)), np.zeros((bts.size, mu.size)), np.zeros((bts.size, mu.size)))
        call("ftlm_gpu_batched_sweep_checked", C.byref(p._c()), n_random, lanczos_steps, C.c_uint(seed & 0xFFFFFFFF),
             bts.ctypes.data_as(C.c_void_p), bts.size, mu.ctypes.data_as(C.c_void_p), mu.size, int(check), *outs,
             *[x.ctypes.data_as(C.c_void_p) for x in errs])
    elif method == "batched":
        call("ftlm_gpu_batched_sweep", C.byref(p._c()), n_random, lanczos_steps, C.c_uint(seed & 0xFFFFFFFF),
             bts.ctypes.data_as(C.c_void_p), bts.size, mu.ctypes.data_as(C.c_void_p), mu.size, *outs)
    else:
        call("ftlm_gpu_gc_sweep", C.byref(p._c()), n_random, lanczos_steps, C.c_uint(seed & 0xFFFFFFFF),
             START_MODES[start], bts.ctypes.data_as(C.c_void_p), bts.size, mu.ctypes.data_as(C.c_void_p), mu.size,
             *outs)
    N = np.array([nu + nd for nu in range(n + 1) for nd in range(n + 1)])
    r = SweepResult(T, bts, mu, lz, es, g1, g2, g3, N)
    if errs is not None:
        r.lnz_sector_err, r.lnz_gc_err, r.n_err = errs
    return r
