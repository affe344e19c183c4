"""Differentiable grand-canonical FTLM: ln Z_GC(U, V, t', mu, beta) as a torch.autograd.Function.

Forward: every (N_up, N_dn) sector's FTLM ln Z_s at beta (batched complex64 chains, or the plain
complex128 chains with the reference's start vectors; the tridiagonal quadrature from a converged
eigen-decomposition, which the gradient differentiates exactly), combined as
    ln Z_GC = log sum_s exp(ln Z_s + beta mu N_s)
(the grand-canonical reduction of benchmarks/bench_ftlm_nmu_rect.cpp:186-219 at one (T, mu)).
Only per-sector ln Z_s and energies are kept; no Krylov vector outlives the forward.

Backward (the reference has no derivatives):
    d/dmu   = beta <N>,
    d/dbeta = <mu N - E>          (E_s: the FTLM energy of the same quadrature, exact derivative),
    d/dtheta for theta in (U, V, t'): sum_s w_s d ln Z_s/dtheta, w_s = exp(ln Z_s + beta mu N_s - ln Z_GC),
where d ln Z_s/dtheta re-runs the sector's chains from their seed on the GPU
(ftlm_gpu_grad_sector: Duhamel derivative in each chain's Krylov space, start vectors fixed).
Sectors with w_s < 1e-13 are skipped (their term is below 1e-13 * beta * n_sites).  The sector loop,
quadrature and combination run in the native library (ftlm_gpu_gc_logz / ftlm_gpu_gc_logz_grad).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

import ctypes as C

from ._lib import FTLM_START_PHILOX, FTLM_START_REFERENCE, call
from .api import HubbardParams

START_MODES = {"reference": FTLM_START_REFERENCE, "philox": FTLM_START_PHILOX}


@dataclass(frozen=True)
class Lattice:
    Lx: int
    Ly: int
    t: float = 1.0
    phi_x: float = 0.0
    phi_y: float = 0.0


METHODS = {"plain": 0, "batched": 1}


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _params(lat: Lattice, U, V, tp) -> HubbardParams:
    return HubbardParams(lat.Lx, lat.Ly, lat.t, float(tp), float(U), float(V), lat.phi_x, lat.phi_y)


def sector_table(lat: Lattice, theta, R, M, seed, method="batched", start="reference"):
    """ln Z_s, E_s, N_s for every sector at theta = (U, V, t', mu, beta), and ln Z_GC (ftlm_gpu_gc_logz).
    Chains as the forward FTLM calls make them: method "batched" = complex64 32-chain blocks (sectors
    with dim <= 2M on the complex128 Philox path), "plain" = complex128 with `start`; the small
    sectors' chains in one fused launch; converged tridiagonal quadrature."""
    U, V, tp, mu, beta = (float(v) for v in theta)
    n = lat.Lx * lat.Ly
    nsec = (n + 1) ** 2
    lnz = np.zeros(nsec)
    en = np.zeros(nsec)
    gc = C.c_double()
    pc = _params(lat, U, V, tp)._c()
    call("ftlm_gpu_gc_logz", C.byref(pc), mu, beta, int(R), int(M), C.c_uint(seed & 0xFFFFFFFF), METHODS[method],
         START_MODES[start], _p(lnz), _p(en), C.byref(gc))
    N = np.array([nu + nd for nu in range(n + 1) for nd in range(n + 1)], dtype=np.float64)
    return lnz, en, N, gc.value


def sector_table_grad(lat: Lattice, theta, R, M, seed, lnz, en, method="batched", start="reference"):
    """d ln Z_GC / d(U, V, t', mu, beta) from the forward's sector table (ftlm_gpu_gc_logz_grad)."""
    U, V, tp, mu, beta = (float(v) for v in theta)
    g = np.zeros(5)
    lnz = np.ascontiguousarray(lnz, np.float64)
    en = np.ascontiguousarray(en, np.float64)
    pc = _params(lat, U, V, tp)._c()
    call("ftlm_gpu_gc_logz_grad", C.byref(pc), mu, beta, int(R), int(M), C.c_uint(seed & 0xFFFFFFFF),
         METHODS[method], START_MODES[start], _p(lnz), _p(en), _p(g))
    return g


def _lse(x):
    m = np.max(x)
    return float(m + np.log(np.sum(np.exp(x - m))))


def grand_canonical_logz_value(lat: Lattice, theta, R, M, seed, method="batched", start="reference") -> float:
    return sector_table(lat, theta, R, M, seed, method, start)[3]


def gc_combine(lnz, en, N, mu: float, beta: float):
    """ln Z_GC = log sum_s exp(ln Z_s + beta mu N_s) and the parts of its gradient that need no chain
    replay: the sector weights w_s, d/dmu = beta <N> and d/dbeta = <mu N - E> (E_s: the FTLM energy
    of the same quadrature, which is -d ln Z_s / d beta exactly)."""
    lnz = np.asarray(lnz, dtype=np.float64)
    x = lnz + beta * mu * np.asarray(N, dtype=np.float64)
    lnZ = _lse(x)
    w = np.exp(x - lnZ)
    dmu = beta * float(np.sum(w * N))
    dbeta = float(np.sum(w * (mu * np.asarray(N, dtype=np.float64) - np.asarray(en, dtype=np.float64))))
    return lnZ, w, dmu, dbeta


class GrandCanonicalLogZ(torch.autograd.Function):
    """theta: float64 tensor (U, V, t', mu, beta).  Returns the scalar ln Z_GC."""

    @staticmethod
    def forward(ctx, theta, lat: Lattice, R: int, M: int, seed: int, method: str = "batched",
                start: str = "reference"):
        th = theta.detach().cpu().double().numpy()
        lnz, en, N, lnZ = sector_table(lat, th, R, M, seed, method, start)
        ctx.save_for_backward(theta)
        ctx.cfg = (lat, R, M, seed, method, start)
        ctx.table = (lnz, en)
        return theta.new_tensor(lnZ)

    @staticmethod
    def backward(ctx, grad_out):
        (theta,) = ctx.saved_tensors
        lat, R, M, seed, method, start = ctx.cfg
        lnz, en = ctx.table
        g = sector_table_grad(lat, theta.detach().cpu().double().numpy(), R, M, seed, lnz, en, method, start)
        return grad_out * theta.new_tensor(g), None, None, None, None, None, None


def grand_canonical_logz(theta: torch.Tensor, lat: Lattice, R: int, M: int, seed: int, method: str = "batched",
                         start: str = "reference") -> torch.Tensor:
    return GrandCanonicalLogZ.apply(theta, lat, R, M, seed, method, start)
