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
(Sector.ftlm_grad: Duhamel derivative in each chain's Krylov space, start vectors fixed).
Sectors with w_s < 1e-13 are skipped (their term is below 1e-13 * beta * n_sites).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

import ctypes as C

from ._lib import call
from .api import HubbardParams, Sector, lanczos_sectors

WEIGHT_CUTOFF = 1e-13


@dataclass(frozen=True)
class Lattice:
    Lx: int
    Ly: int
    t: float = 1.0
    phi_x: float = 0.0
    phi_y: float = 0.0


FUSED_MAX_DIM = 1 << 17  # plain method: sectors up to this size run in one fused launch


def _quadrature(A, B, used, beta, dim):
    """ln Z_s and E_s from chains (converged tridiagonal quadrature, then the sector combine)."""
    R, M = A.shape
    A = np.ascontiguousarray(A)
    B = np.ascontiguousarray(B)
    used = np.ascontiguousarray(used, np.int32)
    bt = np.array([float(beta)])
    lq = np.zeros((R, 1))
    eq = np.zeros((R, 1))
    call("ftlm_gpu_tridiag_quadrature_exact", _p(A), _p(B), _p(used), R, M, _p(bt), 1, _p(lq), _p(eq))
    lnz = np.zeros(1)
    en = np.zeros(1)
    call("ftlm_gpu_ftlm_combine", _p(lq), _p(eq), _p(used), R, 1, float(np.log(dim)), _p(lnz), _p(en))
    return float(lnz[0]), float(en[0])


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def sector_table(lat: Lattice, theta, R, M, seed, method="batched", start="reference"):
    """ln Z_s, E_s, N_s for every sector at theta = (U, V, t', mu, beta).  Chains as the forward FTLM
    calls make them: method "batched" = complex64 32-chain blocks (sectors with dim <= 2M on the
    complex128 Philox path), "plain" = complex128 with `start`; the small sectors' chains all in one
    fused launch."""
    U, V, tp, mu, beta = (float(v) for v in theta)
    n = lat.Lx * lat.Ly
    p = HubbardParams(lat.Lx, lat.Ly, lat.t, tp, U, V, lat.phi_x, lat.phi_y)
    keys = [(nu, nd) for nu in range(n + 1) for nd in range(n + 1)]
    secs = {k: Sector(p, *k) for k in keys}
    limit = 2 * M if method == "batched" else FUSED_MAX_DIM
    small = [k for k in keys if secs[k].dim() <= limit]
    st = "philox" if method == "batched" else start
    A, B, used = lanczos_sectors([secs[k] for k in small], R, M, seed, start=st)
    out = {}
    for i, k in enumerate(small):
        out[k] = _quadrature(A[i * R:(i + 1) * R], B[i * R:(i + 1) * R], used[i * R:(i + 1) * R], beta,
                             secs[k].dim())
    for k in keys:
        if k in out:
            continue
        s = secs[k]
        if method == "batched":
            a, b, u = s.batched_lanczos(R, M, seed)
        else:
            a, b, u = _plain_chains(s, R, M, seed, st)
        out[k] = _quadrature(a, b, u, beta, s.dim())
    for s in secs.values():
        s.close()
    lnz = np.array([out[k][0] for k in keys])
    en = np.array([out[k][1] for k in keys])
    N = np.array([nu + nd for nu, nd in keys], dtype=np.float64)
    return lnz, en, N


def _plain_chains(s: Sector, R, M, seed, start):
    A = np.zeros((R, M))
    B = np.zeros((R, M))
    used = np.zeros(R, np.int32)
    for r in range(R):
        a, b, u = s.lanczos(M, (seed + r * 100003) & 0xFFFFFFFF, start=start)
        A[r, :a.size] = a
        B[r, :b.size] = b
        used[r] = u
    return A, B, used


def _sector_lnz(lat: Lattice, U, V, tp, beta, nu, nd, R, M, seed, method, start):
    """One sector's ln Z_s, E_s (same chains and quadrature as sector_table)."""
    s = Sector(HubbardParams(lat.Lx, lat.Ly, lat.t, tp, U, V, lat.phi_x, lat.phi_y), nu, nd)
    if method == "batched" and s.dim() > 2 * M:
        a, b, u = s.batched_lanczos(R, M, seed)
    elif s.dim() <= (2 * M if method == "batched" else FUSED_MAX_DIM):
        a, b, u = lanczos_sectors([s], R, M, seed, start="philox" if method == "batched" else start)
    else:
        a, b, u = _plain_chains(s, R, M, seed, "philox" if method == "batched" else start)
    return _quadrature(a, b, u, beta, s.dim())


def _lse(x):
    m = np.max(x)
    return float(m + np.log(np.sum(np.exp(x - m))))


def grand_canonical_logz_value(lat: Lattice, theta, R, M, seed, method="batched", start="reference") -> float:
    lnz, _, N = sector_table(lat, theta, R, M, seed, method, start)
    return _lse(lnz + float(theta[4]) * float(theta[3]) * N)


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
        lnz, en, N = sector_table(lat, th, R, M, seed, method, start)
        lnZ = gc_combine(lnz, en, N, th[3], th[4])[0]
        ctx.save_for_backward(theta)
        ctx.cfg = (lat, R, M, seed, method, start)
        ctx.table = (lnz, en, N, lnZ)
        return theta.new_tensor(lnZ)

    @staticmethod
    def backward(ctx, grad_out):
        (theta,) = ctx.saved_tensors
        lat, R, M, seed, method, start = ctx.cfg
        lnz, en, N, lnZ = ctx.table
        U, V, tp, mu, beta = (float(v) for v in theta.detach().cpu().double().numpy())
        _, w, dmu, dbeta = gc_combine(lnz, en, N, mu, beta)
        d = np.zeros(3)
        n = lat.Lx * lat.Ly
        k = 0
        for nu in range(n + 1):
            for nd in range(n + 1):
                ws = w[k]
                k += 1
                if not ws >= WEIGHT_CUTOFF:
                    continue
                p = HubbardParams(lat.Lx, lat.Ly, lat.t, tp, U, V, lat.phi_x, lat.phi_y)
                s = Sector(p, nu, nd)
                op = Sector(HubbardParams(lat.Lx, lat.Ly, 0.0, 1.0, 0.0, 0.0, lat.phi_x, lat.phi_y), nu, nd)
                lz, g = s.ftlm_grad(beta, R, M, seed, op_tp=op, method=method, start=start)
                if not abs(lz - lnz[k - 1]) <= 1e-9 * max(1.0, abs(lz)):
                    raise RuntimeError(f"gradient replay of sector ({nu},{nd}) did not reproduce the forward "
                                       f"ln Z ({lz} vs {lnz[k - 1]})")
                d += ws * g
        grad = theta.new_tensor([d[0], d[1], d[2], dmu, dbeta])
        return grad_out * grad, None, None, None, None, None, None


def grand_canonical_logz(theta: torch.Tensor, lat: Lattice, R: int, M: int, seed: int, method: str = "batched",
                         start: str = "reference") -> torch.Tensor:
    return GrandCanonicalLogZ.apply(theta, lat, R, M, seed, method, start)
