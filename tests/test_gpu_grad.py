"""Parameter gradient of FTLM ln Z on the GPU (ftlm_gpu_grad_sector and the autograd Function).

Bars: per-sector d ln Z/d(U, V, t') within 1e-6 of central differences (h = 1e-4) of the same
estimator; complex64 batched gradients within 1e-5 of the complex128 gradients with the same start
vectors; the autograd gradient of ln Z_GC within 1e-5 of central differences of the oracle (the
reference's CPU FTLM, restated) at shifted parameters."""
import numpy as np
import pytest
import torch

import ftlm_extended_hubbard_b200 as F
from ftlm_extended_hubbard_b200 import autograd as AG
import oracle as O

pytestmark = pytest.mark.gpu

H = 1e-4


def _lnz(lat, U, V, tp, nu, nd, beta, R, M, seed, start="reference"):
    s = F.Sector(F.HubbardParams(lat[0], lat[1], 1.0, tp, U, V, 0.0, 0.0), nu, nd)
    return s.ftlm(beta, R, M, seed, start=start)[0][0]


@pytest.mark.parametrize("lat,nu,nd,beta", [((3, 2), 2, 3, 1.5), ((4, 2), 3, 3, 3.0), ((4, 2), 4, 4, 0.7),
                                            ((2, 2), 1, 0, 2.0)])
def test_sector_gradient_matches_central_differences(gpu, lat, nu, nd, beta):
    U, V, tp, R, M, seed = 4.0, 1.0, -0.2, 6, 40, 11
    s = F.Sector(F.HubbardParams(lat[0], lat[1], 1.0, tp, U, V, 0.0, 0.0), nu, nd)
    op = F.Sector(F.HubbardParams(lat[0], lat[1], 0.0, 1.0, 0.0, 0.0, 0.0, 0.0), nu, nd)
    lz, g = s.ftlm_grad(beta, R, M, seed, op_tp=op)
    lz0 = _lnz(lat, U, V, tp, nu, nd, beta, R, M, seed)
    assert abs(lz - lz0) <= 1e-10 * max(1.0, abs(lz0))
    fd = [(_lnz(lat, U + H, V, tp, nu, nd, beta, R, M, seed) - _lnz(lat, U - H, V, tp, nu, nd, beta, R, M, seed)) / (2 * H),
          (_lnz(lat, U, V + H, tp, nu, nd, beta, R, M, seed) - _lnz(lat, U, V - H, tp, nu, nd, beta, R, M, seed)) / (2 * H),
          (_lnz(lat, U, V, tp + H, nu, nd, beta, R, M, seed) - _lnz(lat, U, V, tp - H, nu, nd, beta, R, M, seed)) / (2 * H)]
    scale = max(1.0, np.abs(fd).max())
    assert np.all(np.abs(g - np.array(fd)) <= 1e-6 * scale), (g, fd)


def test_batched_gradient_follows_complex128(gpu):
    lat, nu, nd, beta, R, M, seed = (4, 3), 3, 3, 2.0, 32, 50, 5
    p = F.HubbardParams(lat[0], lat[1], 1.0, -0.2, 4.0, 1.0, 0.0, 0.0)
    s = F.Sector(p, nu, nd)
    op = F.Sector(F.HubbardParams(lat[0], lat[1], 0.0, 1.0, 0.0, 0.0, 0.0, 0.0), nu, nd)
    lz_b, g_b = s.ftlm_grad(beta, R, M, seed, op_tp=op, method="batched")
    lz_p, g_p = s.ftlm_grad(beta, R, M, seed, op_tp=op, method="plain", start="philox")
    lz_f, _ = s.batched_ftlm(beta, R, M, seed)
    assert abs(lz_b - lz_f[0]) <= 1e-10 * abs(lz_f[0])  # replay reproduces the forward
    assert abs(lz_b - lz_p) <= 1e-6 * abs(lz_p)
    assert np.all(np.abs(g_b - g_p) <= 1e-5 * np.abs(g_p).max()), (g_b, g_p)


def test_autograd_matches_reference_ftlm_at_shifted_parameters(gpu):
    """ln Z_GC of a 3x2 lattice (all 49 sectors, R=8, M=40, reference start vectors): autograd
    against central differences of the oracle's grand-canonical ln Z (the reference algorithm)."""
    lat = AG.Lattice(3, 2)
    R, M, seed = 8, 40, 7
    theta0 = np.array([4.0, 1.0, -0.2, 2.0, 2.5])
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    lnZ = AG.grand_canonical_logz(theta, lat, R, M, seed, method="plain", start="reference")
    (grad,) = torch.autograd.grad(lnZ, theta)

    def oracle_lnz(th):
        U, V, tp, mu, beta = th
        _, _, _, _, (g_lnz, _, _) = O.oracle_sweep(lat.Lx, lat.Ly, 1.0, tp, U, V, 0.0, 0.0, R, M, seed,
                                                   np.array([beta]), np.array([mu]), mode=0)
        return float(np.asarray(g_lnz).ravel()[0])

    assert abs(lnZ.item() - oracle_lnz(theta0)) <= 1e-10 * abs(lnZ.item())
    fd = []
    for k in range(5):
        e = np.zeros(5)
        e[k] = H
        fd.append((oracle_lnz(theta0 + e) - oracle_lnz(theta0 - e)) / (2 * H))
    fd = np.array(fd)
    assert np.all(np.abs(grad.numpy() - fd) <= 1e-5 * np.maximum(1.0, np.abs(fd))), (grad.numpy(), fd)


def test_autograd_batched_matches_its_own_differences(gpu):
    """Batched complex64 forward on 4x2 (dims up to 4900 > 2M use complex64 blocks): autograd
    against central differences of the same forward; complex64 rounding bounds the agreement."""
    lat = AG.Lattice(4, 2)
    R, M, seed = 32, 40, 3
    theta0 = np.array([4.0, 1.0, -0.2, 2.0, 2.0])
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    lnZ = AG.grand_canonical_logz(theta, lat, R, M, seed, method="batched")
    lnZ.backward()
    h = 1e-3
    for k in range(5):
        e = np.zeros(5)
        e[k] = h
        fd = (AG.grand_canonical_logz_value(lat, theta0 + e, R, M, seed) -
              AG.grand_canonical_logz_value(lat, theta0 - e, R, M, seed)) / (2 * h)
        assert abs(theta.grad[k].item() - fd) <= 2e-4 * max(1.0, abs(fd)), (k, theta.grad[k].item(), fd)
