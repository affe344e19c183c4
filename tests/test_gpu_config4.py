"""The differentiable workload at full size: ln Z_GC(U, V, t', mu, beta) of the 4x3 periodic lattice
(169 sectors, largest (6,6) with dim 853,776), R = 32 chains, M = 80 steps, at
theta = (U, V, t', mu, beta) = (4, 1, -0.2, 2, 5), batched complex64 chains with FP64 scalars.

Bars: the autograd gradient (hand-written backward, chains replayed from their seeds) within 1e-5
(relative to max(1, |g|)) of central differences with h = 1e-4 of the complex128 forward from the
same Philox start vectors; the batched forward within 1e-6 relative of that complex128 forward.
The complex128 forward's own parity with the reference's CPU FTLM (reference start vectors) is
pinned on smaller lattices (tests/test_gpu_grad.py, smoke); the 4x3 oracle sweep at R = 32, M = 80
is hours of CPU time."""
import time

import numpy as np
import pytest
import torch

from ftlm_extended_hubbard_b200 import autograd as AG

pytestmark = pytest.mark.gpu

H = 1e-4


def test_config4_gradient_matches_central_differences(gpu):
    lat = AG.Lattice(4, 3)
    R, M, seed = 32, 80, 7
    th0 = np.array([4.0, 1.0, -0.2, 2.0, 5.0])
    theta = torch.tensor(th0, dtype=torch.float64, requires_grad=True)
    t0 = time.perf_counter()
    lnZ = AG.grand_canonical_logz(theta, lat, R, M, seed, method="batched")
    t1 = time.perf_counter()
    lnZ.backward()
    t2 = time.perf_counter()
    g = theta.grad.numpy()

    def plain(th):
        return AG.grand_canonical_logz_value(lat, th, R, M, seed, method="plain", start="philox")

    t3 = time.perf_counter()
    lz128 = plain(th0)
    fd = np.array([(plain(th0 + H * e) - plain(th0 - H * e)) / (2 * H) for e in np.eye(5)])
    t4 = time.perf_counter()
    rel = np.abs(g - fd) / np.maximum(1.0, np.abs(fd))
    print(f"4x3 R=32 M=80: ln Z_GC {lnZ.item():.10f} (complex128 {lz128:.10f}); grad {g}; central differences {fd}; "
          f"rel {rel}; forward {t1 - t0:.1f} s, backward {t2 - t1:.1f} s, 11 complex128 forwards {t4 - t3:.1f} s")
    assert abs(lnZ.item() - lz128) <= 1e-6 * abs(lz128)
    assert np.all(rel <= 1e-5), rel
