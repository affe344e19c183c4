"""Fused small-sector sweep (one CTA per chain, chains.cu) against the per-sector path: same start
vectors and recurrence, so sector ln Z agree to rounding (1e-12 relative); and the switch works."""
import numpy as np
import pytest

import ftlm_extended_hubbard_b200 as F
from ftlm_extended_hubbard_b200._lib import call

pytestmark = pytest.mark.gpu

T = np.array([0.05, 0.3, 1.0, 2.0])
MU = np.array([-2.0, 1.0, 3.0, 6.0])


@pytest.mark.parametrize("start", ["reference", "philox"])
def test_fused_sweep_matches_per_sector_path(gpu, start):
    p = F.HubbardParams(4, 2, 1.0, -0.25, 8.0, 1.0, 0.2, 0.0)
    try:
        call("ftlm_gpu_set_fused_max_dim", 0)
        r0 = F.grand_canonical_sweep(p, 6, 40, 7, T, MU, start=start)
        call("ftlm_gpu_set_fused_max_dim", 1 << 17)
        r1 = F.grand_canonical_sweep(p, 6, 40, 7, T, MU, start=start)
    finally:
        call("ftlm_gpu_set_fused_max_dim", 1 << 17)
    ok = np.isfinite(r0.lnz_sector)
    assert np.array_equal(ok, np.isfinite(r1.lnz_sector))
    rel = np.abs(r1.lnz_sector[ok] - r0.lnz_sector[ok]) / np.maximum(1.0, np.abs(r0.lnz_sector[ok]))
    assert rel.max() <= 1e-12, rel.max()
    assert np.abs(r1.n_avg - r0.n_avg).max() <= 1e-12


def test_fused_sweep_reproduces_4x2_golden(gpu, golden):
    g = golden("sweep_4x2.npz")
    Lx, Ly, t, tp, U, V, px, py, R, M, seed = g["params"]
    p = F.HubbardParams(int(Lx), int(Ly), t, tp, U, V, px, py)
    r = F.grand_canonical_sweep(p, int(R), int(M), int(seed), g["T"], g["mu"], start="reference")
    rel = np.abs(r.lnz_sector - g["lnz_sector"]) / np.maximum(1.0, np.abs(g["lnz_sector"]))
    assert rel.max() <= 1e-10
    assert np.abs(r.n_avg - g["n_gc"]).max() <= 1e-10
