"""The reference's published n(mu) tables at beta=20 (t'=-0.35, U=5.75, V=0.9, R=12, M=72, seed 7;
benchmarks/data/n_vs_mu_*_beta20_*.tsv) reproduced by the GPU sweep with the reference's start
vectors, at the printed precision (6 significant digits; ties in the last digit allowed)."""
import numpy as np
import pytest

import ftlm_extended_hubbard_b200 as F

pytestmark = pytest.mark.gpu

CASES = [("2x2", 2, 2), ("4x2", 4, 2), ("3x2_nonmom", 3, 2), ("3x3", 3, 3), ("2x5", 2, 5)]


def mu_grid(mu):
    """benchmarks/bench_ftlm_nmu_rect.cpp:186-188: mu_k = mu_min + k/(n_mu-1) * (mu_max - mu_min)."""
    lo, hi, n = float(mu[0]), float(mu[-1]), mu.size
    return np.array([lo + (k / (n - 1.0)) * (hi - lo) for k in range(n)])


@pytest.mark.parametrize("key,Lx,Ly", CASES, ids=[c[0] for c in CASES])
def test_gpu_sweep_reproduces_published_table(gpu, golden, key, Lx, Ly):
    g = golden("published_tsv.npz")
    mus = mu_grid(g[f"{key}_mu"])
    assert np.array_equal(np.array([float(f"{m:g}") for m in mus]), g[f"{key}_mu"])
    p = F.HubbardParams(Lx, Ly, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0)
    r = F.grand_canonical_sweep(p, 12, 72, 7, [1.0 / 20.0], mus, start="reference")
    n_pub = g[f"{key}_n"]
    n = r.n_avg[0]
    bad = [(m, a, b) for m, a, b in zip(mus, n, n_pub) if f"{a:g}" != f"{b:g}" and abs(a - b) > 1e-5 * abs(b)]
    assert not bad, bad[:5]
