"""The single-sector workload at full size: 4x4 periodic square, sector (8,8), dim 165,636,900,
complex128, t=1 t'=-0.25 U=8 V=1 phi_x=0.1 phi_y=0, the reference's start vector (mt19937 + normal
distribution, seed 7), M = 150 Lanczos steps (src/lanczos.cpp:125-208).

The oracle's chain for the same inputs (row-gather H·v with the reference recurrence, threaded on
the host; hours of CPU time) is committed as tests/golden/ritz_4x4_8_8.npz by
tests/golden/make_golden.py.  Bars: the lowest 5 Ritz values of the 150-step tridiagonal within 1e-10
relative, on every fused kernel pair; alpha of the first 8 steps within 1e-11 relative (each alpha is a
sum of 1.66e8 terms, which the oracle and the GPU add in different orders: alpha_0 already differs by
~2.5e-13, about the size of that sum's rounding, and the recurrence roughly doubles such differences
per step)."""
import numpy as np
import pytest

import ftlm_extended_hubbard_b200 as F

pytestmark = pytest.mark.gpu


def test_config1_lowest_ritz_values_match_oracle_chain(gpu, golden):
    g = golden("ritz_4x4_8_8.npz")
    Lx, Ly, t, tp, U, V, px, py, nu, nd = g["params"].tolist()
    M, seed = int(g["M"][0]), int(g["seed"][0])
    assert (int(nu), int(nd), M, seed) == (8, 8, 150, 7)
    s = F.Sector(F.HubbardParams(int(Lx), int(Ly), t, tp, U, V, px, py), int(nu), int(nd))
    assert s.dim() == 165_636_900
    ao, bo = g["alpha"], g["beta"]
    r_cpu = g["ritz5"]
    assert int(g["used"][0]) == M
    assert np.allclose(F.ritz_values(ao, bo[:M - 1], 5), r_cpu, rtol=1e-14, atol=0.0)
    for path in (2, 3):  # both fused row + column pass pairs
        s.set_apply_path(path)
        a, b, used = s.lanczos(M, seed)
        assert used == M
        r_gpu = F.ritz_values(a, b[:M - 1], 5)
        print(f"path {path}: lowest 5 Ritz values {r_gpu}, oracle {r_cpu}, "
              f"max rel {np.max(np.abs(r_gpu - r_cpu) / np.abs(r_cpu)):.2e}; alpha[:8] max rel "
              f"{np.max(np.abs(a[:8] - ao[:8]) / np.abs(ao[:8])):.2e}")
        assert np.all(np.abs(a[:8] - ao[:8]) <= 1e-11 * np.abs(ao[:8])), (path, a[:8], ao[:8])
        assert np.all(np.abs(r_gpu - r_cpu) <= 1e-10 * np.abs(r_cpu)), (path, r_gpu, r_cpu)
