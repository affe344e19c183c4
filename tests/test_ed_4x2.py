"""The 4x2 grand-canonical sweep (t=1 t'=-0.25 U=8 V=1, phi=0; 81 sectors, R=20, M=60, seed 7;
T = 0.1..2.0 x mu = -4..8) against full exact diagonalisation of all 65,536 levels, computed by the
reference's own NumPy ED mirror (benchmarks/hubbard_rect_ed.py; fixture tests/golden/ed_4x2.npz made
by tests/golden/make_golden.py ed_4x2).

FTLM is a stochastic estimator: with R = 20 random vectors per sector its error at these temperatures
is set by the sampling, not by rounding (at T = 0.1 the ground-state weight carries an O(1/sqrt(R))
error, about 0.2 in ln Z_GC).  The bars: the reference's own published FTLM-vs-ED accuracy for this
lattice, max |delta <n>| = 1.2e-2 (beta = 20, R = 16, M = 96; benchmarks/data/mem_ed_time.txt),
rounded up to |delta <n>| <= 1.5e-2; and the grand potential per site, -T ln Z_GC / 8, within 1e-2
(in units of t) on the whole grid (ln Z_GC itself crosses zero on the grid, so a relative bar on it is
ill-defined).  The CPU test checks the golden FTLM sweep (the reference algorithm, pinned to the
reference library); the GPU test checks the GPU sweep itself."""
import numpy as np
import pytest

import ftlm_extended_hubbard_b200 as F

TOL_N = 1.5e-2
TOL_OMEGA = 1e-2


def _check(lnz_gc, n_gc, ed):
    dn = np.abs(n_gc - ed["n_gc"]).max()
    domega = (np.abs(lnz_gc - ed["lnz_gc"]) * ed["T"][:, None]).max() / 8.0
    assert dn <= TOL_N, dn
    assert domega <= TOL_OMEGA, domega
    return dn, domega


def test_golden_ftlm_sweep_against_full_ed(golden):
    ed, g = golden("ed_4x2.npz"), golden("sweep_4x2.npz")
    assert np.array_equal(ed["T"], g["T"]) and np.array_equal(ed["mu"], g["mu"])
    _check(g["lnz_gc"], g["n_gc"], ed)
    # the dim-1 sectors are exact in FTLM (ln Z = -beta H_00)
    for idx in (0, 80):
        assert np.allclose(g["lnz_sector"][idx], ed["lnz_sector"][idx], rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_gpu_sweep_against_full_ed(gpu, golden):
    ed = golden("ed_4x2.npz")
    p = F.HubbardParams(4, 2, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0)
    r = F.grand_canonical_sweep(p, 20, 60, 7, ed["T"], ed["mu"])
    dn, dl = _check(r.lnz_gc, r.n_avg, ed)
    print(f"4x2 GPU FTLM sweep vs full ED: max |dn| {dn:.2e}, max |d Omega| per site {dl:.2e}")
