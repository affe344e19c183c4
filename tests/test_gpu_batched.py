"""Batched complex64 FTLM path (ftlm_gpu_batched_*) against the complex128 path with the same Philox
start vectors.  Bars: early alpha/beta within 2e-5 relative (complex64 vectors), extremal Ritz values
within 1e-5, sector and grand-canonical ln Z within 1e-6 relative, <n> within 1e-6 absolute."""
import time

import numpy as np
import pytest

import ftlm_extended_hubbard_b200 as F

pytestmark = pytest.mark.gpu

P44 = F.HubbardParams(4, 4, 1.0, -0.25, 8.0, 1.0, 0.1, 0.0)
P43 = F.HubbardParams(4, 3, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0)
T_GRID = np.round(np.arange(1, 21) * 0.1, 10)
MU_GRID = np.round(np.arange(49) * 0.25 - 4.0, 10)


def test_batched_chains_follow_complex128_chains(gpu):
    s = F.Sector(P44, 4, 4)
    R, M = 32, 40
    A, B, used = s.batched_lanczos(R, M, 11)
    assert (used == M).all()
    for r in (0, 5, 31):
        a, b, u = s.lanczos(M, 11 + r * 100003, start="philox")
        assert u == M
        assert np.all(np.abs(A[r, :6] - a[:6]) <= 2e-5 * np.abs(a[:6]).max())
        assert np.all(np.abs(B[r, :6] - b[:6]) <= 2e-5 * np.abs(b[:6]).max())
        r1 = F.ritz_values(A[r], B[r, :M - 1], 2)
        r2 = F.ritz_values(a, b[:M - 1], 2)
        assert np.abs(r1 - r2).max() <= 1e-5 * np.abs(r2).max()


def test_batched_is_deterministic(gpu):
    s = F.Sector(P43, 5, 6)
    A1, B1, _ = s.batched_lanczos(32, 25, 3)
    A2, B2, _ = s.batched_lanczos(32, 25, 3)
    assert np.array_equal(A1, A2) and np.array_equal(B1, B2)


@pytest.mark.parametrize("nu,nd", [(4, 4), (6, 5), (3, 2)])
def test_batched_sector_lnz_within_1e6(gpu, nu, nd):
    s = F.Sector(P44 if nu + nd < 11 else P43, nu, nd)
    bts = 1.0 / T_GRID
    lz_b, e_b = s.batched_ftlm(bts, 32, 60, 7)
    lz_p, e_p = s.ftlm(bts, 32, 60, 7, start="philox")
    assert np.all(np.abs(lz_b - lz_p) <= 1e-6 * np.abs(lz_p))
    assert np.all(np.abs(e_b - e_p) <= 1e-6 * np.maximum(1.0, np.abs(e_p)))


def test_batched_sweep_4x3_matches_complex128(gpu):
    """All 169 sectors of the 4x3 lattice, R=32, M=60: batched vs plain (same Philox starts)."""
    t0 = time.perf_counter()
    rb = F.grand_canonical_sweep(P43, 32, 60, 7, T_GRID, MU_GRID, method="batched")
    tb = time.perf_counter() - t0
    t0 = time.perf_counter()
    rp = F.grand_canonical_sweep(P43, 32, 60, 7, T_GRID, MU_GRID, start="philox")
    tp = time.perf_counter() - t0
    ok = np.isfinite(rp.lnz_sector)
    rel_s = np.abs(rb.lnz_sector[ok] - rp.lnz_sector[ok]) / np.maximum(1.0, np.abs(rp.lnz_sector[ok]))
    rel_g = np.abs(rb.lnz_gc - rp.lnz_gc) / np.maximum(1.0, np.abs(rp.lnz_gc))
    dn = np.abs(rb.n_avg - rp.n_avg)
    print(f"4x3 sweep R=32 M=60: batched {tb:.2f} s, plain {tp:.2f} s, speed-up {tp / tb:.2f}; "
          f"max rel err sector lnZ {rel_s.max():.2e}, GC lnZ {rel_g.max():.2e}, max |dn| {dn.max():.2e}")
    assert rel_s.max() <= 1e-6 and rel_g.max() <= 1e-6 and dn.max() <= 1e-6
    F.batched_release()
