"""Batched complex64 FTLM path (ftlm_gpu_batched_*) against the complex128 path with the same Philox
start vectors, both evaluated with the converged quadrature (the reference's rotation-capped Jacobi
is a discontinuous function of alpha/beta at low temperature, which would mask the comparison).  Bars: early alpha/beta within 2e-5 relative (complex64 vectors), extremal Ritz values
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
    with F.quadrature("converged"):  # the batched path's quadrature, so that only the chains differ
        lz_p, e_p = s.ftlm(bts, 32, 60, 7, start="philox")
    assert np.all(np.abs(lz_b - lz_p) <= 1e-6 * np.abs(lz_p))
    assert np.all(np.abs(e_b - e_p) <= 1e-6 * np.maximum(1.0, np.abs(e_p)))


def test_batched_sweep_4x3_matches_complex128(gpu):
    """All 169 sectors of the 4x3 lattice, R=32, M=60: batched vs plain (same Philox starts)."""
    t0 = time.perf_counter()
    rb = F.grand_canonical_sweep(P43, 32, 60, 7, T_GRID, MU_GRID, method="batched")
    tb = time.perf_counter() - t0
    t0 = time.perf_counter()
    with F.quadrature("converged"):
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


@pytest.mark.parametrize("nu,nd", [(8, 8), (7, 8)])
def test_batched_largest_4x4_sectors_within_1e6(gpu, nu, nd):
    """The largest sectors of the full 4x4 sweep (dims 165,636,900 and 147,232,800), R=32, M=100,
    the T grid of the sweep: batched complex64 sector ln Z against complex128 chains from the same
    Philox starts (same converged quadrature) within 1e-6 relative; the per-result error estimate (chain 0 rerun in complex128)
    is reported alongside and bounded by the same bar."""
    s = F.Sector(P44, nu, nd)
    bts = 1.0 / T_GRID
    lz_b, e_b, err = s.batched_ftlm(bts, 32, 100, 7, check=1)
    F.batched_release()
    with F.quadrature("converged"):
        lz_p, e_p = s.ftlm(bts, 32, 100, 7, start="philox")
    rel = np.abs(lz_b - lz_p) / np.maximum(1.0, np.abs(lz_p))
    print(f"({nu},{nd}): max rel err sector lnZ {rel.max():.2e}; estimate {np.max(err / np.maximum(1.0, np.abs(lz_p))):.2e}")
    assert rel.max() <= 1e-6
    assert np.all(np.isfinite(err)) and np.all(err / np.maximum(1.0, np.abs(lz_p)) <= 1e-6)


def test_batched_cols_variants_agree(gpu):
    """The column-pass variants (16/8/4-column chunks) sum the same terms in the same order per
    element; only the grouping of the FP64 dot partials differs, so the chains agree to rounding."""
    s = F.Sector(P44, 4, 4)
    out = []
    for v in (0, 1, 2):
        s.batched_set_cols_variant(v)
        A, B, used = s.batched_lanczos(32, 8, 11)
        assert (used == 8).all()
        out.append((A, B))
    for A, B in out[1:]:
        assert np.abs(A - out[0][0]).max() <= 1e-6 * np.abs(out[0][0]).max()
        assert np.abs(B - out[0][1]).max() <= 1e-6 * np.abs(out[0][1]).max()
    v, ms = s.batched_autotune(1)
    assert v in (0, 1, 2) and ms > 0
    assert F.Sector(P44, 4, 4).batched_autotune(1) == (v, -1.0)  # cached per sector shape
    F.batched_release()
