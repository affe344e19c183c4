"""Translation-orbit momentum blocks on the GPU (ftlm_gpu_orbit_*) against the reference's
OrbitKBlockBasis / apply_orbit_k_block (golden vectors from the reference library) and the oracle.

Bars: representatives and orbit dimensions exact; |A(K)| within 4 ulp (device hypot); H_K x within
1e-13 of max|y| (gather order on the GPU, scatter order in the reference); block and k-resolved
sector ln Z within 1e-10 relative with the reference's start vectors."""
import numpy as np
import pytest

import ftlm_extended_hubbard_b200 as F
import oracle as O

pytestmark = pytest.mark.gpu

RTOL_APPLY = 1e-13
RTOL_LNZ = 1e-10


def _case(c):
    c = [float(v) for v in c]
    return (F.HubbardParams(int(c[0]), int(c[1]), c[2], c[3], c[4], c[5], c[6], c[7]), int(c[8]), int(c[9]),
            int(c[10]), int(c[11]))


def test_orbit_blocks_match_reference_golden(gpu, golden):
    g = golden("orbit_small.npz")
    for k, c in enumerate(g["cases"]):
        p, nu, nd, kx, ky = _case(c)
        s = F.Sector(p, nu, nd)
        o = s.orbit_block(kx, ky)
        rep, absA = o.entries()
        assert o.dim == g[f"rep{k}"].size
        assert np.array_equal(rep, g[f"rep{k}"])
        np.testing.assert_allclose(absA, g[f"absA{k}"], rtol=4 * 2.2e-16, atol=0)
        y = o.apply_host(g[f"x{k}"])
        yr = g[f"y{k}"]
        assert np.abs(y - yr).max() <= RTOL_APPLY * np.abs(yr).max(), k
        lz, _ = o.ftlm(1.3, 5, 30, 17 + k)
        assert abs(lz[0] - g[f"lnz{k}"][0]) <= RTOL_LNZ * abs(g[f"lnz{k}"][0]), k


ORACLE_CASES = [
    # lattice params, nu, nd, momenta
    ((4, 4, 1.0, -0.25, 6.0, 0.5, 0.0, 0.0), 3, 2, [(0, 0), (1, 2), (2, 2), (3, 1)]),
    ((4, 4, 1.0, -0.25, 6.0, 0.5, 0.0, 0.0), 4, 4, [(2, 0)]),
    ((4, 3, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0), 3, 3, [(0, 0), (1, 1), (3, 2)]),
    ((3, 3, 1.0, 0.3, 2.0, 0.7, 0.0, 0.0), 4, 2, [(0, 0), (2, 1)]),
]


@pytest.mark.parametrize("case", ORACLE_CASES, ids=lambda c: f"{c[0][0]}x{c[0][1]}_{c[1]}{c[2]}")
def test_orbit_apply_matches_oracle(gpu, case):
    lat, nu, nd, ks = case
    s = F.Sector(F.HubbardParams(*lat), nu, nd)
    so = O.OracleSector(*lat, nu, nd)
    rng = np.random.default_rng(nu * 31 + nd)
    for kx, ky in ks:
        o = s.orbit_block(kx, ky)
        oo = O.OracleOrbit(so, kx, ky)
        assert o.dim == oo.dim
        rep, absA = o.entries()
        rep2, absA2, _ = oo.entries()
        assert np.array_equal(rep, rep2)
        np.testing.assert_allclose(absA, absA2, rtol=4 * 2.2e-16, atol=0)
        x = rng.standard_normal(o.dim) + 1j * rng.standard_normal(o.dim)
        x[rng.random(o.dim) < 0.05] = 0.0
        x[rng.random(o.dim) < 0.05] = 3e-15  # below the 1e-28 |x|^2 skip threshold
        yr = oo.apply(x)
        for path in (0, 1):
            o.set_apply_path(path)
            y = o.apply_host(x)
            assert np.abs(y - yr).max() <= RTOL_APPLY * np.abs(yr).max(), path


def test_orbit_apply_device_pointers(gpu):
    torch = gpu
    s = F.Sector(F.HubbardParams(4, 3, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0), 3, 3)
    o = s.orbit_block(1, 1)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(o.dim) + 1j * rng.standard_normal(o.dim)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    o.apply(xd, yd)
    torch.cuda.synchronize()
    assert np.array_equal(yd.cpu().numpy(), o.apply_host(x))


def test_orbit_blocks_partition_the_sector(gpu):
    """The block dimensions over all momenta add up to the sector dimension; H_K is Hermitian."""
    s = F.Sector(F.HubbardParams(4, 2, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0), 3, 3)
    total = 0
    for ky in range(2):
        for kx in range(4):
            o = s.orbit_block(kx, ky)
            total += o.dim
            H = np.zeros((o.dim, o.dim), np.complex128)
            for j in range(o.dim):
                e = np.zeros(o.dim, np.complex128)
                e[j] = 1.0
                H[:, j] = o.apply_host(e)
            assert np.abs(H - H.conj().T).max() <= 1e-13 * np.abs(H).max()
    assert total == s.dim()


def test_k_resolved_sector_lnz_matches_oracle(gpu):
    """ftlm_gpu_orbit_sector_ftlm: seed_K = seed + sector_index*257 + ky*17 + kx, LSE over the blocks."""
    lat = (3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0)
    nu, nd, idx, seed, R, M = 2, 3, 17, 7, 6, 30
    bts = np.array([0.5, 2.0, 20.0])
    s = F.Sector(F.HubbardParams(*lat), nu, nd)
    lz, en, dims = s.orbit_ftlm(bts, R, M, seed, sector_index=idx, ed_cutoff=0)
    so = O.OracleSector(*lat, nu, nd)
    parts = []
    for ky in range(lat[1]):
        for kx in range(lat[0]):
            oo = O.OracleOrbit(so, kx, ky)
            assert dims[ky, kx] == oo.dim
            if oo.dim:
                parts.append(oo.ftlm(bts, R, M, seed + idx * 257 + ky * 17 + kx)[0])
    ref = np.logaddexp.reduce(np.array(parts), axis=0)
    assert np.all(np.abs(lz - ref) <= RTOL_LNZ * np.abs(ref))
    assert dims.sum() == s.dim()


def test_k_resolved_lnz_estimates_the_sector(gpu):
    """Different estimator, same quantity: the k-resolved ln Z of a 4x4 sector agrees with the
    unsymmetrised FTLM ln Z within the stochastic error at high temperature."""
    p = F.HubbardParams(4, 4, 1.0, -0.25, 6.0, 0.5, 0.0, 0.0)
    s = F.Sector(p, 3, 3)
    bts = np.array([0.2, 0.5])
    lz_k, _, dims = s.orbit_ftlm(bts, 8, 60, 7, start="philox")
    lz_f, _ = s.ftlm(bts, 8, 60, 7, start="philox")
    assert dims.sum() == s.dim()
    assert np.all(np.abs(lz_k - lz_f) <= 2e-3 * np.abs(lz_f))


def test_orbit_rejects_bad_arguments(gpu):
    s = F.Sector(F.HubbardParams(3, 2, 1.0, 0.0, 4.0, 0.0, 0.0, 0.0), 2, 2)
    with pytest.raises(ValueError):
        s.orbit_block(3, 0)
    hs, ps = F.build_hubbard_geometry(F.HubbardParams(3, 2, 1.0, 0.0, 4.0, 0.0, 0.0, 0.0))
    s2 = F.Sector(None, 2, 2, hops=hs, pairs=ps, n_sites=6, U=4.0, V=0.0)
    with pytest.raises(F.FtlmError):
        s2.orbit_block(0, 0)


def test_k_resolved_sweep_reproduces_published_korbit_run(gpu, golden):
    """All 49 sectors of the reference's published 3x2 k-orbit run (beta=20, R=12, M=72, seed 7,
    reference start vectors, ed-cutoff 64) at printed precision where it used the orbit basis."""
    g = golden("published_korbit.npz")
    p = F.HubbardParams(3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0)
    for i in range(g["nu"].size):
        nu, nd = int(g["nu"][i]), int(g["nd"][i])
        s = F.Sector(p, nu, nd)
        lz, _, dims = s.orbit_ftlm([20.0], 12, 72, 7, sector_index=nu * 7 + nd, ed_cutoff=64)
        if 0 < nu < 6 and 0 < nd < 6:
            assert dims.sum() == g["dim_k_total"][i]
            assert abs(lz[0] - g["lnz"][i]) <= 0.6 * 10.0 ** -int(g["decimals"][i]), (nu, nd, lz[0], g["lnz"][i])
        else:
            assert dims.sum() == g["dim_full"][i]


@pytest.mark.parametrize("nu,nd,k", [(4, 4, (1, 2)), (3, 3, (0, 0)), (5, 3, (2, 3))])
def test_batched_orbit_ftlm_follows_complex128(gpu, nu, nd, k):
    """complex64 32-chain blocks of one momentum block against the complex128 chains with the same
    Philox start vectors: block ln Z within 1e-6 relative."""
    s = F.Sector(F.HubbardParams(4, 4, 1.0, -0.25, 6.0, 0.5, 0.0, 0.0), nu, nd)
    o = s.orbit_block(*k)
    bts = 1.0 / np.array([0.1, 0.5, 1.0, 2.0])
    lz_b, e_b = o.batched_ftlm(bts, 32, 60, 11)
    with F.quadrature("converged"):  # the batched path's quadrature
        lz_p, e_p = o.ftlm(bts, 32, 60, 11, start="philox")
    assert np.all(np.abs(lz_b - lz_p) <= 1e-6 * np.abs(lz_p)), (lz_b, lz_p)
    assert np.all(np.abs(e_b - e_p) <= 1e-6 * np.maximum(1.0, np.abs(e_p)))


def test_batched_k_resolved_sector_follows_complex128(gpu):
    s = F.Sector(F.HubbardParams(4, 3, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0), 4, 3)
    bts = 1.0 / np.array([0.2, 1.0])
    lz_b, _, d1 = s.orbit_ftlm(bts, 24, 60, 7, sector_index=68, method="batched")
    with F.quadrature("converged"):
        lz_p, _, d2 = s.orbit_ftlm(bts, 24, 60, 7, sector_index=68, start="philox")
    assert np.array_equal(d1, d2)
    assert np.all(np.abs(lz_b - lz_p) <= 1e-6 * np.abs(lz_p)), (lz_b, lz_p)
