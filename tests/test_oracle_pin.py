"""Pins the oracle (oracle/ftlm_oracle.cpp) to the reference: against the reference library built
from its own sources (oracle/_ref) where present, and against the committed golden vectors."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

CASES = [
    (2, 2, 1.0, 0.0, 0.0, 0.0, 0.31, -0.27, 2, 2),
    (3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0, 2, 3),
    (4, 2, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0, 4, 4),
    (3, 3, 1.0, -0.35, 5.75, 0.9, 0.2, 0.1, 4, 5),
    (5, 1, 1.0, 0.3, 2.0, 0.5, 0.4, 0.0, 2, 3),
    (1, 4, 1.0, 0.0, 3.0, 0.0, 0.0, 0.7, 2, 1),
    (2, 1, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1, 1),
]

needs_ref = pytest.mark.skipif(not O.have_reference(), reason="reference sources/library not present")


@needs_ref
@pytest.mark.parametrize("c", CASES)
def test_masks_apply_lanczos_bit_exact_vs_reference(c):
    R = O.reference()
    h = R.ref_sector_create(*c)
    try:
        s = O.OracleSector(*c)
        dim = R.ref_sector_dim(h)
        assert dim == s.dim
        up = np.zeros(dim, np.uint64)
        dn = np.zeros(dim, np.uint64)
        R.ref_sector_masks(h, O.P(up), O.P(dn))
        u2, d2 = s.masks()
        assert (up == u2).all() and (dn == d2).all()
        rng = np.random.default_rng(3)
        x = rng.standard_normal(dim) + 1j * rng.standard_normal(dim)
        x[rng.random(dim) < 0.1] = 0.0
        x[rng.random(dim) < 0.05] = 1e-15  # below the reference's 1e-28 |x|^2 skip threshold
        y = np.zeros(dim, np.complex128)
        R.ref_sector_apply(h, O.P(x), O.P(y))
        assert np.array_equal(s.apply(x, mode=0), y)  # same scatter order: bit-exact
        yg = s.apply(x, mode=1, nthreads=4)
        assert np.abs(yg - y).max() <= 1e-14 * max(1.0, np.abs(y).max())
        M = 30
        a = np.zeros(M)
        b = np.zeros(M)
        nb = C.c_int()
        used = R.ref_sector_lanczos(h, M, 99, O.P(a), O.P(b), C.byref(nb))
        a2, b2, u2_ = s.lanczos(M, 99, mode=0)
        assert used == u2_ and np.array_equal(a[:used], a2) and np.array_equal(b[:nb.value], b2)
        mn, mx = C.c_double(), C.c_double()
        ue = R.ref_sector_lanczos_extrema(h, 25, 5, C.byref(mn), C.byref(mx))
        e2 = s.lanczos_extrema(25, 5, mode=0)
        assert (mn.value, mx.value, ue) == e2
        lz = R.ref_sector_ftlm_complex(h, 1.7, 5, 25, 3)
        lz2, _ = s.ftlm(1.7, 5, 25, 3, mode=0)
        assert lz == lz2[0]
    finally:
        R.ref_sector_destroy(h)


@needs_ref
@pytest.mark.parametrize("lat", [(4, 4, 0.1, 0.0), (4, 2, 0.0, 0.0), (3, 3, 0.2, -0.3), (2, 2, 0.31, -0.27),
                                 (1, 4, 0.0, 0.7), (5, 1, 0.4, 0.0), (1, 1, 0.0, 0.0)])
def test_geometry_bit_exact_vs_reference(lat):
    Lx, Ly, px, py = lat
    R = O.reference()
    L = O.oracle()
    out = []
    for lib, fn in ((R, "ref"), (L, "or")):
        f = np.zeros(1024, np.int32)
        t = np.zeros(1024, np.int32)
        s = np.zeros(1024, np.int32)
        cf = np.zeros(2048)
        pi = np.zeros(256, np.int32)
        pj = np.zeros(256, np.int32)
        npair = C.c_int()
        if fn == "ref":
            nh = R.ref_geometry(Lx, Ly, 1.0, -0.25, 8.0, 1.0, px, py, 1024, O.P(f), O.P(t), O.P(s), O.P(cf), 256,
                                O.P(pi), O.P(pj), C.byref(npair))
        else:
            nh = L.or_geometry(Lx, Ly, 1.0, -0.25, px, py, 1024, O.P(f), O.P(t), O.P(s), O.P(cf), 256, O.P(pi),
                               O.P(pj), C.byref(npair))
        out.append((nh, f[:nh], t[:nh], s[:nh], cf[:2 * nh], pi[:npair.value], pj[:npair.value]))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_oracle_vs_golden_ref_small(golden):
    g = golden("ref_small.npz")
    for k, c in enumerate(g["cases"]):
        c = tuple(int(v) if i in (0, 1, 8, 9) else float(v) for i, v in enumerate(c))
        s = O.OracleSector(*c)
        up, dn = s.masks()
        assert np.array_equal(up, g[f"up{k}"]) and np.array_equal(dn, g[f"dn{k}"])
        assert np.array_equal(s.apply(g[f"x{k}"], mode=0), g[f"y{k}"])
        a, b, used = s.lanczos(40, 11 + k, mode=0)
        assert np.array_equal(a, g[f"alpha{k}"]) and np.array_equal(b, g[f"beta{k}"])
        mn, mx, ue = s.lanczos_extrema(30, 5, mode=0)
        assert np.array_equal(np.array([mn, mx, ue]), g[f"extrema{k}"])
        lz, _ = s.ftlm(2.0, 6, 30, 3, mode=0)
        assert lz[0] == g[f"lnz{k}"][0]


def test_known_answer_diag23(golden):
    """tests/test_ftlm_thermo.cpp: diag(2,3), beta=1, R=48, M=32, seed 12345, |err| < 0.15."""
    g = golden("ref_small.npz")
    exact = np.log(np.exp(-2.0) + np.exp(-3.0))
    est = g["diag23_lnz"][0]
    assert abs(est - exact) < 0.15
    # the oracle's quadrature on the same chains: Lanczos of a diagonal 2x2 stops after 2 steps
    q = O.start_vector(2, 12345)
    assert abs(np.linalg.norm(q) - 1.0) < 1e-15


def _fmt(v):
    return f"{v:g}"


def _oracle_nmu(Lx, Ly, tp, U, V, R, M, seed, beta, mus, mode=1, nthreads=8):
    lz, es, N, dims, _ = O.oracle_sweep(Lx, Ly, 1.0, tp, U, V, 0.0, 0.0, R, M, seed, np.array([beta]), mus, mode=mode,
                                        nthreads=nthreads)
    n = Lx * Ly
    _, nav, _ = O.gc_reduce(lz, es, N, np.array([beta]), mus, n)
    return lz[:, 0], nav[0]


@pytest.mark.parametrize("key,Lx,Ly", [("2x2", 2, 2), ("3x2_nonmom", 3, 2)])
def test_oracle_reproduces_published_tsv(golden, key, Lx, Ly):
    """The reference's published n(mu) tables (beta=20, t'=-0.35, U=5.75, V=0.9, R=12, M=72, seed 7)."""
    g = golden("published_tsv.npz")
    mu = g[f"{key}_mu"]
    n_pub = g[f"{key}_n"]
    # bench_ftlm_nmu_rect.cpp:186-188: mu_k = mu_min + k/(n_mu-1) * (mu_max - mu_min)
    lo, hi, nmu = float(mu[0]), float(mu[-1]), mu.size
    mus = np.array([lo + (k / (nmu - 1.0)) * (hi - lo) for k in range(nmu)])
    assert np.array_equal(np.array([float(_fmt(m)) for m in mus]), mu)
    lz, nav = _oracle_nmu(Lx, Ly, -0.35, 5.75, 0.9, 12, 72, 7, 20.0, mus)
    mism = [(m, a, b) for m, a, b in zip(mus, nav, n_pub) if _fmt(a) != _fmt(b)]
    # printed with 6 significant digits; allow last-digit ties from summation order in the gather oracle
    assert all(abs(a - b) <= 1e-5 * abs(b) + 1e-300 for _, a, b in mism), mism[:5]
    if key == "3x2_nonmom":
        for (nu, nd, dim), lzp in zip(g["3x2_sector"], g["3x2_sector_lnz"]):
            assert abs(lz[nu * 7 + nd] - lzp) <= 5e-6 * max(1.0, abs(lzp))


def test_sweep_4x2_golden_is_self_consistent(golden):
    g = golden("sweep_4x2.npz")
    lz = g["lnz_sector"]
    assert lz.shape == (81, 20)
    assert np.isfinite(lz).all()
    o1, o2, o3 = O.gc_reduce(lz, g["e_sector"], g["N"], 1.0 / g["T"], g["mu"], 8)
    assert np.array_equal(o1, g["lnz_gc"]) and np.array_equal(o2, g["n_gc"]) and np.array_equal(o3, g["e_gc"])
    # dims are the binomial products of the 4x2 sectors
    from math import comb
    assert [int(d) for d in g["dims"]] == [comb(8, a) * comb(8, b) for a in range(9) for b in range(9)]


# ---- translation-orbit momentum blocks ----------------------------------------------------------
ORBIT_CASES = [
    # Lx, Ly, t, tp, U, V, phix, phiy, nu, nd, K list
    ((2, 2, 1.0, 0.0, 4.0, 0.5, 0.0, 0.0, 2, 2), [(0, 0), (1, 0), (0, 1), (1, 1)]),
    ((2, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0, 1, 1), [(0, 0), (1, 1)]),
    ((3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0, 2, 3), [(1, 0), (2, 1)]),
    ((3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0, 3, 3), [(1, 0)]),
    ((4, 2, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0, 3, 3), [(0, 0), (2, 1), (3, 0)]),
    ((3, 3, 1.0, -0.25, 6.0, 0.5, 0.0, 0.0, 2, 2), [(0, 0), (1, 2)]),
    ((4, 3, 1.0, -0.25, 6.0, 0.5, 0.0, 0.0, 2, 1), [(1, 1), (3, 2)]),
]


def _orbit_ids():
    return [f"{c[0]}x{c[1]}_{c[8]}{c[9]}" for c, _ in ORBIT_CASES]


@needs_ref
@pytest.mark.parametrize("case", ORBIT_CASES, ids=_orbit_ids())
def test_orbit_block_bit_exact_vs_reference(case):
    c, ks = case
    R = O.reference()
    h = R.ref_sector_create(*c)
    s = O.OracleSector(*c)
    try:
        for kx, ky in ks:
            ro = R.ref_orbit_create(h, kx, ky)
            assert ro
            try:
                o = O.OracleOrbit(s, kx, ky)
                dk = R.ref_orbit_dim(ro)
                assert dk == o.dim
                rep = np.zeros(dk, np.uint32)
                absA = np.zeros(dk)
                size = np.zeros(dk, np.int32)
                R.ref_orbit_entries(ro, O.P(rep), O.P(absA), O.P(size))
                rep2, absA2, size2 = o.entries()
                assert np.array_equal(rep, rep2) and np.array_equal(size, size2)
                assert np.array_equal(absA, absA2)
                rng = np.random.default_rng(11 + kx + 7 * ky)
                x = rng.standard_normal(dk) + 1j * rng.standard_normal(dk)
                x[rng.random(dk) < 0.1] = 1e-15
                y = np.zeros(dk, np.complex128)
                R.ref_orbit_apply(ro, O.P(x), O.P(y))
                assert np.array_equal(o.apply(x), y)
                if dk >= 1:
                    lz = R.ref_orbit_ftlm_complex(ro, 0.9, 4, 20, 5)
                    lz2, _ = o.ftlm(0.9, 4, 20, 5)
                    assert lz == lz2[0]
            finally:
                R.ref_orbit_destroy(ro)
    finally:
        R.ref_sector_destroy(h)


def _dense(op, n):
    H = np.zeros((n, n), np.complex128)
    for j in range(n):
        e = np.zeros(n, np.complex128)
        e[j] = 1.0
        H[:, j] = op(e)
    return H


def test_orbit_known_answers():
    """tests/test_orbit_k_block_basis.cpp:19-101: dims 12 (2x2 (2,2) Gamma) and 66 (3x2 (3,3) K=(1,0));
    |A| = |Stab| on 2x2 Gamma; orbit sizes of the surviving reps sum to the mapped states."""
    s = O.OracleSector(2, 2, 1.0, 0.0, 4.0, 0.5, 0.0, 0.0, 2, 2)
    o = O.OracleOrbit(s, 0, 0)
    assert o.dim == 12
    _, absA, size = o.entries()
    assert np.allclose(absA, 4.0 / size, atol=1e-9)
    s32 = O.OracleSector(3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0, 3, 3)
    assert O.OracleOrbit(s32, 1, 0).dim == 66


@pytest.mark.parametrize("case", ORBIT_CASES[:6], ids=_orbit_ids()[:6])
def test_orbit_blocks_partition_spectrum(case):
    """The momentum blocks are Hermitian and their spectra together are the sector's spectrum."""
    c, _ = case
    s = O.OracleSector(*c)
    Lx, Ly = c[0], c[1]
    ev = []
    total = 0
    for ky in range(Ly):
        for kx in range(Lx):
            o = O.OracleOrbit(s, kx, ky)
            total += o.dim
            if o.dim == 0:
                continue
            Hk = _dense(o.apply, o.dim)
            assert np.abs(Hk - Hk.conj().T).max() < 1e-12
            ev.append(np.linalg.eigvalsh(Hk))
    assert total == s.dim
    Hf = _dense(lambda v: s.apply(v, mode=0), s.dim)
    np.testing.assert_allclose(np.sort(np.concatenate(ev)), np.linalg.eigvalsh(Hf), atol=1e-10)


def _korbit_oracle_lnz(nu, nd, beta, R, M, seed, ed_cutoff, lat=(3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0)):
    """k-resolved sector ln Z with the oracle: dense ED of blocks with dim <= ed_cutoff, FTLM above
    (benchmarks/bench_ftlm_nmu_4x4_k.cpp:1071-1081)."""
    s = O.OracleSector(*lat, nu, nd)
    n = lat[0] * lat[1]
    idx = nu * (n + 1) + nd
    parts, total = [], 0
    for ky in range(lat[1]):
        for kx in range(lat[0]):
            o = O.OracleOrbit(s, kx, ky)
            total += o.dim
            if o.dim == 0:
                continue
            if o.dim <= ed_cutoff:
                w = np.linalg.eigvalsh(_dense(o.apply, o.dim))
                parts.append(np.logaddexp.reduce(-beta * w))
            else:
                parts.append(o.ftlm(beta, R, M, seed + idx * 257 + ky * 17 + kx)[0][0])
    return (np.logaddexp.reduce(parts) if parts else -np.inf), total


def test_oracle_k_resolved_reproduces_published_korbit_run(golden):
    """The reference's published 3x2 k-orbit run (beta=20, R=12, M=72, seed 7, ed-cutoff 64): every
    sector where it used the orbit basis (0 < N_up, N_dn < 6) at printed precision, incl. the FTLM
    sector (3,3).  Sectors with an empty or full species ran its Gram path, which drops states
    (dim_k_total 12 of 15, 0 of 1): there the orbit blocks keep the full sector."""
    g = golden("published_korbit.npz")
    for i in range(g["nu"].size):
        nu, nd = int(g["nu"][i]), int(g["nd"][i])
        lz, total = _korbit_oracle_lnz(nu, nd, 20.0, 12, 72, 7, 64)
        if 0 < nu < 6 and 0 < nd < 6:
            assert total == g["dim_k_total"][i]
            assert abs(lz - g["lnz"][i]) <= 0.6 * 10.0 ** -int(g["decimals"][i]), (nu, nd, lz, g["lnz"][i])
        else:
            assert total == g["dim_full"][i]
