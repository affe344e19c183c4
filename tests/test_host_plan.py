"""Host-side logic of the native library (no GPU calls): exported C ABI, basis ranking, geometry,
diagonal tables, plan statistics, and the reference's argument errors."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

import oracle as O
import ftlm_extended_hubbard_b200 as F
from ftlm_extended_hubbard_b200 import _lib
from conftest import ROOT, has_gpu


def declared_symbols():
    with open(os.path.join(ROOT, "include", "ftlm_gpu.h")) as f:
        txt = f.read()
    return sorted(set(re.findall(r"\b(ftlm_gpu_\w+)\s*\(", txt)))


def test_library_loads_and_exports_every_declared_symbol():
    L = _lib.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) <= set(_lib.SIGNATURES), set(syms) - set(_lib.SIGNATURES)
    assert "sm_100a" in F.version_string()


@pytest.mark.parametrize("n,k", [(1, 0), (1, 1), (4, 2), (8, 4), (12, 6), (16, 8), (16, 3), (20, 10), (24, 2)])
def test_rank_closed_form_matches_enumeration(n, k):
    b = F.FockBasis(n, k, 0)
    assert b.dim() == math.comb(n, k)
    ref = np.zeros(math.comb(n, k), np.uint64)
    assert O.oracle().or_enumerate(n, k, O.P(ref)) == ref.size
    up, dn = b.masks()
    assert np.array_equal(up, ref)
    assert (dn == 0).all()
    idx = [b.index_of(int(m), 0) for m in ref[:: max(1, ref.size // 2000)]]
    assert idx == list(range(0, ref.size, max(1, ref.size // 2000)))


@pytest.mark.parametrize("c", [(4, 2, 4, 4), (3, 3, 4, 5), (4, 3, 2, 3), (2, 2, 0, 4), (1, 1, 1, 0)])
def test_fock_basis_matches_oracle(c):
    Lx, Ly, nu, nd = c
    b = F.FockBasis(Lx * Ly, nu, nd)
    s = O.OracleSector(Lx, Ly, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, nu, nd)
    up, dn = b.masks()
    u2, d2 = s.masks()
    assert np.array_equal(up, u2) and np.array_equal(dn, d2)
    for i in range(0, b.dim(), max(1, b.dim() // 97)):
        assert b.index_of(int(up[i]), int(dn[i])) == i == s.L.or_sector_index_of(s.h, int(up[i]), int(dn[i]))
        assert b.up_mask(i) == int(up[i]) and b.down_mask(i) == int(dn[i])
    # outside the sector -> -1 (FockBasis::index_of)
    assert b.index_of(int(up[0]) ^ 1, int(dn[0])) == -1 or nu == 0 or nu == Lx * Ly
    assert b.index_of(1 << 40, 0) == -1


@pytest.mark.parametrize("lat", [(4, 4, 0.1, 0.0), (4, 2, 0.0, 0.0), (3, 3, 0.2, -0.3), (2, 2, 0.31, -0.27),
                                 (1, 4, 0.0, 0.7), (1, 1, 0.0, 0.0)])
def test_geometry_matches_oracle_bit_exact(lat):
    Lx, Ly, px, py = lat
    hops, pairs = F.build_hubbard_geometry(F.HubbardParams(Lx, Ly, 1.0, -0.25, 8.0, 1.0, px, py))
    f = np.zeros(1024, np.int32)
    t = np.zeros(1024, np.int32)
    s = np.zeros(1024, np.int32)
    cf = np.zeros(2048)
    pi = np.zeros(256, np.int32)
    pj = np.zeros(256, np.int32)
    npair = C.c_int()
    nh = O.oracle().or_geometry(Lx, Ly, 1.0, -0.25, px, py, 1024, O.P(f), O.P(t), O.P(s), O.P(cf), 256, O.P(pi),
                                O.P(pj), C.byref(npair))
    assert nh == len(hops) and npair.value == len(pairs)
    for k, h in enumerate(hops):
        assert (h.from_, h.to, h.spin) == (f[k], t[k], s[k])
        assert h.coeff.real == cf[2 * k] and h.coeff.imag == cf[2 * k + 1]
    assert [(p.i, p.j) for p in pairs] == list(zip(pi[:npair.value], pj[:npair.value]))


def test_4x4_counts_from_survey():
    """4x4: 384 directed hops (192 per spin), 32 NN pairs; mean distinct up-hop sources 34.133 at N=8."""
    hops, pairs = F.build_hubbard_geometry(F.HubbardParams(4, 4, 1.0, -0.25, 8.0, 1.0, 0.1, 0.0))
    assert len(hops) == 384 and len(pairs) == 32
    h = C.c_void_p()
    ch = F.api._c_hops(hops)
    cp = F.api._c_pairs(pairs)
    _lib.call("ftlm_gpu_sector_create_host", 16, 8, 8, 8.0, 1.0, ch, len(hops), cp, len(pairs), C.byref(h))
    mu, md = C.c_double(), C.c_double()
    du, dd = C.c_longlong(), C.c_longlong()
    _lib.call("ftlm_gpu_sector_stats", h, C.byref(mu), C.byref(md), C.byref(du), C.byref(dd))
    assert du.value == dd.value == 12870
    assert abs(mu.value - 34.1333333333) < 1e-6 and abs(md.value - 34.1333333333) < 1e-6
    _lib.lib().ftlm_gpu_sector_destroy(h)


@pytest.mark.parametrize("c", [(4, 2, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0, 4, 4), (3, 3, 1.0, -0.35, 5.75, 0.9, 0.2, 0.1, 4, 5),
                               (2, 2, 1.0, 0.0, 3.0, 0.7, 0.0, 0.0, 2, 1)])
def test_diagonal_tables_match_oracle(c):
    Lx, Ly, t, tp, U, V, px, py, nu, nd = c
    hops, pairs = F.build_hubbard_geometry(F.HubbardParams(Lx, Ly, t, tp, U, V, px, py))
    h = C.c_void_p()
    _lib.call("ftlm_gpu_sector_create_host", Lx * Ly, nu, nd, U, V, F.api._c_hops(hops), len(hops),
              F.api._c_pairs(pairs), len(pairs), C.byref(h))
    s = O.OracleSector(*c)
    up, dn = s.masks()
    v = C.c_double()
    for i in range(0, s.dim, max(1, s.dim // 500)):
        _lib.call("ftlm_gpu_sector_diag", h, i, C.byref(v))
        ref = s.L.or_sector_diag(s.h, int(up[i]), int(dn[i]))
        assert abs(v.value - ref) <= 4e-16 * max(1.0, abs(ref))
    _lib.lib().ftlm_gpu_sector_destroy(h)


def test_argument_errors_follow_reference():
    with pytest.raises(ValueError):
        F.FockBasis(0, 0, 0)
    with pytest.raises(ValueError):
        F.FockBasis(33, 1, 1)
    with pytest.raises(ValueError):
        F.FockBasis(4, 5, 0)
    with pytest.raises(ValueError):
        F.FockBasis(4, -1, 0)
    with pytest.raises(F.FtlmError) as e:  # dim >= 2^31 is outside the reference's int index
        F.FockBasis(20, 10, 10)
    assert e.value.code == _lib.FTLM_ERR_UNSUPPORTED


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_device_calls_fail_cleanly_without_gpu():
    with pytest.raises(F.FtlmError) as e:
        F.Sector(F.HubbardParams(2, 2, 1.0), 1, 1)
    assert e.value.code in (_lib.FTLM_ERR_CUDA, _lib.FTLM_ERR_NOMEM)


@pytest.mark.parametrize("c", [(4, 4, 8, 8), (4, 4, 6, 5), (4, 3, 6, 6), (3, 3, 4, 5), (4, 4, 3, 1)])
def test_down_table_schedule_is_bank_conflict_free(c):
    """Every round of every quarter-warp reads 8 distinct bank groups (src % 8), and each lane keeps
    exactly its valid down hops: the sources of its entries are the down strings one hop away."""
    Lx, Ly, nu, nd = c
    hops, pairs = F.build_hubbard_geometry(F.HubbardParams(Lx, Ly, 1.0, -0.25, 8.0, 1.0, 0.1, 0.0))
    h = C.c_void_p()
    _lib.call("ftlm_gpu_sector_create_host", Lx * Ly, nu, nd, 8.0, 1.0, F.api._c_hops(hops), len(hops),
              F.api._c_pairs(pairs), len(pairs), C.byref(h))
    ng, ne, pad = C.c_longlong(), C.c_longlong(), C.c_int()
    _lib.call("ftlm_gpu_sector_down_table", h, C.byref(ng), C.byref(ne), None, None, C.byref(pad))
    gptr = np.zeros(ng.value + 1, np.int64)
    ent = np.zeros(ne.value, np.uint32)
    _lib.call("ftlm_gpu_sector_down_table", h, C.byref(ng), C.byref(ne), gptr.ctypes.data_as(C.c_void_p),
              ent.ctypes.data_as(C.c_void_p), C.byref(pad))
    b = F.FockBasis(Lx * Ly, nd, 0)
    dn, _ = b.masks()
    Dd = dn.size
    moves = {(x.from_, x.to) for x in hops if x.spin == 1}
    for g in range(ng.value):
        blk = ent[gptr[g]:gptr[g + 1]].reshape(-1, 32)
        src = blk >> 10
        hop = (blk >> 1) & 511
        for qw in range(4):
            for row in src[:, 8 * qw: 8 * qw + 8] % 8:
                assert len(set(row.tolist())) == 8
        for l in range(32):
            r = 32 * g + l
            if r >= Dd:
                continue
            d2 = int(dn[r])
            expect = sorted(b.index_of(d2 ^ (1 << f) ^ (1 << t), 0) for f, t in moves
                            if (d2 >> t) & 1 and not (d2 >> f) & 1)
            assert sorted(src[:, l][hop[:, l] != pad.value].tolist()) == expect
    _lib.lib().ftlm_gpu_sector_destroy(h)


def _gauge_table(h):
    ok, ng, ne, nt = C.c_int(), C.c_longlong(), C.c_longlong(), C.c_int()
    _lib.call("ftlm_gpu_sector_down_table_gauge", h, C.byref(ok), C.byref(ng), C.byref(ne), C.byref(nt), None, None,
              None, None)
    if not ok.value:
        return None
    grp = np.zeros(4 * ng.value, np.int32)
    ent = np.zeros(ne.value, np.uint32)
    tab, real2 = np.zeros(2 * max(nt.value, 1)), np.zeros(2)
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    _lib.call("ftlm_gpu_sector_down_table_gauge", h, C.byref(ok), C.byref(ng), C.byref(ne), C.byref(nt), P(grp),
              P(ent), P(tab), P(real2))
    return grp.reshape(-1, 4), ent, tab[0::2] + 1j * tab[1::2], real2


def _prefix_parity_shifted(d):
    q, par = 0, 0
    for k in range(32):  # bit k = parity of d's bits in [0, k)
        q |= par << k
        par ^= (d >> k) & 1
    return q


@pytest.mark.parametrize("c", [(4, 4, 1.0, -0.25, 8.0, 1.0, 0.1, 0.0, 3, 3), (4, 4, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0, 4, 5),
                               (4, 3, 1.0, -0.2, 4.0, 1.0, 0.0, 0.0, 3, 4), (3, 3, 1.0, -0.35, 5.75, 0.9, 0.2, 0.1, 4, 4)])
def test_gauge_down_table_reproduces_oracle_row(c):
    """The gauge-basis row-pass table, decoded on the CPU: with g(u,d) = (-1)^popc(u & pps(d)), the
    diagonal plus g * sum_h (-1)^s c_h g x over one row equals the oracle's H x for an x supported on
    that row (up hops leave the row), to 1e-14; every round of every quarter-warp, padding included,
    reads 8 distinct bank groups; padding reads the zero sentinels only."""
    Lx, Ly, t, tp, U, V, px, py, nu, nd = c
    hops, pairs = F.build_hubbard_geometry(F.HubbardParams(Lx, Ly, t, tp, U, V, px, py))
    h = C.c_void_p()
    _lib.call("ftlm_gpu_sector_create_host", Lx * Ly, nu, nd, U, V, F.api._c_hops(hops), len(hops),
              F.api._c_pairs(pairs), len(pairs), C.byref(h))
    tab = _gauge_table(h)
    assert tab is not None
    grp, ent, table, real2 = tab
    phase, pcps, xor = C.c_int(), np.zeros(2), C.c_int()
    perm = np.zeros(32 * len(grp), np.uint8)
    _lib.call("ftlm_gpu_sector_down_table_form", h, C.byref(phase), pcps.ctypes.data_as(C.c_void_p), C.byref(xor),
              perm.ctypes.data_as(C.c_void_p))
    perm = perm.reshape(-1, 32).astype(np.int64)
    # lane L of group g serves string 32 g + perm[g, L]: a permutation of the group, the identity on a
    # partial last group
    assert all(sorted(row.tolist()) == list(range(32)) for row in perm)
    # one Peierls phase (phi_y == 0, or phi_x == 0) gives the phase form; two phases need the table
    assert phase.value == (1 if (px == 0.0) != (py == 0.0) else 0)
    # the XOR form needs the two real values to share their low words (t' = -0.25: -1 and 2 * 0.25)
    assert xor.value == (1 if tp == -0.25 else 0)
    a0_bits = int(np.array([real2[0]]).view(np.uint64)[0])
    assert np.all(grp[:, 1] % 4 == 0) and np.all(grp[:, 2] % 4 == 0)
    o = O.OracleSector(*c)
    up, dn = o.masks()
    Dd = int(np.count_nonzero(up == up[0]))
    assert len(grp) == (Dd + 31) // 32
    if Dd % 32:
        assert np.array_equal(perm[-1], np.arange(32))
    pps = np.array([_prefix_parity_shifted(int(d)) for d in dn[:Dd]], dtype=np.int64)
    rng = np.random.default_rng(5)
    for r in (0, (o.dim // Dd) // 2, o.dim // Dd - 1):
        x = np.zeros(o.dim, np.complex128)
        x[r * Dd:(r + 1) * Dd] = rng.standard_normal(Dd) + 1j * rng.standard_normal(Dd)
        ref = o.apply(x, mode=0)[r * Dd:(r + 1) * Dd]
        u = int(up[r * Dd])
        g = np.array([1.0 - 2.0 * (bin(u & int(q)).count("1") & 1) for q in pps])
        xs = np.concatenate([g * x[r * Dd:(r + 1) * Dd], np.zeros(8)])
        y = np.zeros(Dd, np.complex128)
        v = C.c_double()
        for col in range(Dd):
            _lib.call("ftlm_gpu_sector_diag", h, r * Dd + col, C.byref(v))
            y[col] = v.value * x[r * Dd + col]
        for gi, (off, kr, kt, k0) in enumerate(grp):
            k4 = (kr + kt + 3) // 4 * 4
            blk = ent[off:off + 32 * k4].reshape(k4 // 4, 32, 4).transpose(0, 2, 1).reshape(k4, 32)
            src = (blk >> 4) & 0x3FFF
            kr0, kt0 = k0 & 0xFFFF, k0 >> 16  # rounds before the padding to whole loads: the rest is padding
            assert kr0 <= kr < kr0 + 4 and kt0 <= kt < kt0 + 4
            assert np.all(src[kr0:kr] >= Dd) and np.all(src[kr + kt0:kr + kt] >= Dd)
            for qw in range(4):
                for row in src[:, 8 * qw: 8 * qw + 8]:
                    assert len(set((row % 8).tolist())) == 8
            for l in range(32):
                col = 32 * gi + int(perm[gi, l])
                if col >= Dd:
                    assert np.all(src[:, l] >= Dd)
                    continue
                for k, e in enumerate(blk[:, l].tolist()):
                    sidx = (e >> 4) & 0x3FFF
                    if sidx >= Dd:
                        assert sidx < Dd + 8
                        continue
                    assert k < kr + kt
                    cf = real2[(e >> 30) & 1] if k < kr else table[(e >> 18) & 511]
                    sign = -1.0 if e >> 31 else 1.0
                    if k < kr and xor.value:  # (-1)^s real2[cls]: real2[0] with high-word bits ^ e
                        cf = float(np.array([a0_bits ^ ((e & 0xFFFC0000) << 32)], np.uint64).view(np.float64)[0])
                        assert cf in (real2[0], -real2[0], real2[1], -real2[1])
                        sign = 1.0
                    if k >= kr and phase.value:  # the row pass forms it as real2[cls] * (pc, +-ps)
                        a = real2[(e >> 30) & 1]
                        pf = complex(a * pcps[0], a * (-pcps[1] if (e >> 27) & 1 else pcps[1]))
                        assert pf == cf, (pf, cf)
                    y[col] += sign * g[col] * cf * xs[sidx]
        assert np.abs(y - ref).max() <= 1e-14 * np.abs(ref).max()
    _lib.lib().ftlm_gpu_sector_destroy(h)



@pytest.mark.parametrize("c", [(4, 4, 1.0, -0.25, 8.0, 1.0, 0.1, 0.0, 3, 3), (4, 3, 1.0, -0.2, 4.0, 1.0, 0.0, 0.0, 3, 4),
                               (3, 3, 1.0, -0.35, 5.75, 0.9, 0.2, 0.1, 4, 4)])
def test_packed_up_list_reproduces_oracle_columns(c):
    """The column pass's packed up list, decoded on the CPU: for x supported on one column c, the
    oracle's (H x)[:, c] minus the diagonal equals sum_j (-1)^s real2[cls] [p or conj p] times the
    column sign (-1)^(#down sites of c in [lo, hi)) times x[src_j, c] (up hops keep the column), to
    1e-14; a lattice with two Peierls phases has no packed list."""
    Lx, Ly, t, tp, U, V, px, py, nu, nd = c
    hops, pairs = F.build_hubbard_geometry(F.HubbardParams(Lx, Ly, t, tp, U, V, px, py))
    h = C.c_void_p()
    _lib.call("ftlm_gpu_sector_create_host", Lx * Ly, nu, nd, U, V, F.api._c_hops(hops), len(hops),
              F.api._c_pairs(pairs), len(pairs), C.byref(h))
    ok, ne = C.c_int(), C.c_longlong()
    _lib.call("ftlm_gpu_sector_up_table_packed", h, C.byref(ok), C.byref(ne), None, None, None, None)
    assert ok.value == (0 if (px != 0.0 and py != 0.0) else 1)
    if not ok.value:
        _lib.lib().ftlm_gpu_sector_destroy(h)
        return
    o = O.OracleSector(*c)
    up, dn = o.masks()
    Dd = int(np.count_nonzero(up == up[0]))
    Du = o.dim // Dd
    ptr = np.zeros(Du + 1, np.int32)
    ent = np.zeros(ne.value, np.uint32)
    real2, pcps = np.zeros(2), np.zeros(2)
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    _lib.call("ftlm_gpu_sector_up_table_packed", h, C.byref(ok), C.byref(ne), P(ptr), P(ent), P(real2), P(pcps))
    rng = np.random.default_rng(11)
    for col in (0, Dd // 2, Dd - 1):
        x = np.zeros(o.dim, np.complex128)
        x[col::Dd] = rng.standard_normal(Du) + 1j * rng.standard_normal(Du)
        ref = o.apply(x, mode=0)[col::Dd]
        d = int(dn[col])
        y = np.zeros(Du, np.complex128)
        v = C.c_double()
        for r in range(Du):
            _lib.call("ftlm_gpu_sector_diag", h, r * Dd + col, C.byref(v))
            y[r] = v.value * x[r * Dd + col]
            for e in ent[ptr[r]:ptr[r + 1]].tolist():
                src, lo, hi = e & 0x3FFF, (e >> 14) & 31, (e >> 19) & 31
                a = real2[(e >> 30) & 1] * (-1.0 if e >> 31 else 1.0)
                cf = complex(a * pcps[0], a * (-pcps[1] if (e >> 28) & 1 else pcps[1])) if (e >> 29) & 1 else a
                colsign = -1.0 if bin(d & ((1 << hi) - (1 << lo))).count("1") & 1 else 1.0
                y[r] += colsign * cf * x[src * Dd + col]
        assert np.abs(y - ref).max() <= 1e-14 * np.abs(ref).max()
    _lib.lib().ftlm_gpu_sector_destroy(h)
