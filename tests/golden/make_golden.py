"""Generates the golden fixtures under tests/golden/ (run where the reference sources exist):

    python tests/golden/make_golden.py

published_tsv.npz  the reference's own published n(mu) tables (benchmarks/data/*.tsv of
                   PeizhiMai/FTLM_extended_Hubbard), parsed: 2x2 and 4x2 from bench_ftlm_nmu_rect,
                   3x2 from the non-momentum solver; plus the per-sector ln Z lines of the 3x2 run log.
ref_small.npz      outputs of the reference library itself (oracle/_ref): H·x on seeded vectors,
                   Lanczos alpha/beta, lanczos_extrema, and sector ln Z for small sectors.
published_korbit.npz  the reference's published k-orbit run on 3x2 (benchmarks/data/
                   n_vs_mu_3x2_beta20_four_solver_monitoring.txt, "solver=k-orbit" block): per-sector
                   dim_k_total and ln Z (printed digits kept) at beta=20, R=12, M=72, seed 7, ed-cutoff 64.
orbit_small.npz    translation-orbit momentum blocks from the reference library (OrbitKBlockBasis::build,
                   apply_orbit_k_block, ftlm_log_partition_complex): representatives, |A|, orbit sizes,
                   H_K x on seeded vectors and block ln Z.
ritz_4x4_8_8.npz   the 4x4 (8,8) Lanczos chain of the single-sector workload (dim 165,636,900,
                   t=1 t'=-0.25 U=8 V=1 phi_x=0.1, reference start vector seed 7, M=150): alpha, beta
                   and the lowest 5 Ritz values, computed by the oracle's threaded row gather with the
                   reference recurrence (about 1.5-2 h on 8 host threads; made only on request:
                   `python tests/golden/make_golden.py ritz_4x4_8_8`).
ed_4x2.npz         full exact diagonalisation of the 4x2 lattice (t=1 t'=-0.25 U=8 V=1, phi=0, all 65,536
                   levels) by the reference's own NumPy ED mirror (benchmarks/hubbard_rect_ed.py,
                   imported from the reference checkout): exact per-sector ln Z and ln Z_GC / <n> on
                   the T x mu grid of sweep_4x2 (a few minutes; `python tests/golden/make_golden.py ed_4x2`).
sweep_4x2.npz    the plain FTLM sweep of 4x2, t=1 t'=-0.25 U=8 V=1, phi=0, R=20, M=60, seed 7,
                   T = 0.1..2.0 (20) x mu = -4..8 (49), computed by the oracle in the reference's
                   scatter order (bit-identical to the reference library; this script checks the
                   sector ln Z of several sectors against the reference itself before writing).
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

REF_DATA = os.path.join(O.REFERENCE_SRC, "benchmarks", "data")

SMALL_CASES = [
    # Lx, Ly, t, tp, U, V, phix, phiy, nu, nd
    (2, 2, 1.0, 0.0, 0.0, 0.0, 0.31, -0.27, 2, 2),
    (2, 1, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1, 1),
    (3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0, 2, 3),
    (4, 2, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0, 4, 4),
    (4, 2, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0, 3, 1),
    (3, 3, 1.0, -0.35, 5.75, 0.9, 0.2, 0.1, 4, 5),
    (4, 3, 1.0, -0.25, 8.0, 1.0, 0.1, 0.0, 3, 2),
    (5, 1, 1.0, 0.3, 2.0, 0.5, 0.4, 0.0, 2, 3),
    (1, 4, 1.0, 0.0, 3.0, 0.0, 0.0, 0.7, 2, 1),
]


def parse_tsv(path):
    mu, n = [], []
    hdr = []
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                hdr.append(line.strip())
                continue
            a, b = line.split()
            mu.append(float(a))
            n.append(float(b))
    return np.array(mu), np.array(n), "\n".join(hdr)


def published():
    out = {}
    for key, fn in [("2x2", "n_vs_mu_2x2_beta20_ftlm.tsv"), ("4x2", "n_vs_mu_4x2_beta20_ftlm.tsv"),
                    ("3x2_nonmom", "n_vs_mu_3x2_beta20_solver_nonmom.tsv"), ("3x3", "n_vs_mu_3x3_beta20_ftlm.tsv"),
                    ("2x5", "n_vs_mu_2x5_beta20_ftlm.tsv"), ("3x2_korbit", "n_vs_mu_3x2_beta20_solver_k_orbit.tsv")]:
        mu, n, hdr = parse_tsv(os.path.join(REF_DATA, fn))
        out[f"{key}_mu"] = mu
        out[f"{key}_n"] = n
        out[f"{key}_header"] = np.array(hdr)
    # per-sector ln Z printed by the 3x2 non-momentum run (6 significant digits)
    sec, lz = [], []
    with open(os.path.join(REF_DATA, "n_vs_mu_3x2_beta20_four_solver_monitoring.txt")) as f:
        in_block = False
        for line in f:
            if "solver=nonmom" in line:
                in_block = True
            elif in_block and line.startswith("---"):
                break
            m = re.match(r"sector \((\d+),(\d+)\) dim=(\d+) logZ=(\S+)", line.strip())
            if in_block and m:
                sec.append((int(m.group(1)), int(m.group(2)), int(m.group(3))))
                lz.append(float(m.group(4)))
    out["3x2_sector"] = np.array(sec, np.int64)
    out["3x2_sector_lnz"] = np.array(lz)
    return out


def ref_small():
    R = O.reference()
    assert R is not None, "reference library unavailable"
    out = {"cases": np.array(SMALL_CASES, dtype=np.float64)}
    rng = np.random.default_rng(20240601)
    import ctypes as C
    for k, c in enumerate(SMALL_CASES):
        h = R.ref_sector_create(*c)
        dim = R.ref_sector_dim(h)
        x = rng.standard_normal(dim) + 1j * rng.standard_normal(dim)
        x[rng.random(dim) < 0.05] = 0.0  # zero columns exercise the skip rule
        y = np.zeros(dim, np.complex128)
        R.ref_sector_apply(h, O.P(x), O.P(y))
        M = 40
        a = np.zeros(M)
        b = np.zeros(M)
        nb = C.c_int()
        used = R.ref_sector_lanczos(h, M, 11 + k, O.P(a), O.P(b), C.byref(nb))
        mn, mx = C.c_double(), C.c_double()
        ue = R.ref_sector_lanczos_extrema(h, 30, 5, C.byref(mn), C.byref(mx))
        lz = R.ref_sector_ftlm_complex(h, 2.0, 6, 30, 3)
        up = np.zeros(dim, np.uint64)
        dn = np.zeros(dim, np.uint64)
        R.ref_sector_masks(h, O.P(up), O.P(dn))
        out[f"x{k}"] = x
        out[f"y{k}"] = y
        out[f"up{k}"] = up
        out[f"dn{k}"] = dn
        out[f"alpha{k}"] = a[:used]
        out[f"beta{k}"] = b[:nb.value]
        out[f"extrema{k}"] = np.array([mn.value, mx.value, ue])
        out[f"lnz{k}"] = np.array([lz])
        R.ref_sector_destroy(h)
    # tests/test_ftlm_thermo.cpp known answer: diag(2,3), beta=1, R=48, M=32, seed 12345
    d = np.array([2.0, 3.0])
    out["diag23_lnz"] = np.array([R.ref_ftlm_diag_real(O.P(d), 2, 1.0, 48, 32, 12345)])
    return out


def published_korbit():
    txt = open(os.path.join(REF_DATA, "n_vs_mu_3x2_beta20_four_solver_monitoring.txt")).read()
    sec = txt[txt.index("--- 3) solver=k-orbit"):]
    rows = re.findall(r"sector \((\d+),(\d+)\) dim_full=(\d+) dim_k_total=(\d+) ed_blocks=(\d+) "
                      r"ftlm_blocks=(\d+) logZ=(\S+)", sec)[:49]
    assert len(rows) == 49
    nu, nd, dfull, dk, ed, fb, lz = zip(*rows)
    dec = [len(v.split(".")[1]) if "." in v else 0 for v in lz]
    return {"nu": np.array(nu, np.int32), "nd": np.array(nd, np.int32), "dim_full": np.array(dfull, np.int64),
            "dim_k_total": np.array(dk, np.int64), "ed_blocks": np.array(ed, np.int32),
            "ftlm_blocks": np.array(fb, np.int32), "lnz": np.array([float(v) for v in lz]),
            "decimals": np.array(dec, np.int32),
            "params": np.array([3, 2, 1.0, -0.35, 5.75, 0.9, 20.0, 12, 72, 7, 64], np.float64)}


ORBIT_CASES = [
    # Lx, Ly, t, tp, U, V, phix, phiy, nu, nd, kx, ky
    (2, 2, 1.0, 0.0, 4.0, 0.5, 0.0, 0.0, 2, 2, 0, 0),
    (2, 2, 1.0, 0.0, 4.0, 0.5, 0.0, 0.0, 2, 2, 1, 1),
    (3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0, 2, 3, 1, 0),
    (3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0, 3, 3, 1, 0),
    (4, 2, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0, 3, 3, 2, 1),
    (3, 3, 1.0, -0.25, 6.0, 0.5, 0.0, 0.0, 2, 2, 1, 2),
    (4, 3, 1.0, -0.25, 6.0, 0.5, 0.0, 0.0, 2, 1, 3, 2),
    (4, 4, 1.0, -0.25, 6.0, 0.5, 0.0, 0.0, 2, 1, 1, 3),
]


def orbit_small():
    R = O.reference()
    assert R is not None, "reference library unavailable"
    out = {"cases": np.array(ORBIT_CASES, dtype=np.float64)}
    rng = np.random.default_rng(20240602)
    for k, c in enumerate(ORBIT_CASES):
        h = R.ref_sector_create(*c[:10])
        o = R.ref_orbit_create(h, c[10], c[11])
        dk = R.ref_orbit_dim(o)
        rep = np.zeros(dk, np.uint32)
        absA = np.zeros(dk)
        size = np.zeros(dk, np.int32)
        R.ref_orbit_entries(o, O.P(rep), O.P(absA), O.P(size))
        x = rng.standard_normal(dk) + 1j * rng.standard_normal(dk)
        x[rng.random(dk) < 0.05] = 0.0
        y = np.zeros(dk, np.complex128)
        R.ref_orbit_apply(o, O.P(x), O.P(y))
        out[f"rep{k}"] = rep
        out[f"absA{k}"] = absA
        out[f"size{k}"] = size
        out[f"x{k}"] = x
        out[f"y{k}"] = y
        out[f"lnz{k}"] = np.array([R.ref_orbit_ftlm_complex(o, 1.3, 5, 30, 17 + k)])
        R.ref_orbit_destroy(o)
        R.ref_sector_destroy(h)
    return out


SWEEP_4X2 = dict(Lx=4, Ly=2, t=1.0, tp=-0.25, U=8.0, V=1.0, phix=0.0, phiy=0.0, R=20, M=60, seed=7)
T_GRID = np.round(np.arange(1, 21) * 0.1, 10)
MU_GRID = np.round(np.arange(49) * 0.25 - 4.0, 10)


def sweep_4x2():
    c = SWEEP_4X2
    betas = 1.0 / T_GRID
    lz, es, N, dims, (g_lnz, g_n, g_e) = O.oracle_sweep(c["Lx"], c["Ly"], c["t"], c["tp"], c["U"], c["V"], c["phix"],
                                                       c["phiy"], c["R"], c["M"], c["seed"], betas, MU_GRID, mode=0)
    # Pin against the reference library on sectors spanning small to largest, two temperatures.
    R = O.reference()
    n = c["Lx"] * c["Ly"]
    for nu, nd in [(0, 1), (1, 1), (2, 3), (4, 4), (8, 8), (3, 5)]:
        idx = nu * (n + 1) + nd
        h = R.ref_sector_create(c["Lx"], c["Ly"], c["t"], c["tp"], c["U"], c["V"], c["phix"], c["phiy"], nu, nd)
        for bi in (0, 9):
            ref = R.ref_sector_ftlm_real(h, float(betas[bi]), c["R"], c["M"], c["seed"])
            assert ref == lz[idx, bi], (nu, nd, bi, ref, lz[idx, bi])
        R.ref_sector_destroy(h)
    return {"lnz_sector": lz, "e_sector": es, "N": N, "dims": dims, "T": T_GRID, "mu": MU_GRID,
            "lnz_gc": g_lnz, "n_gc": g_n, "e_gc": g_e,
            "params": np.array([c["Lx"], c["Ly"], c["t"], c["tp"], c["U"], c["V"], c["phix"], c["phiy"], c["R"],
                                c["M"], c["seed"]], dtype=np.float64)}


RITZ_4X4 = (4, 4, 1.0, -0.25, 8.0, 1.0, 0.1, 0.0, 8, 8)


def ritz_4x4_8_8(nthreads=None):
    """The single-sector workload's chain (src/lanczos.cpp:125-208 restated, threaded gather H·v)."""
    import time
    nthreads = nthreads or os.cpu_count() or 8
    s = O.OracleSector(*RITZ_4X4)
    t0 = time.time()
    a, b, used = s.lanczos(150, 7, mode=1, nthreads=nthreads)
    secs = time.time() - t0
    n = len(a)
    T = np.diag(a) + np.diag(b[:n - 1], 1) + np.diag(b[:n - 1], -1)
    ritz = np.linalg.eigvalsh(T)[:5]
    return {"params": np.array(RITZ_4X4, np.float64), "M": np.array([150]), "seed": np.array([7]),
            "alpha": a, "beta": b, "used": np.array([used]), "ritz5": ritz, "seconds": np.array([secs]),
            "threads": np.array([nthreads])}


ED_4X2 = dict(t=1.0, tp=-0.25, U=8.0, V=1.0)


def ed_4x2():
    """Exact spectrum of every (N_up, N_dn) sector of 4x2 from the reference's NumPy ED mirror
    (benchmarks/hubbard_rect_ed.py:45-213); the grand-canonical reduction follows its
    grand_canonical_n (log-sum-exp over all levels)."""
    sys.path.insert(0, os.path.join(O.REFERENCE_SRC, "benchmarks"))
    import hubbard_rect_ed as ED  # the reference's own ED script
    lx, ly = 4, 2
    n = lx * ly
    hops, pairs = ED.build_hubbard_geometry_py(lx, ly, ED_4X2["t"], ED_4X2["tp"], 0.0, 0.0)
    betas = 1.0 / T_GRID
    lnz_s = np.full(((n + 1) ** 2, betas.size), -np.inf)
    N = np.zeros((n + 1) ** 2, np.int32)
    levels = []
    for nu in range(n + 1):
        for nd in range(n + 1):
            idx = nu * (n + 1) + nd
            N[idx] = nu + nd
            basis = ED.enumerate_sector(n, nu, nd)
            h = ED.build_h_sector(basis, hops, pairs, ED_4X2["U"], ED_4X2["V"])
            w = np.linalg.eigvalsh((h + np.conjugate(h.T)) * 0.5)
            levels.append((w, nu + nd))
            for bi, b in enumerate(betas):
                a = -b * w
                m = a.max()
                lnz_s[idx, bi] = m + np.log(np.exp(a - m).sum())
    lnz_gc = np.zeros((betas.size, MU_GRID.size))
    n_gc = np.zeros_like(lnz_gc)
    E = np.concatenate([w for w, _ in levels])
    Nl = np.concatenate([np.full(w.size, k, np.float64) for w, k in levels])
    for bi, b in enumerate(betas):
        for mi, mu in enumerate(MU_GRID):
            a = -b * (E - mu * Nl)
            m = a.max()
            wts = np.exp(a - m)
            lnz_gc[bi, mi] = m + np.log(wts.sum())
            n_gc[bi, mi] = (Nl * wts).sum() / wts.sum() / n
            # cross-check against the reference script's own reduction on a few points
            if bi % 9 == 0 and mi % 16 == 0:
                ref_n = ED.grand_canonical_n(float(b), float(mu), list(zip(E.tolist(), Nl.astype(int).tolist())), n)
                assert abs(ref_n - n_gc[bi, mi]) < 1e-12, (b, mu, ref_n, n_gc[bi, mi])
    return {"lnz_sector": lnz_s, "N": N, "T": T_GRID, "mu": MU_GRID, "lnz_gc": lnz_gc, "n_gc": n_gc,
            "params": np.array([lx, ly, ED_4X2["t"], ED_4X2["tp"], ED_4X2["U"], ED_4X2["V"], 0.0, 0.0])}


ON_REQUEST = {"ritz_4x4_8_8": ritz_4x4_8_8, "ed_4x2": ed_4x2}


def main():
    wanted = [a for a in sys.argv[1:] if a in ON_REQUEST]
    if wanted:
        O.build(ref=False)
        for name in wanted:
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **ON_REQUEST[name]())
            print("wrote", name + ".npz")
        return
    O.build(ref=True)
    np.savez_compressed(os.path.join(HERE, "published_tsv.npz"), **published())
    np.savez_compressed(os.path.join(HERE, "ref_small.npz"), **ref_small())
    np.savez_compressed(os.path.join(HERE, "orbit_small.npz"), **orbit_small())
    np.savez_compressed(os.path.join(HERE, "published_korbit.npz"), **published_korbit())
    np.savez_compressed(os.path.join(HERE, "sweep_4x2.npz"), **sweep_4x2())
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
