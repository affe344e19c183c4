"""The C++ drop-in of the reference's orbit k-block API (OrbitKBlockBasis, apply_orbit_k_block):
a reference-style caller (tests/dropin_orbit.cpp) is compiled against ftlm_extended_hubbard_b200/cpp/include
and libftlm_dropin.so, then checked against the facts of the reference's tests/test_orbit_k_block_basis.cpp
and against the reference library's golden block entries and H_K x."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

PKG = os.path.join(ROOT, "ftlm_extended_hubbard_b200")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("orbit_dropin") / "dropin_orbit")
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(PKG, "cpp", "include"), "-o", out,
           os.path.join(ROOT, "tests", "dropin_orbit.cpp"), "-L", PKG, "-lftlm_dropin", "-lftlm_gpu",
           f"-Wl,-rpath,{PKG}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_dropin_orbit_basis_facts(gpu, exe):
    r = subprocess.run([exe, "facts"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "ok orbit dims 12 66" in r.stdout


def test_dropin_orbit_apply_matches_reference(gpu, exe, golden, tmp_path):
    g = golden("orbit_small.npz")
    for k, c in enumerate(g["cases"]):
        Lx, Ly, t, tp, U, V, phx, phy, nu, nd, kx, ky = c
        assert phx == 0.0 and phy == 0.0
        x = g[f"x{k}"]
        xf, of = tmp_path / f"x{k}.bin", tmp_path / f"o{k}.bin"
        x.astype(np.complex128).tofile(xf)
        args = [exe, "apply"] + [str(int(Lx)), str(int(Ly))] + [repr(float(v)) for v in (t, tp, U, V)] + [
                                 str(int(nu)), str(int(nd)), str(int(kx)), str(int(ky)), str(xf), str(of)]
        r = subprocess.run(args, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (k, r.returncode, r.stderr)
        raw = of.read_bytes()
        dk = int(np.frombuffer(raw[:4], np.int32)[0])
        assert dk == g[f"rep{k}"].size
        rec = np.frombuffer(raw[4:4 + dk * 24], dtype=np.dtype([("rep", "<u4"), ("absA", "<f8"), ("size", "<i4"),
                                                                  ("oidx", "<i8")]))
        y = np.frombuffer(raw[4 + dk * 24:], np.complex128)
        assert np.array_equal(rec["rep"], g[f"rep{k}"])
        np.testing.assert_allclose(rec["absA"], g[f"absA{k}"], rtol=4 * 2.2e-16, atol=0)
        assert np.array_equal(rec["size"], g[f"size{k}"])
        assert np.all(np.diff(rec["oidx"]) > 0)  # orbit indices follow the ascending representatives
        assert np.abs(y - g[f"y{k}"]).max() <= 1e-13 * np.abs(g[f"y{k}"]).max(), k
