"""The reference's own test and driver programs, compiled unmodified against the C++ drop-in
(ftlm_extended_hubbard_b200/cpp/include, libftlm_dropin.so) by `make -C oracle dropin`, run on the GPU."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref", "dropin")


def prog(name):
    p = os.path.join(BIN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not built (make -C oracle dropin needs the reference sources)")
    return p


def run(args, timeout=600):
    r = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    return r.returncode, r.stdout, r.stderr


def test_reference_smoke_and_pipeline_tests(gpu):
    assert run([prog("smoke")])[0] == 0
    rc, out, err = run([prog("test_hubbard_pipeline")])
    assert rc == 0, out + err
    assert "test_hubbard_pipeline ok" in out


def test_reference_ftlm_thermo_test(gpu):
    rc, out, err = run([prog("test_ftlm_thermo")])
    assert rc == 0, out + err


def test_reference_driver_reproduces_published_2x2_table(gpu, golden, tmp_path):
    """bench_ftlm_nmu_rect --Lx=2 --Ly=2 (reference defaults: beta=20, t'=-0.35, U=5.75, V=0.9,
    R=12, M=72, seed 7, mu in [-5,25] x 221) through the GPU library vs the published TSV."""
    g = golden("published_tsv.npz")
    mu_pub, n_pub = g["2x2_mu"], g["2x2_n"]
    out = tmp_path / "n.tsv"
    rc, so, se = run([prog("bench_ftlm_nmu_rect"), "--Lx=2", "--Ly=2", f"--mu-min={mu_pub[0]}",
                      f"--mu-max={mu_pub[-1]}", f"--n-mu={mu_pub.size}", f"--out={out}", "--no-monitor=1"])
    assert rc == 0, so + se
    rows = [ln.split() for ln in open(out) if not ln.startswith("#")]
    mu = np.array([float(a) for a, _ in rows])
    n = np.array([float(b) for _, b in rows])
    assert np.array_equal(mu, mu_pub)
    # printed with 6 significant digits by the driver on both sides
    assert np.all(np.abs(n - n_pub) <= 1e-5 * np.abs(n_pub) + 1e-300)


def test_reference_4x2_lanczos_driver(gpu):
    rc, out, err = run([prog("bench_4x2_ftlm"), "--samples=2", "--lanczos-steps=20"])
    assert rc == 0, out + err
