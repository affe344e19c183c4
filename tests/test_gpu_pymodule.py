"""The reference's Python package layout (python/ftlm over the pybind11 module _ftlm_core) with the
GPU path behind it: `import ftlm`, H·v on a CUDA tensor, Lanczos, a grand-canonical sweep and the
differentiable ln Z_GC with lnZ.backward(), each against the oracle (the reference's algorithm,
pinned bit-exact to the reference build).

Bars as elsewhere: H·v 1e-13 relative, Lanczos alpha of the first steps 1e-12, ln Z / <n> 1e-10
relative, the autograd gradient within 1e-5 of central differences (h = 1e-4) of the oracle."""
import os
import sys

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
H = 1e-4


@pytest.fixture(scope="module")
def ftlm(gpu):
    sys.path.insert(0, os.path.join(ROOT, "ftlm_extended_hubbard_b200", "python"))
    import ftlm as mod
    return mod


def test_reference_exports_unchanged(ftlm):
    p = ftlm.HubbardParams()
    assert (p.Lx, p.Ly, p.t, p.tp, p.U, p.V, p.phi_x, p.phi_y) == (2, 2, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    q = ftlm.HubbardParams(Lx=4, Ly=3, tp=-0.25, U=8.0)
    assert ftlm.nsites(q) == 12 and ftlm.nsites(params=p) == 4
    assert isinstance(ftlm.version_string(), str)


def test_apply_on_cuda_tensor_matches_oracle(ftlm, gpu):
    torch = gpu
    c = (4, 4, 1.0, -0.25, 8.0, 1.0, 0.1, 0.0, 3, 4)
    s = ftlm.Sector(ftlm.HubbardParams(*c[:8]), c[8], c[9])
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(s.dim(), dtype=torch.complex128, device="cuda", generator=g)
    y = s.apply(x)
    yo = O.OracleSector(*c).apply(x.cpu().numpy(), mode=1, nthreads=8)
    err = np.abs(y.cpu().numpy() - yo).max() / np.abs(yo).max()
    assert err < 1e-13, err
    out = torch.empty_like(x)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # runs on torch's current stream
        s.apply(x, out=out)
    torch.cuda.current_stream().wait_stream(side)
    assert torch.equal(out, y)
    with pytest.raises(RuntimeError, match="CUDA tensor"):
        s.apply(x.cpu())  # no CPU fallback
    b = ftlm.Sector(ftlm.HubbardParams(*c[:8]), c[8], c[9])
    assert b.index_of(b.up_mask(17), b.down_mask(17)) == 17


def test_lanczos_and_ftlm_match_oracle(ftlm):
    c = (4, 2, 1.0, -0.25, 8.0, 1.0, 0.0, 0.0, 4, 4)
    s = ftlm.Sector(ftlm.HubbardParams(*c[:8]), 4, 4)
    o = O.OracleSector(*c)
    a, b = s.lanczos(30, 7)
    ao, bo, _ = o.lanczos(30, 7, mode=0)
    assert np.all(np.abs(a.numpy()[:10] - ao[:10]) <= 1e-12 * np.abs(ao[:10]).max())
    lz, en = s.ftlm(np.array([0.5, 2.0]), 4, 30, 7)
    lzo, eno = o.ftlm([0.5, 2.0], 4, 30, 7, mode=0)
    assert np.all(np.abs(lz.numpy() - lzo) <= 1e-10 * np.abs(lzo))
    assert np.all(np.abs(en.numpy() - eno) <= 1e-10 * np.abs(eno))


def test_sweep_matches_golden(ftlm, gpu, golden):
    torch = gpu
    g = golden("sweep_4x2.npz")
    Lx, Ly, t, tp, U, V, px, py, R, M, seed = g["params"]
    p = ftlm.HubbardParams(int(Lx), int(Ly), t, tp, U, V, px, py)
    out = ftlm.grand_canonical_sweep(p, int(R), int(M), int(seed), g["T"], g["mu"])
    assert np.all(np.abs(out["lnz"].numpy() - g["lnz_gc"]) <= 1e-10 * np.abs(g["lnz_gc"]))
    assert np.all(np.abs(out["n"].numpy() - g["n_gc"]) <= 1e-10 * np.maximum(1.0, np.abs(g["n_gc"])))


def test_differentiable_lnz_backward_matches_oracle(ftlm, gpu):
    """ln Z_GC of 2x2 (25 sectors, R=6, M=20, reference start vectors) through the module's
    autograd Function: forward against the oracle, lnZ.backward() against central differences of
    the oracle's ln Z_GC at shifted (U, V, t', mu, beta)."""
    torch = gpu
    Lx, Ly, R, M, seed = 2, 2, 6, 20, 7
    th0 = np.array([4.0, 1.0, -0.2, 1.0, 2.0])
    theta = torch.tensor(th0, dtype=torch.float64, requires_grad=True)
    lnZ = ftlm.grand_canonical_logz(theta, Lx, Ly, R, M, seed, method="plain", start="reference")
    lnZ.backward()

    def oracle_lnz(th):
        U, V, tp, mu, beta = th
        gl = O.oracle_sweep(Lx, Ly, 1.0, tp, U, V, 0.0, 0.0, R, M, seed, np.array([beta]), np.array([mu]))[4][0]
        return float(np.asarray(gl).ravel()[0])

    assert abs(lnZ.item() - oracle_lnz(th0)) <= 1e-10 * abs(lnZ.item())
    fd = np.array([(oracle_lnz(th0 + H * e) - oracle_lnz(th0 - H * e)) / (2 * H) for e in np.eye(5)])
    assert np.all(np.abs(theta.grad.numpy() - fd) <= 1e-5 * np.maximum(1.0, np.abs(fd))), (theta.grad, fd)
