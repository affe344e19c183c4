"""The allocation-free quadrature entry point, ftlm_gpu_tridiag_quadrature_noalloc.

It serves callers that must not call cudaMalloc/cudaFree on this path: code whose device memory is
owned by another allocator (a framework pool that has already reserved most of HBM, where a direct
cudaMalloc can fail or fragment the pool) and latency-critical loops where an allocation would
implicitly synchronise the device.  The caller passes device inputs and outputs; the library keeps
the intermediate Ritz pairs in its own fixed 1 MiB device array.

Checked here, through the C ABI: the output equals the allocating entry point
(ftlm_gpu_tridiag_quadrature) within the tests' thermodynamic tolerance on two calls in a row with
different inputs (the shared scratch carries nothing over), the second call changes no device
allocation, and requests larger than the scratch are rejected before any GPU work.  Edge cases:
a batch that fills the scratch exactly (512 chains x ld 128), the largest ld (160), chains of
length 0 (-inf, as the allocating path), work queued on a side stream behind other work, and a
device-resident chain length above ld (skipped in-bounds, NaN outputs, FTLM_ERR_INVALID).
This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import ftlm_extended_hubbard_b200 as F
from ftlm_extended_hubbard_b200 import _lib

pytestmark = pytest.mark.gpu

RTOL_THERMO = 1e-10


def _batch(seed, n_chains, ld, n_zero=0):
    rng = np.random.default_rng(seed)
    n = rng.integers(1, ld + 1, n_chains).astype(np.int32)
    n[0] = ld
    n[1:1 + n_zero] = 0
    A = np.zeros((n_chains, ld))
    B = np.zeros((n_chains, ld))
    for c in range(n_chains):
        A[c, :n[c]] = rng.standard_normal(n[c]) * 4.0
        B[c, :n[c]] = np.abs(rng.standard_normal(n[c])) + 0.05
    return A, B, n


def _mem_free(torch):
    free, _ = torch.cuda.mem_get_info()
    return free


def test_noalloc_quadrature_matches_allocating_entry_point(gpu):
    torch = gpu
    bts = np.array([0.05, 0.5, 1.0, 5.0, 20.0])
    bts_d = torch.tensor(bts, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for call, (seed, n_chains, ld) in enumerate([(1, 24, 60), (2, 9, 37)]):
        A, B, n = _batch(seed, n_chains, ld)
        ref_q, ref_e = F.tridiag_quadrature(A, B, n, bts)
        a_d = torch.tensor(A, device="cuda")
        b_d = torch.tensor(B, device="cuda")
        n_d = torch.tensor(n, device="cuda")
        q_d = torch.full((n_chains, bts.size), float("nan"), dtype=torch.float64, device="cuda")
        e_d = torch.full_like(q_d, float("nan"))
        torch.cuda.synchronize()
        free0 = _mem_free(torch)
        _lib.call("ftlm_gpu_tridiag_quadrature_noalloc", C.c_void_p(a_d.data_ptr()), C.c_void_p(b_d.data_ptr()),
                  C.c_void_p(n_d.data_ptr()), n_chains, ld, C.c_void_p(bts_d.data_ptr()), bts.size,
                  C.c_void_p(q_d.data_ptr()), C.c_void_p(e_d.data_ptr()), C.c_void_p(stream.cuda_stream))
        torch.cuda.synchronize()
        if call == 1:  # after the first call's one-time set-up, no device memory may change hands
            assert _mem_free(torch) == free0
        q, e = q_d.cpu().numpy(), e_d.cpu().numpy()
        assert np.all(np.abs(q - ref_q) <= RTOL_THERMO * np.maximum(1.0, np.abs(ref_q))), call
        assert np.all(np.abs(e - ref_e) <= RTOL_THERMO * np.maximum(1.0, np.abs(ref_e))), call


def test_noalloc_rejects_oversized_batch(gpu):
    torch = gpu
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    ni = torch.ones(8, dtype=torch.int32, device="cuda")
    with pytest.raises(F.FtlmError) as e:
        _lib.call("ftlm_gpu_tridiag_quadrature_noalloc", C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()),
                  C.c_void_p(ni.data_ptr()), 500, 150, C.c_void_p(x.data_ptr()), 1, C.c_void_p(x.data_ptr()),
                  C.c_void_p(x.data_ptr()), None)
    assert e.value.code == _lib.FTLM_ERR_UNSUPPORTED
    assert "65536" in str(e.value)


def _noalloc(torch, A, B, n, bts, stream, n_override=None):
    n_chains, ld = A.shape
    a_d = torch.tensor(A, device="cuda")
    b_d = torch.tensor(B, device="cuda")
    n_d = torch.tensor(n if n_override is None else n_override, device="cuda")
    bts_d = torch.tensor(bts, dtype=torch.float64, device="cuda")
    q_d = torch.full((n_chains, bts.size), 7.0, dtype=torch.float64, device="cuda")
    e_d = torch.full_like(q_d, 7.0)
    err = None
    try:
        _lib.call("ftlm_gpu_tridiag_quadrature_noalloc", C.c_void_p(a_d.data_ptr()), C.c_void_p(b_d.data_ptr()),
                  C.c_void_p(n_d.data_ptr()), n_chains, ld, C.c_void_p(bts_d.data_ptr()), bts.size,
                  C.c_void_p(q_d.data_ptr()), C.c_void_p(e_d.data_ptr()), C.c_void_p(stream.cuda_stream))
    except F.FtlmError as ex:
        err = ex
    torch.cuda.synchronize()
    return q_d.cpu().numpy(), e_d.cpu().numpy(), err


def _close(x, ref):
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(x))
    assert np.array_equal(x[~fin], ref[~fin])
    return np.all(np.abs(x[fin] - ref[fin]) <= RTOL_THERMO * np.maximum(1.0, np.abs(ref[fin])))


@pytest.mark.parametrize("n_chains,ld,n_zero", [(512, 128, 3), (5, 160, 1)])
def test_noalloc_edges_full_scratch_max_ld_empty_chains(gpu, n_chains, ld, n_zero):
    torch = gpu
    bts = np.array([0.1, 1.0, 10.0])
    A, B, n = _batch(40 + ld, n_chains, ld, n_zero)
    ref_q, ref_e = F.tridiag_quadrature(A, B, n, bts)
    assert np.all(np.isneginf(ref_q[1:1 + n_zero]))
    q, e, err = _noalloc(torch, A, B, n, bts, torch.cuda.current_stream())
    assert err is None
    assert _close(q, ref_q) and _close(e, ref_e)


def test_noalloc_on_side_stream_behind_other_work(gpu):
    torch = gpu
    bts = np.array([0.3, 3.0])
    A, B, n = _batch(77, 64, 90)
    ref_q, ref_e = F.tridiag_quadrature(A, B, n, bts)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        big = torch.randn(1 << 24, device="cuda")
        for _ in range(4):  # queued work the quadrature has to wait behind
            big = big * 1.0001 + 0.5
        q, e, err = _noalloc(torch, A, B, n, bts, side)
    assert err is None
    assert _close(q, ref_q) and _close(e, ref_e)


def test_noalloc_chain_longer_than_ld_is_reported(gpu):
    """A device-resident chain length of ld + 1 cannot be checked on the host: the kernels skip
    that chain without touching memory past its rows, set its outputs to NaN and the call returns
    FTLM_ERR_INVALID; the other chains are still correct, and the next call works normally."""
    torch = gpu
    bts = np.array([0.5, 2.0])
    ld = 40
    A, B, n = _batch(5, 6, ld)
    bad = n.copy()
    bad[2] = ld + 1
    ref_q, ref_e = F.tridiag_quadrature(A, B, n, bts)
    q, e, err = _noalloc(torch, A, B, n, bts, torch.cuda.current_stream(), n_override=bad)
    assert err is not None and err.code == _lib.FTLM_ERR_INVALID
    assert np.all(np.isnan(q[2])) and np.all(np.isnan(e[2]))
    keep = np.arange(6) != 2
    assert _close(q[keep], ref_q[keep]) and _close(e[keep], ref_e[keep])
    q, e, err = _noalloc(torch, A, B, n, bts, torch.cuda.current_stream())
    assert err is None and _close(q, ref_q) and _close(e, ref_e)
