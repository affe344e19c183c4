"""The allocation-free quadrature entry point, ftlm_gpu_tridiag_quadrature_noalloc.

It serves callers that must not call cudaMalloc/cudaFree on this path: code whose device memory is
owned by another allocator (a framework pool that has already reserved most of HBM, where a direct
cudaMalloc can fail or fragment the pool) and latency-critical loops where an allocation would
implicitly synchronise the device.  The caller passes device inputs and outputs; the library keeps
the intermediate Ritz pairs in its own fixed 1 MiB device array.

Checked here, through the C ABI: the output equals the allocating entry point
(ftlm_gpu_tridiag_quadrature) within the tests' thermodynamic tolerance on two calls in a row with
different inputs (the shared scratch carries nothing over), the second call changes no device
allocation, and requests larger than the scratch are rejected before any GPU work.
This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import ftlm_extended_hubbard_b200 as F
from ftlm_extended_hubbard_b200 import _lib

pytestmark = pytest.mark.gpu

RTOL_THERMO = 1e-10


def _batch(seed, n_chains, ld):
    rng = np.random.default_rng(seed)
    n = rng.integers(1, ld + 1, n_chains).astype(np.int32)
    n[0] = ld
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
