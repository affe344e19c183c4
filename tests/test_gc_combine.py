"""Host-side combination of the differentiable ln Z_GC (autograd.gc_combine), on CPU: with the
oracle's per-sector ln Z_s(beta) and FTLM energies from fixed chains, d/dmu and d/dbeta of
log sum_s exp(ln Z_s + beta mu N_s) match central differences of the same estimator."""
import numpy as np

import oracle as O
from ftlm_extended_hubbard_b200.autograd import gc_combine

LAT = (3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0)
R, M, SEED = 4, 24, 7


def _table(betas):
    lz, es, N, _, _ = O.oracle_sweep(*LAT, R, M, SEED, np.atleast_1d(betas), np.array([0.0]), mode=1, nthreads=4)
    return lz, es, N.astype(np.float64)


def test_mu_and_beta_derivatives_match_central_differences():
    mu, beta, h = 1.3, 2.5, 1e-5
    lz, es, N = _table([beta - h, beta, beta + h])
    lnZ, w, dmu, dbeta = gc_combine(lz[:, 1], es[:, 1], N, mu, beta)
    assert abs(np.sum(w) - 1.0) < 1e-12
    fd_mu = (gc_combine(lz[:, 1], es[:, 1], N, mu + h, beta)[0] - gc_combine(lz[:, 1], es[:, 1], N, mu - h, beta)[0]) / (2 * h)
    fd_beta = (gc_combine(lz[:, 2], es[:, 2], N, mu, beta + h)[0] - gc_combine(lz[:, 0], es[:, 0], N, mu, beta - h)[0]) / (2 * h)
    assert abs(dmu - fd_mu) <= 1e-7 * max(1.0, abs(fd_mu)), (dmu, fd_mu)
    assert abs(dbeta - fd_beta) <= 1e-6 * max(1.0, abs(fd_beta)), (dbeta, fd_beta)
