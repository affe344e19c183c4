"""B200-native FTLM hot path for the 2D extended Hubbard model.

The compute lives in libftlm_gpu.so (hand-written sm_100a CUDA behind the C ABI in
include/ftlm_gpu.h); this package is the host-side mirror of the reference's interface.
"""
from .api import (FockBasis, FtlmParams, HubbardParams, LanczosExtrema, NearestPair, RectLattice, Sector,
                  OrbitKBlock, SpinfulHopping, SweepResult, apply_extended_hubbard, batched_release, build_hubbard_geometry,
                  ftlm_log_partition_complex, ftlm_log_partition_real, grand_canonical_sweep, lanczos_extrema,
                  lanczos_tridiagonal, nsites, quadrature, ritz_values, set_quadrature, tridiag_eig,
                  tridiag_quadrature, version_string)
from ._lib import FtlmError

__all__ = [
    "FockBasis", "FtlmParams", "HubbardParams", "LanczosExtrema", "NearestPair", "RectLattice", "Sector",
    "OrbitKBlock", "SpinfulHopping", "SweepResult", "apply_extended_hubbard", "batched_release", "build_hubbard_geometry",
    "ftlm_log_partition_complex", "ftlm_log_partition_real", "grand_canonical_sweep", "lanczos_extrema",
    "lanczos_tridiagonal", "nsites", "quadrature", "ritz_values", "set_quadrature", "tridiag_eig",
    "tridiag_quadrature", "version_string",
    "FtlmError",
]
