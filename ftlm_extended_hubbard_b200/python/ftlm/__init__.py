"""Python package of ftlm_extended_hubbard, laid out as the reference's python/ftlm.

The reference's package re-exports its pybind11 module _ftlm_core (HubbardParams, nsites,
version_string).  Here the same module also carries the GPU hot path on torch tensors: Sector
(FockBasis + apply_extended_hubbard / lanczos / ftlm on the B200), grand_canonical_sweep, and the
differentiable grand_canonical_logz (a torch.autograd.Function with a hand-written backward).
Put this directory (ftlm_extended_hubbard_b200/python) on sys.path to `import ftlm`.
"""

import torch  # noqa: F401  (the extension links libtorch; import it first)

from ._ftlm_core import (HubbardParams, Sector, grand_canonical_logz, grand_canonical_sweep, nsites,
                         release_workspaces, version_string)

__all__ = ["HubbardParams", "nsites", "version_string", "Sector", "grand_canonical_sweep", "grand_canonical_logz",
           "release_workspaces"]
