"""aeromhd_cuda_b200 -- the AeroMHD-CUDA solver hot path on NVIDIA B200 (sm_100a).

A drop-in for the reference's ``config`` / ``physics`` / ``solver`` modules:

    from aeromhd_cuda_b200.config import Config
    from aeromhd_cuda_b200.solver import MHDSolver
    from aeromhd_cuda_b200.physics import cons_to_prim, prim_to_cons

State lives in PyTorch CUDA tensors; the arithmetic runs in libaeromhd.so
(hand-written CUDA for sm_100a, C ABI in include/aeromhd.h).  Importing the
package needs no GPU; constructing a solver does.
"""
from .config import (BX, BY, BZ, EN, FLOOR_PR, FLOOR_RHO, MX, MY, MZ, NVAR, PSI, RHO, RHOC, Config, ConsVar,
                     PrimVar, iBX, iBY, iBZ, iCLR, iPR, iPSI, iRHO, iVX, iVY, iVZ)

__version__ = "0.1.0"


def __getattr__(name):
    # heavy modules (torch) load on first use
    if name == "MHDSolver":
        from .solver import MHDSolver
        return MHDSolver
    if name in ("physics", "solver", "ensemble", "initial_conditions"):
        import importlib
        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
