"""phlegethon_b200 -- B200-native explicit finite-volume step of the Phlegethon stellar
(M)HD code: PLM reconstruction with well-balanced hydrostatic subtraction, LHLLC/HLLC/HLLD/
LHLLD Riemann solvers, constrained transport, the Helmholtz EoS with its (rho, e) -> T
Newton inversion, RK stages and the CFL dt reduction, as hand-written sm_100a CUDA behind the
C ABI of include/phl_gpu.h.
"""
from .grid import Config, HostGrid  # noqa: F401
from . import helm_table, problems  # noqa: F401

__all__ = ["Config", "HostGrid", "helm_table", "problems", "Simulation", "load_library", "build"]


def load_library():
    from .abi import load_library as _ll
    return _ll()


def build(force=False, verbose=False):
    from .build import build as _b
    return _b(force=force, verbose=verbose)


def __getattr__(name):
    if name == "Simulation":
        from .abi import Simulation
        return Simulation
    raise AttributeError(name)
