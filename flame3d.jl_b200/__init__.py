"""flame3d_b200 — B200-native (sm_100a) per-stage RHS and RK3 stage update of Flame3D.jl.

The compute path is the C-ABI library libflame3d_b200.so (include/flame3d_b200.h), built from
csrc/ by build.py.  This package is its host side: ctypes bindings (abi), seeded synthetic cases
(cases), a mirror of the reference stage loop (solver), batching and serving (serving).
There is no CPU fallback: without the library or a GPU every entry point raises.
"""
from .abi import (FLAME_MAX_NS, FLAME_NG, FlameError, FlameGrid, FlameMetrics,  # noqa: F401
                  FlameStageBuffers, FlameThermo, FlameTransport, header_symbols, load_library)
from .cases import (Case, Thermo, Transport, curvilinear_jet, ideal_air,  # noqa: F401
                    inflow_jet, mixing_layer, random_curvilinear, synthetic_species,
                    taylor_green)

__all__ = ["FlameError", "FlameGrid", "FlameMetrics", "FlameStageBuffers", "FlameThermo",
           "FlameTransport", "Case", "Thermo", "Transport", "load_library", "header_symbols",
           "taylor_green", "curvilinear_jet", "mixing_layer", "random_curvilinear",
           "inflow_jet", "ideal_air", "synthetic_species"]


def batch_module():
    """The batched-stage module (torch-backed, imported lazily)."""
    import importlib
    return importlib.import_module(__name__ + ".batch")


def solver_module():
    """The torch-backed solver module (imported lazily so `import flame3d_b200` stays light)."""
    import importlib
    return importlib.import_module(__name__ + ".solver")
