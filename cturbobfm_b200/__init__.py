"""B200-native explicit residual-and-update loop of CTurboBFM.

The product is libctbfm.so (CUDA kernels for sm_100a behind the C ABI in
include/ctbfm.h); ``cturbobfm_b200.solver`` binds it for Python, and
``cturbobfm_b200.cases`` writes synthetic operating points in the reference's
input formats.
"""

from .solver import Batch, Server, Solver, SolverDiverged, CtbfmError, load_library  # noqa: F401

__all__ = ["Batch", "Server", "Solver", "SolverDiverged", "CtbfmError", "load_library"]
