"""dissolve_tp -- B200-native P1-tetrahedral reaction-diffusion transport path.

Drop-in for the transport hot path of Dissolve 2.0: GPUSparseAssembler
(gpu/gpu_assembler.py), CeedDiffusionMassOp (gpu/ceed_operators.py) and the Krylov
solve of solve_transport (numerics/solvers.py), on hand-written sm_100a kernels
behind the C ABI of include/dissolve_tp.h.
"""
from .mesh import TetMesh, kuhn_cube, kuhn_counts, gyroid_cube, face_dofs  # noqa: F401

__version__ = "1.0.0"


def __getattr__(name):
    # GPU-facing modules load the shared library; import them lazily so the mesh
    # generator stays usable on machines without the library.
    if name in ("GPUSparseAssembler", "DeviceMesh", "CsrMatrix", "LUMP_MASS"):
        from . import assembler
        return getattr(assembler, name)
    if name in ("CsrOperator", "CGSolver"):
        from . import krylov
        return getattr(krylov, name)
    raise AttributeError(name)
