"""Drop-in for the reference's gpu/gpu_assembler.py.

`from gpu_assembler import GPUSparseAssembler` (numerics/solvers.py:313) resolves here
when dissolve-2.0_b200/ is on sys.path.  This module IS dissolve_tp.assembler, so
module globals such as LUMP_MASS (read at call time, gpu_assembler.py:37, :504) behave
as in the reference: `gpu_assembler.LUMP_MASS = 0` switches to consistent mass.
"""
import sys as _sys

from dissolve_tp import assembler as _impl

_sys.modules[__name__] = _impl
