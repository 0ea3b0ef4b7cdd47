"""Minimal DOLFINx-shaped objects for meshes that do not come from DOLFINx.

The reference's entry points read a few attributes of DOLFINx objects
(gpu_assembler.py:370-381, solvers.py:298-309, dissolve.py:785, 893-894):
domain.topology.index_map(3).size_local, domain.geometry.x, V.dofmap.cell_dofs(i),
V.dofmap.index_map.size_local, f.x.array, f.function_space.mesh and the attributes the
driver attaches to coefficient functions (_solver_inv_dt, _solver_bc_dofs).  These
classes provide exactly those for a (coords, cells) mesh with the identity dofmap.
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np


class _IndexMap:
    def __init__(self, n):
        self.size_local = int(n)


class Mesh:
    def __init__(self, coords, cells):
        self.coords = np.ascontiguousarray(coords, dtype=np.float64)
        self.cells = np.ascontiguousarray(cells, dtype=np.int32)
        n = self.cells.shape[0]
        self.topology = SimpleNamespace(dim=3, index_map=lambda d: _IndexMap(n))
        self.geometry = SimpleNamespace(x=self.coords)
        self.comm = SimpleNamespace(rank=0, size=1)


class FunctionSpace:
    def __init__(self, mesh: Mesh):
        self.mesh = mesh
        cells = mesh.cells
        self.dofmap = SimpleNamespace(index_map=_IndexMap(mesh.coords.shape[0]),
                                      cell_dofs=lambda i: cells[i], list=cells)


class _Vector:
    def __init__(self, n):
        self.array = np.zeros(n, dtype=np.float64)

    def scatter_forward(self):
        pass


class Function:
    def __init__(self, V: FunctionSpace, values=None):
        self.function_space = V
        self.x = _Vector(V.dofmap.index_map.size_local)
        if values is not None:
            self.x.array[:] = values


def mesh_from(tet_mesh) -> Mesh:
    return Mesh(tet_mesh.coords, tet_mesh.cells)
