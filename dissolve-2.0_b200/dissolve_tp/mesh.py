"""Synthetic P1 tetrahedral meshes: jittered Kuhn-split cubes and the gyroid level set.

The reference reads DOLFINx meshes (`domain/mesh_utils.py:200` `load_mesh`) and takes
`elem_nodes` from the P1 dofmap (`gpu/gpu_assembler.py:376-378`), with vertex
coordinates indexed by dof (`gpu_assembler.py:380`).  Here a mesh is the plain pair

    coords : float64 (n_verts, 3)
    cells  : int32   (n_cells, 4)   vertex ids, i.e. the identity dofmap

which is what `GPUSparseAssembler` accepts in place of `(domain, V)`.

Kuhn split: each cube of the N^3 grid is cut into the 6 tetrahedra that follow the
monotone lattice paths from the cube's (0,0,0) corner to its (1,1,1) corner, one per
permutation of the axes, with the same main diagonal in every cube.  Vertex id of
lattice point (i, j, k) is i + (N+1)*(j + (N+1)*k); cells are ordered cube by cube
(x fastest) and, inside a cube, by the permutation order below.  Interior vertices
are moved by independent U(-j*h, +j*h) offsets per coordinate from a seeded
numpy Generator; boundary vertices stay on the box faces.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# axis permutations, lexicographic: each gives the path 0 -> e_a -> e_a+e_b -> 1
_KUHN_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))

SEED_MESH = 0
SEED_COEFF = 1
SEED_FIELDS = 2
SEED_MLP = 3


@dataclass
class TetMesh:
    coords: np.ndarray   # (V, 3) float64
    cells: np.ndarray    # (n, 4) int32
    n_side: int = 0
    lo: float = 0.0
    hi: float = 1.0

    @property
    def n_cells(self) -> int:
        return int(self.cells.shape[0])

    @property
    def n_verts(self) -> int:
        return int(self.coords.shape[0])

    @property
    def h(self) -> float:
        return (self.hi - self.lo) / self.n_side if self.n_side else float("nan")


def kuhn_counts(n: int) -> tuple[int, int, int]:
    """(tets, vertices, nnz) of the N^3 Kuhn cube: nnz = V + 2E with
    E = 3N(N+1)^2 + 3N^2(N+1) + N^3 (axis, face-diagonal and body-diagonal edges)."""
    v = (n + 1) ** 3
    e = 3 * n * (n + 1) ** 2 + 3 * n * n * (n + 1) + n ** 3
    return 6 * n ** 3, v, v + 2 * e


def kuhn_cells(n: int) -> np.ndarray:
    """Connectivity of the N^3 Kuhn split, int32 (6 N^3, 4)."""
    s = n + 1
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    # cube order: x fastest -> transpose to (k, j, i) before ravel
    i = i.transpose(2, 1, 0).ravel()
    j = j.transpose(2, 1, 0).ravel()
    k = k.transpose(2, 1, 0).ravel()
    base = np.stack([i, j, k], axis=1)  # (n^3, 3)

    def vid(p):
        return p[:, 0] + s * (p[:, 1] + s * p[:, 2])

    out = np.empty((base.shape[0], 6, 4), dtype=np.int64)
    for t, perm in enumerate(_KUHN_PERMS):
        p = base.copy()
        out[:, t, 0] = vid(p)
        for q, ax in enumerate(perm):
            p[:, ax] += 1
            out[:, t, q + 1] = vid(p)
    return out.reshape(-1, 4).astype(np.int32)


def kuhn_cube(n: int, jitter: float = 0.0, seed: int = SEED_MESH,
              lo: float = 0.0, hi: float = 1.0) -> TetMesh:
    """Jittered Kuhn-split cube [lo, hi]^3 with n cells per side."""
    s = n + 1
    h = (hi - lo) / n
    ax = lo + h * np.arange(s, dtype=np.float64)
    z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
    coords = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    if jitter:
        rng = np.random.default_rng(seed)
        d = rng.uniform(-jitter * h, jitter * h, size=coords.shape)
        idx = np.arange(s)
        kk, jj, ii = np.meshgrid(idx, idx, idx, indexing="ij")
        interior = ((ii > 0) & (ii < n) & (jj > 0) & (jj < n) & (kk > 0) & (kk < n)).ravel()
        coords[interior] += d[interior]
    return TetMesh(coords=np.ascontiguousarray(coords), cells=kuhn_cells(n),
                   n_side=n, lo=lo, hi=hi)


def face_dofs(mesh: TetMesh, axis: int = 0, side: str = "min") -> np.ndarray:
    """Vertex ids on a box face (the x=0 Dirichlet set of the small plain-method case)."""
    c = mesh.coords[:, axis]
    tol = 1e-9 * (mesh.hi - mesh.lo)
    target = mesh.lo if side == "min" else mesh.hi
    return np.nonzero(np.abs(c - target) <= tol)[0].astype(np.int32)


def gyroid(coords: np.ndarray, shift: float = 0.3) -> np.ndarray:
    """phi = sin x cos y + sin y cos z + sin z cos x - shift (scaffold where phi > 0)."""
    x, y, z = coords[:, 0], coords[:, 1], coords[:, 2]
    return (np.sin(x) * np.cos(y) + np.sin(y) * np.cos(z) + np.sin(z) * np.cos(x) - shift)


def gyroid_cube(n: int, jitter: float, seed: int = SEED_MESH) -> tuple[TetMesh, np.ndarray]:
    m = kuhn_cube(n, jitter, seed, lo=0.0, hi=2.0 * math.pi)
    return m, gyroid(m.coords)


def concat_meshes(meshes: list[TetMesh]) -> tuple[TetMesh, np.ndarray, np.ndarray]:
    """Block-diagonal union of independent meshes.

    Returns the union mesh plus vert_ptr (M+1) and cell_ptr (M+1) offsets, int64."""
    vp = np.zeros(len(meshes) + 1, dtype=np.int64)
    cp = np.zeros(len(meshes) + 1, dtype=np.int64)
    for i, m in enumerate(meshes):
        vp[i + 1] = vp[i] + m.n_verts
        cp[i + 1] = cp[i] + m.n_cells
    coords = np.concatenate([m.coords for m in meshes], axis=0)
    cells = np.concatenate([m.cells.astype(np.int64) + vp[i] for i, m in enumerate(meshes)],
                           axis=0)
    if vp[-1] >= 2 ** 31:
        raise ValueError("union mesh exceeds int32 vertex ids")
    return TetMesh(coords=coords, cells=cells.astype(np.int32)), vp, cp
