"""Many independent meshes, one species each, stepped together.

The meshes form one block-diagonal system (`mesh.concat_meshes`): one assembly launch
over the union mesh (per-cell De and alpha carry each mesh's D and k), one right-hand-side
launch, and one solve of every mesh as its own lane (`tp_cg_*` with n_systems = number
of meshes: per-mesh dot products, convergence and iteration counts) run as a single CUDA
graph with a device-side while loop.  Launch shape (threads per row, block, rows per
reduction tile) comes from the project autotuner.  `MeshBatchPlain` is the comparison:
the plain FP64 form, one mesh at a time.

The reference solves one field on one mesh per call (numerics/solvers.py:206-284); this
batching is the multi-mesh form of that call.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import call
from .assembler import GPUSparseAssembler
from .autotune import tune_cg, tune_tiles
from .device import ptr, stream_handle, to_device
from .krylov import CGSolver, CsrOperator, PersistentCG
from .mesh import concat_meshes, kuhn_cube


def uneven_batch_inputs(n_meshes: int = 256, n_min: int = 8, n_max: int = 40,
                        jitter: float = 0.2, seed: int = 0):
    """Cube meshes with N ~ U{n_min..n_max} cells per side (each with its own seeded
    jitter), D ~ LogUniform(0.1, 10), k ~ U(0, 1); returns (meshes, D, k)."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(n_min, n_max + 1, n_meshes)
    D = np.exp(rng.uniform(np.log(0.1), np.log(10.0), n_meshes))
    k = rng.uniform(0.0, 1.0, n_meshes)
    meshes = [kuhn_cube(int(n), jitter, seed=1000 + i) for i, n in enumerate(sizes)]
    return meshes, D, k


def lpt_partition(weights, n_parts: int) -> list[list[int]]:
    """Greedy longest-processing-time partition: items in decreasing weight, each to the
    currently lightest part (ties: lowest part index).  Deterministic."""
    w = np.asarray(weights, dtype=np.float64)
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    parts: list[list[int]] = [[] for _ in range(n_parts)]
    load = np.zeros(n_parts)
    for i in order:
        p = int(np.argmin(load))
        parts[p].append(i)
        load[p] += w[i]
    return [sorted(p) for p in parts]


class MeshBatch:
    """All meshes in one assembly, one RHS and one multi-system solve per step."""

    def __init__(self, meshes, D, k, dt, rtol=1e-8, max_it=5000, inner_fp32=True,
                 autotune=True, cg=None):
        self.n_meshes = len(meshes)
        self.inv_dt = 1.0 / float(dt)
        # the assembly's rows per tile, tuned on the largest mesh before the union is built
        asm_tiles = self.tune_assembly(meshes) if autotune else None
        union, vp, cp = concat_meshes(meshes)
        self.vert_ptr, self.cell_ptr = vp, cp
        self.asm = GPUSparseAssembler(union, tile_rows=asm_tiles)
        dm = self.asm._dm
        self.dm = dm
        dev = dm.device
        self.device = dev
        ncell = np.diff(cp)
        self.De = to_device(np.repeat(np.asarray(D, dtype=np.float64), ncell), torch.float64, dev)
        self.alpha = to_device(np.repeat(np.asarray(k, dtype=np.float64), ncell), torch.float64,
                               dev)
        self.K64 = torch.zeros(dm.nnz, dtype=torch.float64, device=dev)
        self.K32 = torch.zeros(dm.nnz, dtype=torch.float32, device=dev) if inner_fp32 else None
        self.op = CsrOperator(dm.indptr, dm.indices[: dm.nnz], self.K64, K32=self.K32,
                              n_systems=self.n_meshes, sys_row_ptr=vp)
        cg = dict(cg or {})
        if autotune and not {"group", "block", "rows_per_tile"} & set(cg):
            self.assemble_operator()
            cg.update(tune_cg(self.op, inner_fp32=inner_fp32))
        self.cg_config = dict(cg, engine="graph", n_systems=self.n_meshes)
        if asm_tiles is not None:
            self.cg_config["assembly_rows_per_tile"] = asm_tiles
        self.solver = CGSolver(self.op, rtol=rtol, max_it=max_it, inner_fp32=inner_fp32, **cg)
        self.U = torch.zeros(dm.n_verts, dtype=torch.float64, device=dev)

    @property
    def n_cells(self) -> int:
        return self.dm.n_cells

    def tune_assembly(self, meshes) -> int:
        """Rows per tile of the batch's assembly, chosen by the project autotuner
        (autotune.tune_tiles) on the batch's largest mesh: the union of hundreds of
        meshes would need its tile tables rebuilt for every candidate."""
        from .assembler import DeviceMesh
        big = max(meshes, key=lambda m_: m_.n_cells)
        sample = DeviceMesh(big.coords, big.cells, tile_rows=0)
        dev = sample.device
        De = torch.ones(sample.n_cells, dtype=torch.float64, device=dev)
        out = torch.empty(sample.nnz, dtype=torch.float64, device=dev)
        out32 = torch.empty(sample.nnz, dtype=torch.float32, device=dev)

        def run():
            call("tp_assemble_csr", ctypes.byref(sample.tpm), ptr(De), ptr(De), self.inv_dt, 1,
                 _lib.TP_ASM_FULL, None, ptr(out), ptr(out32), stream_handle())

        best = tune_tiles(sample, run, key=(big.n_verts, big.n_cells, sample.nnz))
        del sample
        return best["rows_per_tile"]

    def assemble_operator(self):
        call("tp_assemble_csr", ctypes.byref(self.dm.tpm), ptr(self.De), ptr(self.alpha),
             self.inv_dt, 1, _lib.TP_ASM_FULL, None, ptr(self.K64), ptr(self.K32),
             stream_handle())

    def set_state(self, u):
        self.U.copy_(to_device(u, torch.float64, self.device).reshape(-1))

    def state(self) -> np.ndarray:
        return self.U.cpu().numpy()

    def step(self, sync=True):
        st = stream_handle()
        self.assemble_operator()
        call("tp_assemble_rhs", ctypes.byref(self.dm.tpm), 1, 1, ptr(self.U), None,
             self.inv_dt, 1, 0, None, None, ptr(self.solver.b), st)
        self.solver.x.view(-1).copy_(self.U)
        self.solver.run()
        self.U.copy_(self.solver.x.view(-1))
        return self.solver.result() if sync else None

    def launches_per_step(self) -> int:
        """Kernels of one step: assembly, RHS, the solve graph's launches are counted by
        the solve itself; here the two setup launches plus one graph launch."""
        return 3


class MeshBatchPlain:
    """The plain FP64 form one mesh at a time: per mesh FP64 assembly + RHS + FP64
    Jacobi-PCG (persistent engine)."""

    def __init__(self, meshes, D, k, dt, rtol=1e-8, max_it=5000):
        self.inv_dt = 1.0 / float(dt)
        self.items = []
        for m, d, kk in zip(meshes, D, k):
            asm = GPUSparseAssembler(m)
            dev = asm.device
            De = torch.full((asm.n_cells,), float(d), dtype=torch.float64, device=dev)
            al = torch.full((asm.n_cells,), float(kk), dtype=torch.float64, device=dev)
            op = CsrOperator(asm.d_indptr, asm.d_indices, asm.d_data)
            sol = PersistentCG(op, rtol=rtol, max_it=max_it)
            u = torch.zeros(asm.n_dofs, dtype=torch.float64, device=dev)
            self.items.append((asm, De, al, sol, u))

    def set_state(self, u, vert_ptr):
        u = np.asarray(u)
        for i, it in enumerate(self.items):
            it[4].copy_(torch.from_numpy(np.ascontiguousarray(u[vert_ptr[i]:vert_ptr[i + 1]])))

    def state(self) -> np.ndarray:
        return np.concatenate([it[4].cpu().numpy() for it in self.items])

    def step(self, sync=True):
        for asm, De, al, sol, u in self.items:
            asm.assemble(De, self.inv_dt, alpha=al)
            b = asm.assemble_rhs(u, self.inv_dt)
            sol.b.view(-1).copy_(b)
            sol.x.view(-1).copy_(u)
            sol.refresh_values()
            sol.run()
            u.copy_(sol.x.view(-1))
        return [it[3].result() for it in self.items] if sync else None
