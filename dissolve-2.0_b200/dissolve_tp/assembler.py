"""GPUSparseAssembler: drop-in for gpu/gpu_assembler.py:311-673 on the B200 kernels.

Same constructor (domain, V, comm=None, ref_asm=None), same public attributes
(n_cells, n_dofs, _nnz, d_elem_nodes, d_detJ, d_Gflat, d_JinvT, d_indptr, d_indices,
d_scatter_map, d_data, d_b, mat) and methods (assemble, assemble_rhs, nodal_gradient,
scaffold_volume, _to_cell_avg) with the reference's argument meaning and ValueError
texts.  Device arrays are torch CUDA tensors instead of CuPy arrays; `mat` is a CSR
triple with .mult instead of a PETSc aijcusparse Mat (PETSc is not part of this build).

Differences of mechanism (not of result):
  * setup runs on the GPU (tp_cell_geometry / tp_incidence / tp_pattern) instead of
    numpy + Python sets and dicts (gpu_assembler.py:376-438);
  * the reference-layout geometry arrays (d_detJ, d_Gflat, d_JinvT) and d_scatter_map are
    materialised on first access only -- the kernels read a compact 64-byte record;
  * assembly is atomics-free and deterministic (row-gather over vertex->cell lists).
"""
from __future__ import annotations

import os
import types

import numpy as np
import torch

from . import _lib
from ._lib import TpCsrOp, TpMesh, call
from .device import empty_aligned, ptr, require_cuda, stream_handle, to_device

# gpu_assembler.py:37 -- 1 (default): row-sum lumped mass, 0: consistent mass
LUMP_MASS = int(os.environ.get("DISSOLVE_LUMP_MASS", "1"))


def extract_mesh(domain, V=None):
    """(coords (V,3) f64, cells (n,4) int32) from a TetMesh, a (coords, cells) pair or
    DOLFINx-like objects (topology.index_map(3).size_local, V.dofmap.cell_dofs(i),
    geometry.x), mirroring gpu_assembler.py:370-381."""
    if hasattr(domain, "coords") and hasattr(domain, "cells"):
        return (np.ascontiguousarray(domain.coords[:, :3], dtype=np.float64),
                np.ascontiguousarray(domain.cells, dtype=np.int32))
    if isinstance(domain, (tuple, list)) and len(domain) == 2:
        c, e = domain
        return (np.ascontiguousarray(np.asarray(c)[:, :3], dtype=np.float64),
                np.ascontiguousarray(np.asarray(e), dtype=np.int32))
    tdim = domain.topology.dim
    n_cells = domain.topology.index_map(tdim).size_local
    dm = V.dofmap
    lst = getattr(dm, "list", None)
    if lst is not None and hasattr(lst, "shape"):
        elem = np.asarray(lst[:n_cells], dtype=np.int32)
    else:
        elem = np.array([dm.cell_dofs(i) for i in range(n_cells)], dtype=np.int32)
    coords = np.asarray(domain.geometry.x)[:, :3]
    return np.ascontiguousarray(coords, dtype=np.float64), np.ascontiguousarray(elem)


# rows per tile of the tiled kernels (tp_tiles_create); 0 keeps the row walk
TILE_ROWS = int(os.environ.get("DISSOLVE_TILE_ROWS", "64"))


class DeviceMesh:
    """Mesh state resident on the GPU, built by the setup kernels."""

    def __init__(self, coords: np.ndarray, cells: np.ndarray, device=None,
                 tile_rows: int | None = None):
        self.device = device or require_cuda()
        dev = self.device
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        if cells.ndim != 2 or cells.shape[1] != 4:
            raise ValueError(f"cells must have shape (n, 4), got {cells.shape}")
        self.n_cells = int(cells.shape[0])
        self.n_verts = int(coords.shape[0])
        st = stream_handle()
        self.coords = torch.from_numpy(coords).to(dev)
        self.cells = torch.from_numpy(cells).to(dev)
        self.coords4 = torch.empty((self.n_verts, 4), dtype=torch.float64, device=dev)
        self.geo = torch.empty((self.n_cells, 8), dtype=torch.float64, device=dev)
        self.flags = torch.zeros(4, dtype=torch.int32, device=dev)
        call("tp_cell_geometry", self.n_cells, self.n_verts, ptr(self.cells), ptr(self.coords),
             ptr(self.coords4), ptr(self.geo), None, None, None, ptr(self.flags), st)
        scratch_bytes = _lib.lib.tp_setup_scratch_bytes(self.n_cells, self.n_verts)
        self.scratch = torch.empty(int(scratch_bytes), dtype=torch.uint8, device=dev)
        self.v2c_ptr = torch.empty(self.n_verts + 1, dtype=torch.int32, device=dev)
        self.v2c = torch.empty(max(4 * self.n_cells, 1), dtype=torch.int32, device=dev)
        md = _lib._c_i32(0)
        call("tp_incidence", self.n_cells, self.n_verts, ptr(self.cells), ptr(self.v2c_ptr),
             ptr(self.v2c), ptr(self.scratch), _lib.ctypes.byref(md), st)
        self.max_degree = int(md.value)
        self.indptr = torch.empty(self.n_verts + 1, dtype=torch.int32, device=dev)
        nnz = _lib._c_i64(0)
        mrl = _lib._c_i32(0)
        call("tp_pattern", self.n_cells, self.n_verts, ptr(self.cells), ptr(self.v2c_ptr),
             ptr(self.v2c), self.max_degree, ptr(self.indptr), None, ptr(self.scratch),
             _lib.ctypes.byref(nnz), _lib.ctypes.byref(mrl), st)
        self.nnz = int(nnz.value)
        self.max_row_len = int(mrl.value)
        self.indices = torch.empty(max(self.nnz, 1), dtype=torch.int32, device=dev)
        call("tp_pattern", self.n_cells, self.n_verts, ptr(self.cells), ptr(self.v2c_ptr),
             ptr(self.v2c), self.max_degree, ptr(self.indptr), ptr(self.indices),
             ptr(self.scratch), None, None, st)
        self.slots = torch.empty(max(4 * self.n_cells, 1), dtype=torch.int32, device=dev)
        self.tpm = self._struct()
        call("tp_incidence_slots", _lib.ctypes.byref(self.tpm), ptr(self.slots), ptr(self.flags), st)
        self._tiles = None
        self.tile_rows = TILE_ROWS if tile_rows is None else int(tile_rows)
        self.tpm = self._struct()
        if self.tile_rows > 0 and self.n_verts > 0:
            self.set_tiles(self.tile_rows)
        self._ref_geom = None
        self._scatter_map = None

    def set_tiles(self, rows_per_tile: int):
        """Row tiles for the tiled kernels (0: none, the kernels walk rows); same results."""
        self._free_tiles()
        self.tile_rows = int(rows_per_tile)
        if self.tile_rows > 0:
            h = _lib.ctypes.c_void_p()
            call("tp_tiles_create", _lib.ctypes.byref(self.tpm), self.tile_rows, stream_handle(),
                 _lib.ctypes.byref(h))
            self._tiles = h
        self.tpm = self._struct()

    def tiles_info(self) -> dict:
        if self._tiles is None:
            return {}
        c = _lib.ctypes
        nt, r, mc = _lib._c_i32(0), _lib._c_i32(0), _lib._c_i32(0)
        ne, nb = _lib._c_i64(0), c.c_size_t(0)
        call("tp_tiles_info", self._tiles, c.byref(nt), c.byref(r), c.byref(mc), c.byref(ne),
             c.byref(nb))
        return {"n_tiles": nt.value, "rows_per_tile": r.value, "max_cells": mc.value,
                "entries": ne.value, "bytes": nb.value}

    def _free_tiles(self):
        if getattr(self, "_tiles", None) is not None:
            _lib.lib.tp_tiles_destroy(self._tiles)
            self._tiles = None

    def __del__(self):
        try:
            self._free_tiles()
        except Exception:
            pass

    def _struct(self) -> TpMesh:
        return TpMesh(self.n_cells, self.n_verts, getattr(self, "nnz", 0),
                      getattr(self, "max_row_len", 0), getattr(self, "max_degree", 0),
                      ptr(self.cells), ptr(self.coords4), ptr(self.geo),
                      ptr(self.v2c_ptr), ptr(self.v2c),
                      ptr(getattr(self, "slots", None)), ptr(self.indptr),
                      ptr(getattr(self, "indices", None)),
                      getattr(getattr(self, "_tiles", None), "value", None))

    @property
    def ref_geometry(self):
        """(detJ (n,), Gflat (9n,), JinvT (9n,)) in the reference layout, computed once."""
        if self._ref_geom is None:
            dev = self.device
            detJ = torch.empty(self.n_cells, dtype=torch.float64, device=dev)
            G = torch.empty(9 * self.n_cells, dtype=torch.float64, device=dev)
            JT = torch.empty(9 * self.n_cells, dtype=torch.float64, device=dev)
            geo = torch.empty_like(self.geo)
            call("tp_cell_geometry", self.n_cells, self.n_verts, ptr(self.cells), ptr(self.coords),
                 None, ptr(geo), ptr(detJ), ptr(G), ptr(JT), ptr(self.flags), stream_handle())
            self._ref_geom = (detJ, G, JT)
        return self._ref_geom

    def use_reference_geometry(self, detJ, Gflat):
        """Replace the compact geometry by one packed from given reference-layout arrays."""
        d = to_device(detJ, torch.float64, self.device)
        g = to_device(Gflat, torch.float64, self.device).reshape(-1)
        call("tp_pack_geometry", self.n_cells, ptr(d), ptr(g), ptr(self.geo), stream_handle())

    @property
    def scatter_map(self):
        if self._scatter_map is None:
            sm = torch.empty(max(16 * self.n_cells, 4), dtype=torch.int32, device=self.device)
            call("tp_scatter_map", self.n_cells, ptr(self.cells), ptr(self.indptr),
                 ptr(self.indices), ptr(sm), stream_handle())
            self._scatter_map = sm[: 16 * self.n_cells]
        return self._scatter_map

    def bc_mask(self, bc_dofs) -> torch.Tensor:
        """uint8 mask of Dirichlet dofs (validated on the device)."""
        mask = torch.empty(self.n_verts, dtype=torch.uint8, device=self.device)
        d = to_device(bc_dofs, torch.int32, self.device) if bc_dofs is not None else None
        n = 0 if d is None else int(d.numel())
        call("tp_bc_mask", n, ptr(d) if n else None, self.n_verts, ptr(mask), ptr(self.flags),
             stream_handle())
        return mask


class CsrMatrix:
    """The assembled operator in the PETSc-compatible CSR layout of
    gpu_assembler.py:440-450 (rows in order, sorted columns), FP64 values on the device."""

    def __init__(self, indptr, indices, data, n):
        self.indptr, self.indices, self.data, self.n = indptr, indices, data, n

    def getSize(self):
        return (self.n, self.n)

    def createVecLeft(self):
        return torch.zeros(self.n, dtype=torch.float64, device=self.data.device)

    createVecRight = createVecLeft

    def getValuesCSR(self):
        return (self.indptr.cpu().numpy(), self.indices.cpu().numpy(), self.data.cpu().numpy())

    def mult(self, x, y=None):
        x = to_device(x, torch.float64, self.data.device)
        if y is None:
            y = torch.empty_like(x)
        op = TpCsrOp()
        op.n_rows = self.n
        op.S = 1
        op.ld = 1
        op.indptr, op.indices, op.K64 = ptr(self.indptr), ptr(self.indices), ptr(self.data)
        op.dscale[0] = 1.0
        op.n_systems = 1
        call("tp_csr_apply", _lib.ctypes.byref(op), 0, ptr(x), ptr(y), stream_handle())
        return y

    def to_scipy(self):
        import scipy.sparse as sp

        ip, ix, d = self.getValuesCSR()
        return sp.csr_matrix((d, ix, ip), shape=(self.n, self.n))


class GPUSparseAssembler:
    """P1 (1/dt + alpha) M + De K assembler on the GPU (gpu_assembler.py:311)."""

    def __init__(self, domain=None, V=None, comm=None, ref_asm=None, *, tile_rows=None):
        """tile_rows (keyword, not in the reference's signature): rows per tile of the
        tiled kernels (None: the default, 0: none)."""
        self.comm = comm
        if ref_asm is not None:
            # shared read-only geometry and pattern (gpu_assembler.py:346-367)
            self._dm = ref_asm._dm
        else:
            coords, cells = extract_mesh(domain, V)
            self._dm = DeviceMesh(coords, cells, tile_rows=tile_rows)
        dm = self._dm
        self.n_cells = dm.n_cells
        self.n_dofs = dm.n_verts
        self._nnz = dm.nnz
        self.device = dm.device
        self.d_elem_nodes = dm.cells.reshape(-1)
        self.d_indptr = dm.indptr
        self.d_indices = dm.indices[: self._nnz]
        self.d_data = torch.zeros(self._nnz, dtype=torch.float64, device=self.device)
        self.d_b = torch.zeros(self.n_dofs, dtype=torch.float64, device=self.device)
        self.mat = CsrMatrix(self.d_indptr, self.d_indices, self.d_data, self.n_dofs)
        self._zero_cells = None
        self._vol = torch.zeros(1, dtype=torch.float64, device=self.device)

    # reference-layout arrays, materialised on first use
    @property
    def d_detJ(self):
        return self._dm.ref_geometry[0]

    @property
    def d_Gflat(self):
        return self._dm.ref_geometry[1]

    @property
    def d_JinvT(self):
        return self._dm.ref_geometry[2]

    @property
    def d_scatter_map(self):
        return self._dm.scatter_map

    @property
    def _grad_buf(self):
        return torch.zeros(3 * self.n_dofs, dtype=torch.float64, device=self.device)

    @property
    def _wsum_buf(self):
        return torch.zeros(self.n_dofs, dtype=torch.float64, device=self.device)

    def _to_cell_avg(self, arr_or_func):
        """gpu_assembler.py:452-470."""
        if arr_or_func is None:
            return torch.zeros(self.n_cells, dtype=torch.float64, device=self.device)
        n = int(arr_or_func.shape[0])
        if n == self.n_cells:
            return to_device(arr_or_func, torch.float64, self.device)
        if n == self.n_dofs:
            d = to_device(arr_or_func, torch.float64, self.device)
            out = torch.empty(self.n_cells, dtype=torch.float64, device=self.device)
            call("tp_cell_average", self.n_cells, ptr(self._dm.cells), ptr(d), ptr(out),
                 stream_handle())
            return out
        raise ValueError(
            f"array length {n} matches neither n_cells={self.n_cells} "
            f"nor n_dofs={self.n_dofs}"
        )

    def assemble(self, De, inv_dt: float, alpha=None, bc_dofs=None):
        """(1/dt + alpha_e) M_e + De_e K_e into self.mat, Dirichlet rows when bc_dofs is
        given (gpu_assembler.py:472-532)."""
        d_De = self._to_cell_avg(De)
        d_alpha = self._to_cell_avg(alpha) if alpha is not None else None
        mask = None
        if bc_dofs is not None and len(bc_dofs) > 0:
            mask = self._dm.bc_mask(bc_dofs)
        call("tp_assemble_csr", _lib.ctypes.byref(self._dm.tpm), ptr(d_De), ptr(d_alpha),
             float(inv_dt), int(LUMP_MASS), _lib.TP_ASM_FULL, ptr(mask), ptr(self.d_data), None,
             stream_handle())

    def assemble_rhs(self, u_old, inv_dt: float, f=None, bc_dofs=None, bc_value: float = 0.0):
        """b = M u_old / dt + M f, then b[bc_dofs] = bc_value (gpu_assembler.py:534-603)."""
        if u_old.shape[0] != self.n_dofs:
            raise ValueError(f"u_old length {u_old.shape[0]} != n_dofs {self.n_dofs}")
        d_u = to_device(u_old, torch.float64, self.device)
        if f is None:
            d_f = None
        elif int(f.shape[0]) == self.n_dofs:
            d_f = to_device(f, torch.float64, self.device)
        elif int(f.shape[0]) == self.n_cells:
            d_f = self._cell_to_vertex_lossy(f)
        else:
            raise ValueError(f"f length {f.shape[0]} unrecognised")
        d_bc = None
        n_bc = 0
        if bc_dofs is not None and len(bc_dofs) > 0:
            self._dm.bc_mask(bc_dofs)  # validates the dof ids on the device
            d_bc = to_device(bc_dofs, torch.int32, self.device)
            n_bc = int(d_bc.numel())
        val = (_lib._c_dbl * 1)(float(bc_value))
        call("tp_assemble_rhs", _lib.ctypes.byref(self._dm.tpm), 1, 1, ptr(d_u), ptr(d_f),
             float(inv_dt), int(LUMP_MASS), n_bc, ptr(d_bc), val, ptr(self.d_b), stream_handle())
        return self.d_b

    def _cell_to_vertex_lossy(self, f_cell):
        """gpu_assembler.py:560-571: per-cell f taken at index searchsorted(elem_nodes, dof)
        of the flat connectivity, wrapped modulo n_cells as CuPy fancy indexing does.
        The search is a plain lower-bound binary search on the (unsorted) flat array."""
        flat = self._dm.cells.reshape(-1).to(torch.int64)
        n = flat.numel()
        keys = torch.arange(self.n_dofs, device=self.device, dtype=torch.int64)
        lo = torch.zeros_like(keys)
        hi = torch.full_like(keys, n)
        for _ in range(int(np.ceil(np.log2(max(n, 2)))) + 1):
            active = lo < hi
            mid = torch.where(active, lo + (hi - lo) // 2, lo)
            less = flat[mid.clamp(max=n - 1)] < keys
            lo = torch.where(active & less, mid + 1, lo)
            hi = torch.where(active & ~less, mid, hi)
        idx = lo % self.n_cells
        return to_device(f_cell, torch.float64, self.device)[idx].contiguous()

    def scaffold_volume(self, phi_arr, epsilon: float):
        """Integral of H_eps(phi) (gpu_assembler.py:605-644), a Python float."""
        d = to_device(phi_arr, torch.float64, self.device)
        call("tp_scaffold_volume", _lib.ctypes.byref(self._dm.tpm), ptr(d), float(epsilon),
             ptr(self._vol), ptr(self._dm.scratch), stream_handle())
        return float(self._vol.item())

    def nodal_gradient(self, u_vert):
        """Volume-weighted vertex gradient, (n_dofs, 3) (gpu_assembler.py:646-673)."""
        if hasattr(u_vert, "x"):
            u_vert = u_vert.x.array
        d = to_device(u_vert, torch.float64, self.device)
        g = torch.empty((self.n_dofs, 3), dtype=torch.float64, device=self.device)
        call("tp_nodal_gradient", _lib.ctypes.byref(self._dm.tpm), None, ptr(d), ptr(g),
             stream_handle())
        return g
