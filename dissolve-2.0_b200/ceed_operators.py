"""Drop-in for the reference's gpu/ceed_operators.py (libCEED matrix-free operator).

Same names and call signatures: libceed_available, make_ceed, extract_ceed_mesh_data,
compute_geometric_factors, build_elem_restriction, build_simplex_basis and
CeedDiffusionMassOp(ceed, mesh_data, De_vals, inv_dt, num_comp=1) with .apply(u, out)
and .update_coeffs(De_vals, inv_dt).  libCEED is replaced by the fused matrix-free kernel
tp_matfree_apply, which recomputes each cell's P1 gradients from the vertex coordinates
in FP64 (no stored quadrature-point geometry).

Semantics.  The operator is a(u, v) = (inv_dt u, v) + (De grad u, grad v) with De the
mean of the vertex values on each cell (ceed_operators.py:330-339) and the consistent P1
mass (the reference's degree-2 quadrature integrates it exactly).  The reference
QFunction (ceed_operators.py:100-104) omits wdetJ from the stiffness term, so its
stiffness is 4 De G instead of |detJ|/6 De G; legacy_stiffness=True reproduces that
exactly, the default is the intended operator.  Optional `alpha` adds a reaction term
(alpha M) that the reference operator does not have.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from dissolve_tp import _lib
from dissolve_tp.assembler import DeviceMesh, extract_mesh
from dissolve_tp.device import ptr, require_cuda, stream_handle, to_device

# 4-point degree-2 rule on the reference tetrahedron (barycentric (a, b, b, b) and
# permutations, weight 1/24 each).  The reference takes its rule from basix
# (ceed_operators.py:145), whose point order may differ.
_QA = (5.0 + 3.0 * 5.0 ** 0.5) / 20.0
_QB = (5.0 - 5.0 ** 0.5) / 20.0
Q_PTS = np.array([[_QB, _QB, _QB], [_QA, _QB, _QB], [_QB, _QA, _QB], [_QB, _QB, _QA]])
Q_WTS = np.full(4, 1.0 / 24.0)


def libceed_available():
    """The matrix-free backend of this build is always present (ceed_operators.py:40)."""
    return True


class Ceed:
    """Device context standing in for a libCEED Ceed object."""

    def __init__(self, device):
        self.device = device
        self.resource = f"/gpu/cuda/{device}"


def make_ceed(use_gpu: bool = True):
    """(ceed, backend_name) as in ceed_operators.py:44-61; GPU only (no CPU backend)."""
    if not use_gpu:
        raise RuntimeError("the matrix-free operator of this build runs on the GPU only")
    dev = require_cuda()
    return Ceed(dev), "B200"


def extract_ceed_mesh_data(domain, V=None):
    """ceed_operators.py:125-156: elem_nodes, coords, counts and the quadrature rule."""
    coords, cells = extract_mesh(domain, V)
    return {"elem_nodes": cells, "coords": coords, "num_cells": int(cells.shape[0]),
            "num_dofs": int(coords.shape[0]), "num_qpts": 4, "q_pts": Q_PTS.copy(),
            "q_wts": Q_WTS.copy()}


def compute_geometric_factors(coords, elem_nodes, q_wts):
    """ceed_operators.py:159-199 layout: per cell and quadrature point
    [w_q |detJ|, G (row-major 9)], computed on the GPU and returned as numpy."""
    dm = DeviceMesh(np.asarray(coords)[:, :3], np.asarray(elem_nodes))
    detJ, G, _ = (t.cpu().numpy() for t in dm.ref_geometry)
    nc, nq = detJ.shape[0], len(q_wts)
    geom = np.zeros((nc, nq, 10))
    for q in range(nq):
        geom[:, q, 0] = q_wts[q] * detJ
        geom[:, q, 1:10] = G.reshape(nc, 9)
    return geom.reshape(-1)


def build_elem_restriction(ceed, elem_nodes, num_dofs, num_comp=1):
    """The element -> dof map (libCEED ElemRestriction, ceed_operators.py:202-209)."""
    e = np.asarray(elem_nodes, dtype=np.int32)
    return {"num_elem": e.shape[0], "elem_size": e.shape[1], "num_comp": num_comp,
            "l_size": num_dofs * num_comp, "offsets": e.reshape(-1).copy()}


def build_simplex_basis(ceed, num_comp=1):
    """P1 basis tabulated at the quadrature points (ceed_operators.py:212-242):
    interp (nq, 4) barycentric values, grad (3, nq, 4) reference gradients."""
    lam = np.column_stack([1.0 - Q_PTS.sum(1), Q_PTS])
    grad = np.zeros((3, 4, 4))
    ref = np.array([[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    for d in range(3):
        grad[d, :, :] = ref[:, d][None, :]
    return {"interp": lam, "grad": grad, "q_pts": Q_PTS.copy(), "q_wts": Q_WTS.copy(),
            "num_comp": num_comp}, 4


class CeedDiffusionMassOp:
    """Matrix-free a(u, v) = (u/dt, v) + De (grad u, grad v) (ceed_operators.py:247-353)."""

    def __init__(self, ceed, mesh_data, De_vals, inv_dt, num_comp=1, *, alpha=None,
                 legacy_stiffness=False):
        if num_comp != 1:
            raise ValueError("num_comp must be 1 (scalar transport fields)")
        self.ceed = ceed if ceed is not None else make_ceed(True)[0]
        self.mesh_data = mesh_data
        self.num_comp = num_comp
        self.legacy = bool(legacy_stiffness)
        self._dm = DeviceMesh(np.asarray(mesh_data["coords"])[:, :3],
                              np.asarray(mesh_data["elem_nodes"]))
        self.alpha = None
        if alpha is not None:
            self.alpha = self._cell_avg(alpha)
        self.update_coeffs(De_vals, inv_dt)

    def _cell_avg(self, vals):
        dm = self._dm
        v = to_device(vals, torch.float64, dm.device)
        if v.numel() == dm.n_cells:
            return v
        out = torch.empty(dm.n_cells, dtype=torch.float64, device=dm.device)
        _lib.call("tp_cell_average", dm.n_cells, ptr(dm.cells), ptr(v), ptr(out), stream_handle())
        return out

    def update_coeffs(self, De_vals, inv_dt):
        """Refresh De (per-vertex values averaged per cell) and 1/dt (ceed_operators.py:345)."""
        self.De_vals = De_vals
        self.inv_dt = float(inv_dt)
        self._De = self._cell_avg(De_vals)

    def apply(self, u_vec, out_vec=None):
        """out = A u.  Device tensors are used in place; numpy in, numpy out."""
        dm = self._dm
        host = not isinstance(u_vec, torch.Tensor) or not u_vec.is_cuda
        u = to_device(u_vec, torch.float64, dm.device).reshape(-1)
        y = torch.empty_like(u)
        _lib.call("tp_matfree_apply", ctypes.byref(dm.tpm), 1, 1, 0, ptr(self._De), ptr(self.alpha),
                  None, None, self.inv_dt, 0, int(self.legacy), ptr(u), ptr(y), stream_handle())
        if out_vec is None:
            return y.cpu().numpy() if host else y
        if isinstance(out_vec, torch.Tensor):
            out_vec.copy_(y.reshape(out_vec.shape))
        else:
            out_vec[...] = y.cpu().numpy().reshape(np.shape(out_vec))
        return out_vec
