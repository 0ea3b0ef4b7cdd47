"""Drop-in for the transport solve of the reference's numerics/solvers.py.

solve_transport(name, a_form, L_form, u, bcs=None, ksp_type="gmres", pc_type="bjacobi",
rtol=1e-8, max_it=1000, under_relax=None, comm=None, extra_petsc_opts=None, ceed_op=None,
use_gpu=False, de_field=None, alpha_field=None, u_old=None, source_field=None,
bc_value=0.0) -> {"converged", "iterations", "time_s"}     (solvers.py:206-284)

The GPU-assembled branch (_solve_gpu_asm, solvers.py:287-372) is the one this build
provides: per field name it caches a GPUSparseAssembler (sharing the geometry registered
with set_shared_geometry) and a solver with fixed b / x buffers, refills the operator and
the RHS on the GPU every call, warm-starts from u and copies the solution back into
u.x.array.  Hidden inputs ride on de_field as in the driver: _solver_inv_dt and
_solver_bc_dofs (dissolve.py:785, 893-894).

Differences, stated:
  * The Krylov method is Jacobi-preconditioned CG on the symmetric free block (Dirichlet
    rows are identity rows and the preconditioner is zero on them) run as one persistent
    cooperative kernel; ksp_type "gmres"/"cg" and pc_type "bjacobi"/"jacobi"/None are
    accepted and all run it.  The stopping rule is ||b - A x||_2 <= rtol ||b||_2 in FP64
    (PETSc's default test is relative to the preconditioned initial residual).
  * The matrix-free branch (ceed_op given, _solve_ceed, solvers.py:375-404) runs on the
    GPU as tp_mfcg_solve: Jacobi-PCG whose every product is the fused matrix-free apply
    (the operator of CeedDiffusionMassOp, never assembled).  Its right-hand side is
    assembled on the GPU from u_old (consistent mass, as the operator's) instead of from
    the UFL L_form, and it is preconditioned by the operator's diagonal (computed from the
    same geometry) where the reference's MatShell runs unpreconditioned (pc "none").
  * The DOLFINx/UFL branches without u_old (_solve_ceed with an L_form, _solve_standard)
    need DOLFINx and PETSc, which are not part of this build: they raise
    NotImplementedError instead of silently falling back to the CPU.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from dissolve_tp import _lib
from dissolve_tp.assembler import GPUSparseAssembler
from dissolve_tp.device import ptr, stream_handle, to_device
from dissolve_tp.krylov import CsrOperator, MatrixFreeCG, PersistentCG

_SHARED_GEOM = None
_GPU_ASM_CACHE: dict = {}


def set_shared_geometry(asm) -> None:
    """Register the primary GPUSparseAssembler as the shared geometry (solvers.py:44-47)."""
    global _SHARED_GEOM
    _SHARED_GEOM = asm


def _destroy_gpu_cache():
    for entry in _GPU_ASM_CACHE.values():
        sol = entry.get("solver")
        if sol is not None:
            sol.close()
    _GPU_ASM_CACHE.clear()


def _array(f):
    if f is None:
        return None
    return f.x.array if hasattr(f, "x") else f


class MatrixFreeOperator:
    """Matrix-free operator wrapper (solvers.py:172-203): y = A x through a
    CeedDiffusionMassOp, on device tensors (no host round trip per product)."""

    def __init__(self, ceed_op, ndofs: int, comm=None):
        self.ceed_op = ceed_op
        self.ndofs = ndofs
        self.comm = comm
        self.mat = self

    def mult(self, A, x, y):
        self.ceed_op.apply(x, y)


def solve_transport(name, a_form=None, L_form=None, u=None, bcs=None, ksp_type="gmres",
                    pc_type="bjacobi", rtol=1e-8, max_it=1000, under_relax=None, comm=None,
                    extra_petsc_opts=None, ceed_op=None, use_gpu=False, de_field=None,
                    alpha_field=None, u_old=None, source_field=None, bc_value=0.0) -> dict:
    t0 = time.time()
    if under_relax is not None and under_relax < 1.0 and u is not None:
        # solvers.py:246-247: the pre-solve copy of u replaces u_old (RHS and relaxation)
        ua = _array(u)
        u_old = ua.clone() if isinstance(ua, torch.Tensor) else np.array(ua, copy=True)
    if ceed_op is not None:
        if u_old is None:
            raise NotImplementedError(
                "the MatShell branch without u_old assembles its right-hand side from UFL "
                "forms (DOLFINx); pass u_old (and de_field carrying _solver_bc_dofs) to run "
                "it on the GPU")
        bc_dofs = getattr(de_field, "_solver_bc_dofs", None) if de_field is not None else None
        converged, iterations = _solve_ceed_gpu(name, ceed_op, u, rtol, max_it, u_old=u_old,
                                                source_field=source_field, bc_dofs=bc_dofs,
                                                bc_value=bc_value, under_relax=under_relax)
        if hasattr(u, "x") and hasattr(u.x, "scatter_forward"):
            u.x.scatter_forward()
        return {"converged": bool(converged), "iterations": int(iterations),
                "time_s": time.time() - t0}
    if not (use_gpu and de_field is not None and pc_type in (None, "bjacobi", "jacobi")):
        raise NotImplementedError(
            "only the GPU-assembled transport branch is part of this build "
            "(use_gpu=True, de_field given, pc_type in bjacobi/jacobi/None)")
    if u_old is None:
        raise NotImplementedError("the right-hand side is assembled from u_old on the GPU; "
                                  "the UFL L_form branch needs DOLFINx")
    converged, iterations = _solve_gpu_asm(name, de_field, u, rtol, max_it,
                                           alpha_field=alpha_field, u_old=u_old,
                                           source_field=source_field, bc_value=bc_value,
                                           under_relax=under_relax)
    if hasattr(u, "x") and hasattr(u.x, "scatter_forward"):
        u.x.scatter_forward()
    return {"converged": bool(converged), "iterations": int(iterations),
            "time_s": time.time() - t0}


def _solve_ceed_gpu(name, ceed_op, u, rtol, max_it, u_old, source_field=None, bc_dofs=None,
                    bc_value=0.0, under_relax=None):
    """The matrix-free solve (solvers.py:375-404) on the GPU: b = M (u_old/dt + f) with the
    consistent mass and Dirichlet values, then tp_mfcg_solve with the CeedDiffusionMassOp's
    coefficients, warm-started from u."""
    import ctypes

    op = getattr(ceed_op, "ceed_op", ceed_op)  # MatrixFreeOperator or the operator itself
    dm = op._dm
    if bc_dofs is not None and len(bc_dofs) == 0:
        bc_dofs = None
    key = ("ceed", name, id(op))
    cache = _GPU_ASM_CACHE.get(key)
    if cache is None or cache["solver"].max_it != int(max_it):
        cache = {"solver": MatrixFreeCG(dm, 1, 1, rtol=rtol, max_it=max_it, lumped=0,
                                        legacy=int(op.legacy))}
        _GPU_ASM_CACHE[key] = cache
    sol = cache["solver"]
    sol.rtol[:] = rtol
    d_u = to_device(_array(u_old), torch.float64, dm.device)
    d_f = to_device(_array(source_field), torch.float64, dm.device) if source_field is not None \
        else None
    d_bc = to_device(np.asarray(bc_dofs, dtype=np.int32), torch.int32, dm.device) \
        if bc_dofs is not None else None
    n_bc = 0 if d_bc is None else int(d_bc.numel())
    bcv = (ctypes.c_double * 4)(float(bc_value), 0.0, 0.0, 0.0)
    _lib.call("tp_assemble_rhs", ctypes.byref(dm.tpm), 1, 1, ptr(d_u), ptr(d_f), op.inv_dt, 0,
              n_bc, ptr(d_bc), bcv, ptr(sol.b), stream_handle())
    mask = dm.bc_mask(np.asarray(bc_dofs, dtype=np.int32)) if bc_dofs is not None else None
    u_arr = _array(u)
    sol.x.view(-1).copy_(to_device(u_arr, torch.float64, dm.device))
    res = sol.solve(op._De, op.inv_dt, alpha_cell=op.alpha, bc_mask=mask)
    x = sol.x.view(-1)
    if under_relax is not None and under_relax < 1.0:
        _lib.call("tp_axpby", x.numel(), 1.0 - float(under_relax), ptr(d_u), float(under_relax),
                  ptr(x), stream_handle())
    if isinstance(u_arr, torch.Tensor):
        u_arr.copy_(x)
    else:
        u_arr[...] = x.cpu().numpy()
    return res["converged"], res["iterations"]


def _solve_gpu_asm(name, de_field, u, rtol, max_it, alpha_field=None, u_old=None,
                   source_field=None, bc_value=0.0, under_relax=None):
    V = de_field.function_space
    domain = V.mesh
    inv_dt = float(getattr(de_field, "_solver_inv_dt", 1.0))
    bc_dofs = getattr(de_field, "_solver_bc_dofs", None)
    if bc_dofs is not None and len(bc_dofs) == 0:
        bc_dofs = None
    cache = _GPU_ASM_CACHE.get(name)
    if cache is None:
        asm = GPUSparseAssembler(domain, V, ref_asm=_SHARED_GEOM)
        cache = {"asm": asm, "bc_key": None, "solver": None}
        _GPU_ASM_CACHE[name] = cache
    asm = cache["asm"]
    asm.assemble(_array(de_field), inv_dt, alpha=_array(alpha_field), bc_dofs=bc_dofs)
    b = asm.assemble_rhs(_array(u_old), inv_dt, f=_array(source_field), bc_dofs=bc_dofs,
                         bc_value=bc_value)
    # the solver is rebuilt only when the Dirichlet set changes (its mask is baked in)
    key = None if bc_dofs is None else (len(bc_dofs), hash(np.asarray(bc_dofs).tobytes()))
    sol = cache["solver"]
    if sol is None or cache["bc_key"] != key or sol.max_it != max_it:
        if sol is not None:
            sol.close()
        mask = asm._dm.bc_mask(bc_dofs) if bc_dofs is not None else None
        op = CsrOperator(asm.d_indptr, asm.d_indices, asm.d_data, bc_mask=mask)
        sol = PersistentCG(op, rtol=rtol, max_it=max_it, inner_fp32=False)
        sol.max_it = max_it
        cache["solver"], cache["bc_key"] = sol, key
    sol.set_rtol(rtol)
    sol.refresh_values()
    sol.b.view(-1).copy_(b)
    u_arr = _array(u)
    sol.x.view(-1).copy_(to_device(u_arr, torch.float64, asm.device))
    res = sol.solve()
    x = sol.x.view(-1)
    if under_relax is not None and under_relax < 1.0:
        # u = w u_new + (1 - w) u_old (solvers.py:278-279), on the device
        prev = to_device(_array(u_old), torch.float64, asm.device)
        _lib.call("tp_axpby", x.numel(), 1.0 - float(under_relax), ptr(prev),
                  float(under_relax), ptr(x), stream_handle())
    if isinstance(u_arr, torch.Tensor):
        u_arr.copy_(x)
    else:
        u_arr[:] = x.cpu().numpy()
    return res["converged"], res["iterations"]
