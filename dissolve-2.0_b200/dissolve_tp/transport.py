"""Backward-Euler reaction-diffusion step for several species on one mesh.

Per species s the step solves  [(1/dt + k_s + alpha_s) M + D_s K_xi] u^{n+1} = M (u^n/dt + f_s)
(physics/weak_forms.py:85-143; dissolve.py:780-954 calls solve_transport once per
species), with K_xi the stiffness of the per-cell diffusivity factor shared by all
species (De_s = D_s * coef_cell) and M the lumped (default, gpu_assembler.py:37) mass.

Two forms:

  PlainTransport     the reference's flow, one species at a time: full FP64 assembly of
                     each species' matrix into CSR (GPUSparseAssembler.assemble), FP64
                     RHS, FP64 Jacobi-PCG from the previous step -- the plain FP64 form.
  BatchedTransport   all species in one solve: the shared stiffness is assembled once
                     per step (FP64 and FP32 values), the mass/reaction terms become a
                     per-column diagonal, the RHS is one interleaved (V, 4) array and one
                     CG runs every species as a lane -- FP64, or FP32 inner iterations
                     with FP64 reliable updates.  The initial guess is the previous step
                     or a learned prediction (dissolve_tp.mlp).
"""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import _lib
from ._lib import call
from .assembler import GPUSparseAssembler
from .autotune import tune_cg
from .device import ptr, stream_handle, to_device
from .krylov import CGSolver, CsrOperator, PersistentCG


class PlainTransport:
    """The plain FP64 GPU form: per species assemble + RHS + FP64 Jacobi-PCG."""

    def __init__(self, mesh, coef_cell, D, k, dt, rtol=1e-8, max_it=5000, lumped=True,
                 bc=None, cg=None, engine="persistent"):
        from . import assembler as A

        self.S = len(D)
        self.D, self.k, self.dt = list(D), list(k), float(dt)
        self.inv_dt = 1.0 / self.dt
        self._lumped_prev = A.LUMP_MASS
        self.lumped = bool(lumped)
        self.asm = [GPUSparseAssembler(mesh)]
        for _ in range(1, self.S):
            self.asm.append(GPUSparseAssembler(ref_asm=self.asm[0]))
        dev = self.asm[0].device
        self.device = dev
        nc = self.asm[0].n_cells
        self.coef = to_device(coef_cell, torch.float64, dev)
        self.De = [self.coef * float(d) for d in self.D]
        self.alpha = [torch.full((nc,), float(kk), dtype=torch.float64, device=dev)
                      for kk in self.k]
        self.bc = bc or [None] * self.S
        cg = cg or {}
        self.solvers = []
        for s in range(self.S):
            mask = self.asm[0]._dm.bc_mask(self.bc[s][0]) if self.bc[s] is not None else None
            op = CsrOperator(self.asm[s].d_indptr, self.asm[s].d_indices, self.asm[s].d_data,
                             bc_mask=mask)
            if engine == "persistent":
                self.solvers.append(PersistentCG(op, rtol=rtol, max_it=max_it,
                                                 sell=self.solvers[0].sell if s else None))
            else:
                self.solvers.append(CGSolver(op, rtol=rtol, max_it=max_it, **cg))
        self.engine = engine
        nv = self.asm[0].n_dofs
        self.U = [torch.zeros(nv, dtype=torch.float64, device=dev) for _ in range(self.S)]

    def set_state(self, U):
        U = np.asarray(U) if not isinstance(U, torch.Tensor) else U.cpu().numpy()
        for s in range(self.S):
            self.U[s].copy_(torch.from_numpy(np.ascontiguousarray(U[:, s], dtype=np.float64)))

    def state(self) -> np.ndarray:
        return np.stack([u.cpu().numpy() for u in self.U], axis=1)

    def step(self, sync=True):
        from . import assembler as A

        A.LUMP_MASS = 1 if self.lumped else 0
        try:
            for s in range(self.S):
                asm, sol = self.asm[s], self.solvers[s]
                bc = self.bc[s]
                asm.assemble(self.De[s], self.inv_dt, alpha=self.alpha[s],
                             bc_dofs=None if bc is None else bc[0])
                b = asm.assemble_rhs(self.U[s], self.inv_dt,
                                     bc_dofs=None if bc is None else bc[0],
                                     bc_value=0.0 if bc is None else bc[1])
                sol.b.view(-1).copy_(b)
                sol.x.view(-1).copy_(self.U[s])
                if self.engine == "persistent":
                    sol.refresh_values()
                sol.run()
                self.U[s].copy_(sol.x.view(-1))
        finally:
            A.LUMP_MASS = self._lumped_prev
        if not sync:
            return None
        return [sol.result() for sol in self.solvers]

    def step_host(self, u_host: torch.Tensor, out_host: torch.Tensor):
        """End-to-end step through host buffers: (S, V) float64 pinned in -> out."""
        for s in range(self.S):
            self.U[s].copy_(u_host[s], non_blocking=True)
        self.step(sync=False)
        for s in range(self.S):
            out_host[s].copy_(self.U[s], non_blocking=True)


class BatchedTransport:
    """All species in one multi-column solve (shared stiffness, per-column diagonal)."""

    def __init__(self, mesh, coef_cell, D, k, dt, rtol=1e-8, max_it=5000, lumped=True,
                 inner_fp32=True, delta=0.001, guess="previous", bc_dofs=None, bc_values=None,
                 alpha_cells=None, autotune=True, cg=None, asm=None, engine="persistent"):
        if not lumped:
            raise ValueError("the batched form splits the operator into a shared stiffness "
                             "and a per-column lumped diagonal; use PlainTransport for "
                             "consistent mass")
        self.S = len(D)
        if not 1 <= self.S <= 4:
            raise ValueError("1 to 4 species per batched solve")
        self.ld = {1: 1, 2: 2, 3: 4, 4: 4}[self.S]
        self.D, self.k, self.dt = list(D), list(k), float(dt)
        self.inv_dt = 1.0 / self.dt
        self.asm = asm if asm is not None else GPUSparseAssembler(mesh)
        dm = self.asm._dm
        self.dm = dm
        dev = self.asm.device
        self.device = dev
        n, nnz = dm.n_verts, dm.nnz
        self.coef = to_device(coef_cell, torch.float64, dev)
        self.K64 = torch.empty(nnz, dtype=torch.float64, device=dev)
        self.K32 = torch.empty(nnz, dtype=torch.float32, device=dev) if inner_fp32 else None
        self.D64 = torch.empty((n, self.ld), dtype=torch.float64, device=dev)
        self.D32 = (torch.empty((n, self.ld), dtype=torch.float32, device=dev)
                    if inner_fp32 else None)
        self.alpha = None
        if alpha_cells is not None:
            self.alpha = torch.zeros((dm.n_cells, self.ld), dtype=torch.float64, device=dev)
            self.alpha[:, : self.S] = to_device(alpha_cells, torch.float64, dev)
        self.bc_mask = dm.bc_mask(bc_dofs) if bc_dofs is not None else None
        self.bc_dofs = to_device(bc_dofs, torch.int32, dev) if bc_dofs is not None else None
        self.bc_values = (ctypes.c_double * 4)(*(list(bc_values or [0.0] * self.S) +
                                                 [0.0] * (4 - self.S)))
        self.op = CsrOperator(dm.indptr, dm.indices, self.K64, K32=self.K32, diag64=self.D64,
                              diag32=self.D32, bc_mask=self.bc_mask, dscale=self.D, S=self.S,
                              ld=self.ld)
        self.engine = engine
        cg = dict(cg or {})
        if engine == "persistent":
            self.cg_config = {"engine": "persistent"}
            self.solver = PersistentCG(self.op, rtol=rtol, max_it=max_it, inner_fp32=inner_fp32,
                                       delta=delta, ctas_per_sm=int(cg.get("ctas_per_sm", 0)))
            self.cg_config["grid"], self.cg_config["block"] = self.solver.grid()
            eng = self.solver.engine()
            self.cg_config["form"] = (
                "window (pipelined, vectors in tensor memory)" if eng["pipelined"] else
                "window (Chronopoulos-Gear, vectors in tensor memory)" if eng["tmem"] else
                "window (Chronopoulos-Gear)" if eng["window"] else "streaming")
        else:
            if autotune and not {"group", "block", "rows_per_tile"} & set(cg):
                self.assemble_operator()
                cg.update(tune_cg(self.op, inner_fp32=inner_fp32))
            self.cg_config = dict(cg, engine="graph")
            self.solver = CGSolver(self.op, rtol=rtol, max_it=max_it, inner_fp32=inner_fp32,
                                   delta=delta, **cg)
        self.U = torch.zeros((n, self.ld), dtype=torch.float64, device=dev)
        self.U_prev = torch.zeros_like(self.U)
        # lumped mass per vertex (the cell-order sums of tp_lumped_diag with shift 1): the
        # right-hand side becomes one element-wise pass
        self.mass = torch.zeros(n, dtype=torch.float64, device=dev)
        call("tp_lumped_diag", ctypes.byref(dm.tpm), 1, 1, None, (ctypes.c_double * 4)(1.0),
             None, ptr(self.mass), None, stream_handle())
        # increments of the last steps, newest first (u^n - u^{n-1}, u^{n-1} - u^{n-2}, ...):
        # directions of the projected learned guess
        self.dU = [torch.zeros_like(self.U) for _ in range(5)]
        self.n_hist = 0
        # their stiffness images D_s K dU[k] (written by operator_images when it images the
        # newest increment; kept while the stiffness is unchanged), and which are current
        self.dimg = [torch.zeros_like(self.U) for _ in range(5)]
        self.img_ok = [False] * 5
        self._opU = None
        # False: the history rotates by pointer (cheapest); True: the buffers stay fixed and
        # their contents shift (a captured CUDA graph of the step replays correctly)
        self.history_shift = False
        # D_s K_xi alone (no diagonal): the stiffness images the learned guess reads
        self.stiff_op = CsrOperator(dm.indptr, dm.indices, self.K64, dscale=self.D, S=self.S,
                                    ld=self.ld)
        self.guess = guess
        self.predictor = None
        self.steps_done = 0

    # -- per-step pieces -------------------------------------------------------------
    def assemble_operator(self):
        """Shared stiffness K_xi (FP64, FP32) and the per-column lumped diagonal in one row
        walk (tp_assemble_stiffness_diag); with the persistent FP32 engine the same launch
        writes the solver's FP32 SELL values (no separate scatter)."""
        sol = getattr(self, "solver", None)
        direct = (self.engine == "persistent" and sol is not None and sol.inner_fp32
                  and sol.sM is None)
        call("tp_assemble_stiffness_diag", ctypes.byref(self.dm.tpm), ptr(self.coef), self.S,
             self.ld, ptr(self.alpha), self._shift(), ptr(self.bc_mask), ptr(self.K64),
             ptr(self.K32), ptr(sol.sell.slice_ptr) if direct else None,
             ptr(sol.sK) if direct else None, ptr(self.D64), ptr(self.D32), stream_handle())
        self._sell_fresh = direct

    def _shift(self):
        return (ctypes.c_double * 4)(*([self.inv_dt + kk for kk in self.k] +
                                       [0.0] * (4 - self.S)))

    def assemble_stiffness(self):
        """Shared stiffness K_xi (FP64 and FP32 values)."""
        call("tp_assemble_csr", ctypes.byref(self.dm.tpm), ptr(self.coef), None, 0.0, 1,
             _lib.TP_ASM_STIFF, None, ptr(self.K64), ptr(self.K32), stream_handle())

    def assemble_diagonal(self):
        """Per-column lumped (1/dt + k_s + alpha_s) m."""
        call("tp_lumped_diag", ctypes.byref(self.dm.tpm), self.S, self.ld, ptr(self.alpha),
             self._shift(), ptr(self.bc_mask), ptr(self.D64), ptr(self.D32), stream_handle())

    def assemble_rhs(self):
        """b = M (U/dt + f) per column (lumped M, tp_lumped_rhs); f (V, ld) when a source is
        set (self.f)."""
        n_bc = 0 if self.bc_dofs is None else int(self.bc_dofs.numel())
        call("tp_lumped_rhs", self.dm.n_verts, self.S, self.ld, ptr(self.mass), ptr(self.U),
             ptr(getattr(self, "f", None)), self.inv_dt, n_bc, ptr(self.bc_dofs),
             self.bc_values, ptr(self.solver.b), stream_handle())

    def initial_guess(self):
        x = self.solver.x
        if self.guess == "learned" and self.predictor is not None and self.steps_done > 0:
            self.predictor.predict_into(self, x)
        elif self.guess == "project" and self.steps_done > 0 and self.n_hist > 0:
            self.project_history(x)
        elif self.guess == "extrapolate" and self.steps_done > 0:
            x.copy_(self.U)  # x = 2 u^n - u^{n-1}
            call("tp_axpby", x.numel(), -1.0, ptr(self.U_prev), 2.0, ptr(x), stream_handle())
        else:
            x.copy_(self.U)

    def project_history(self, x, extra=None, extra_img=None, ops=None):
        """x = u^n + sum_k c_k d_k, the energy-norm (Galerkin) projection over the step
        increments d = (u^n - u^{n-1}, ..., at most five) and, when given, one more
        direction `extra` (the learned correction) -- tp_guess_project; ops: the state's
        stiffness images when already computed (operator_images()).  Without `extra`
        this is the projected guess with no network at all (the ablation baseline of the
        learned guess)."""
        if getattr(self, "_gp_work", None) is None:
            self._gp_work = torch.empty(int(_lib.lib.tp_guess_project_workspace_doubles()),
                                        dtype=torch.float64, device=self.device)
        ops = self.operator_images() if ops is None else ops
        nh = max(1, int(self.n_hist))
        dirs = [self.dU[0]] + ([extra] if extra is not None else []) + list(self.dU[1:nh])
        imgs = [ops[1]] + ([extra_img] if extra is not None else []) + \
            [self.dimg[k] if self.img_ok[k] else None for k in range(1, nh)]
        arr = (ctypes.c_void_p * len(dirs))(*[ptr(d) for d in dirs])
        iarr = (ctypes.c_void_p * len(dirs))(*[ptr(d) for d in imgs])
        call("tp_guess_project", ctypes.byref(self.stiff_op.struct), ptr(self.D64),
             ptr(self.bc_mask), ptr(self.solver.b), ptr(self.U), ptr(ops[0]), len(dirs), arr,
             iarr, ptr(x), ptr(self._gp_work), stream_handle())

    def operator_images(self, U=None, U_prev=None, fresh=False):
        """(D_s K U, D_s K (U - U_prev)) with the current stiffness, one launch
        (tp_csr_images).  Defaults to the state: then the second image is that of the newest
        increment dU[0] and is kept in dimg[0].  fresh=True: new buffers."""
        state = U is None and U_prev is None and not fresh
        U = self.U if U is None else U
        Up = self.U_prev if U_prev is None else U_prev
        if state:
            if self._opU is None:
                self._opU = torch.empty_like(self.U)
            opU, opDU = self._opU, self.dimg[0]
            self.img_ok[0] = True
        else:
            opU, opDU = torch.empty_like(self.U), torch.empty_like(self.U)
        call("tp_csr_images", ctypes.byref(self.stiff_op.struct), ptr(U), ptr(Up), ptr(opU),
             ptr(opDU), stream_handle())
        return opU, opDU

    def set_state(self, U, U_prev=None):
        u = to_device(U, torch.float64, self.device).reshape(-1, self.S)
        self.U.zero_()
        self.U[:, : self.S] = u
        self.U_prev.copy_(self.U if U_prev is None else self._pad(U_prev))
        self.steps_done = 0 if U_prev is None else 1
        self.n_hist = 0
        self.img_ok = [False] * len(self.dimg)
        if U_prev is not None:
            self.dU[0].copy_(self.U)
            self.dU[0].sub_(self.U_prev)
            self.n_hist = 1

    def _pad(self, U):
        out = torch.zeros_like(self.U)
        out[:, : self.S] = to_device(U, torch.float64, self.device).reshape(-1, self.S)
        return out

    def step(self, sync=True):
        self.step_operator()
        return self.step_state(sync)

    def step_operator(self):
        """The part of a step that does not read the state: the operator."""
        self.assemble_operator()
        if self.engine == "persistent" and not self._sell_fresh:
            self.solver.refresh_values()

    def step_state(self, sync=True):
        """The rest of a step: right-hand sides, initial guess, solve, state update."""
        self.assemble_rhs()
        self.initial_guess()
        self.solver.run()
        self.advance_state()
        if not sync:
            return None
        res = self.solver.result()
        if self.guess == "learned" and self.predictor is not None and self.steps_done > 1:
            # a timed-out inference left a valid (older) guess; the solve is unaffected
            res["guess_timed_out"] = self.predictor.timed_out()
        return res

    def advance_state(self):
        """After a solve: the increment x - U joins the history (newest first), then
        U_prev = U, U = x."""
        if self.history_shift:
            arr = (ctypes.c_void_p * len(self.dU))(*[ptr(d) for d in self.dU])
            arr2 = (ctypes.c_void_p * len(self.dimg))(*[ptr(d) for d in self.dimg])
            call("tp_advance_history", self.U.numel(), ptr(self.solver.x), ptr(self.U),
                 ptr(self.U_prev), len(self.dU), arr, arr2, stream_handle())
        else:
            d = self.dU.pop()
            call("tp_advance_state", self.U.numel(), ptr(self.solver.x), ptr(self.U),
                 ptr(self.U_prev), ptr(d), stream_handle())
            self.dU.insert(0, d)
            self.dimg.insert(0, self.dimg.pop())
        self.img_ok = [False] + self.img_ok[:-1]
        self.n_hist = min(self.n_hist + 1, len(self.dU))
        self.steps_done += 1

    def state(self) -> np.ndarray:
        return self.U[:, : self.S].cpu().numpy()

    def launches_per_step(self, res: dict) -> int:
        """Kernels of this library one step launched: stiffness assembly, lumped diagonal,
        RHS, the guess, and the solve graph's I1, I2, F1, F2 plus B1, B2, B4 per iteration
        and RU1, RU2 per reliable update."""
        guess = 1 if (self.guess != "previous" and self.steps_done > 1) else 0
        if self.guess == "learned" and self.predictor is not None:
            guess = self.predictor.launches
        elif self.guess == "project":
            guess = 4  # stiffness images, projection dots, coefficients, update
        if self.engine == "persistent":
            # operator (+ SELL scatter for the FP64 engine), RHS, guess, solve, increment
            return 1 + (0 if getattr(self, "_sell_fresh", False) else 1) + 1 + guess + 1 + 1
        return 3 + guess + 4 + 3 * int(res["iterations"]) + 2 * int(res["n_reliable"]) + 1

    def step_host(self, u_host: torch.Tensor, out_host: torch.Tensor):
        """End-to-end step through host buffers: (V, S) float64 pinned in -> out (V, S).
        One H2D copy into a staging array, packing to the interleaved state on the
        device, the step, unpacking and one D2H copy."""
        n = self.U.shape[0]
        if getattr(self, "_stage", None) is None:
            self._stage = torch.empty((n, self.S), dtype=torch.float64, device=self.device)
            self._copy_stream = torch.cuda.Stream(device=self.device)
            self._copied = torch.cuda.Event()
        main = torch.cuda.current_stream(self.device)
        # the H2D copy overlaps the operator assembly, which does not read the state
        self._copy_stream.wait_stream(main)
        with torch.cuda.stream(self._copy_stream):
            self._stage.copy_(u_host, non_blocking=True)
            self._copied.record()
        self._stage.record_stream(self._copy_stream)
        self.step_operator()
        main.wait_event(self._copied)
        st = stream_handle()
        call("tp_pack_columns", n, self.S, self.ld, ptr(self._stage), ptr(self.U), st)
        self.step_state(sync=False)
        call("tp_unpack_columns", n, self.S, self.ld, ptr(self.U), ptr(self._stage), st)
        out_host.copy_(self._stage, non_blocking=True)
