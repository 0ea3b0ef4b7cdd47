"""Coupled step on a gyroid scaffold: interface reaction from the level set, the
three-species transport solve, and the level-set advance.

Per step (the shape of dissolve.py's time loop, :684-954, for the transport part):

  1. grad phi (tp_nodal_gradient), hv = k_ORR H_eps(phi) per vertex, |grad phi|, and the
     explicit OH- source f_OH = orr_factor hv c_O2^n (tp_interface_terms);
  2. O2 consumption: alpha_O2 per cell = mean of hv over the cell's vertices
     (tp_cell_average_col), then the per-species lumped diagonal (1/dt + k_s + alpha_s) m;
  3. right-hand sides M (u^n/dt + f), initial guess (previous step or the learned
     predictor), one 3-column Jacobi-PCG solve (FP32 inner + FP64 refinement);
  4. phi -= dt rate (1 + gain c_Cl^{n+1}) (tp_levelset_advance).

The stiffness K_xi (per-cell diffusivity factor, D_s as a per-column scale) does not
depend on phi and is assembled once.  `GyroidStepPlain` is the plain FP64 form of the same
step: per species full FP64 assembly, RHS and FP64 solve.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import call
from .assembler import GPUSparseAssembler
from .device import ptr, stream_handle, to_device
from .krylov import CsrOperator, PersistentCG
from .mesh import gyroid_cube
from .transport import BatchedTransport

D_S = (1.0, 1.0, 2.6)  # O2, Cl-, OH-
K_S = (0.5, 0.0, 0.2)
O2, CL, OH = 0, 1, 2


def gyroid_inputs(n: int, jitter: float, seed_mesh: int = 0, seed_coef: int = 1,
                  seed_fields: int = 2):
    """Mesh on [0, 2 pi]^3, phi = gyroid - 0.3, per-cell factor exp(0.3 xi), u ~ U(0, 1)."""
    mesh, phi = gyroid_cube(n, jitter, seed_mesh)
    coef = np.exp(0.3 * np.random.default_rng(seed_coef).standard_normal(mesh.n_cells))
    u0 = np.random.default_rng(seed_fields).uniform(0.0, 1.0, (mesh.n_verts, 3))
    return mesh, phi, coef, u0


class GyroidStep:
    def __init__(self, mesh, phi, coef, dt=0.02, rtol=1e-8, max_it=5000, k_orr=2.0,
                 eps_factor=1.5, orr_factor=2.0, rate=0.01, gain=0.5, inner_fp32=True,
                 guess="previous", h=None):
        self.dt = float(dt)
        self.k_orr, self.orr_factor = float(k_orr), float(orr_factor)
        self.rate, self.gain = float(rate), float(gain)
        ext = float(np.ptp(mesh.coords[:, 0]))
        n_side = round(mesh.n_cells ** (1.0 / 3.0) / 6 ** (1.0 / 3.0))
        self.h = float(h) if h is not None else ext / max(n_side, 1)
        self.eps = float(eps_factor) * self.h
        self.tr = BatchedTransport(mesh, coef, D_S, K_S, dt, rtol=rtol, max_it=max_it,
                                   inner_fp32=inner_fp32, guess=guess,
                                   alpha_cells=np.zeros((mesh.n_cells, 3)))
        tr = self.tr
        tr.history_shift = True  # the step is meant to be captured in a CUDA graph
        dev = tr.device
        self.device = dev
        nv = tr.dm.n_verts
        self.phi = to_device(phi, torch.float64, dev).clone()
        self.grad = torch.zeros((nv, 3), dtype=torch.float64, device=dev)
        self.hv = torch.zeros(nv, dtype=torch.float64, device=dev)
        self.ngphi = torch.zeros(nv, dtype=torch.float64, device=dev)
        tr.f = torch.zeros((nv, tr.ld), dtype=torch.float64, device=dev)
        tr.phi, tr.ngphi = self.phi, self.ngphi  # predictor features
        tr.assemble_stiffness()
        tr.assemble_diagonal()
        if tr.engine == "persistent":
            tr.solver.refresh_values()

    # ---- pieces of one step
    def coefficients(self):
        tr, st = self.tr, stream_handle()
        call("tp_nodal_gradient", ctypes.byref(tr.dm.tpm), None, ptr(self.phi), ptr(self.grad),
             st)
        call("tp_interface_terms", tr.dm.n_verts, ptr(self.phi), ptr(self.grad), self.eps,
             self.k_orr, self.orr_factor, tr.ld, ptr(tr.U), O2, OH, ptr(tr.f), ptr(self.hv),
             ptr(self.ngphi), st)
        call("tp_cell_average_col", tr.dm.n_cells, ptr(tr.dm.cells), ptr(self.hv), tr.ld, O2,
             ptr(tr.alpha), st)
        tr.assemble_diagonal()

    def advance_levelset(self):
        tr = self.tr
        call("tp_levelset_advance", tr.dm.n_verts, ptr(self.phi), tr.ld, ptr(tr.U), CL, self.dt,
             self.rate, self.gain, stream_handle())

    def step(self, sync=True):
        tr = self.tr
        self.coefficients()
        tr.assemble_rhs()
        tr.initial_guess()
        tr.solver.run()
        tr.advance_state()
        self.advance_levelset()
        return tr.solver.result() if sync else None

    def set_state(self, U, U_prev=None):
        self.tr.set_state(U, U_prev)

    def state(self) -> np.ndarray:
        return self.tr.state()

    def launches_per_step(self) -> int:
        """gradient, interface terms, cell average, diagonal, RHS, guess, solve, increment,
        level set"""
        guess = self.tr.predictor.launches if (self.tr.guess == "learned"
                                               and self.tr.predictor is not None) else 0
        return 8 + guess

    # ---- learned warm start
    def train_predictor(self, steps: int, every: int = 10, epochs: int = 400, seed: int = 3,
                        verbose: bool = False):
        """Run `steps` steps with the current guess, keep (u^{n-1}, u^n, u^{n+1}) with that
        step's phi and |grad phi| every `every` steps, train a WarmStartMLP on them and
        attach it as the initial guess.  Returns the per-step results of the run."""
        from .mlp import WarmStartMLP

        tr = self.tr
        samples, results = [], []
        for i in range(steps):
            keep = (i % every == every - 1) and tr.steps_done >= 1
            if keep:
                # the step's inputs: u^{n-1}, u^n, their stiffness images and the phi its
                # coefficients use
                up, un, ph = tr.U_prev.clone(), tr.U.clone(), self.phi.clone()
                op = tr.operator_images(un, up, fresh=True)
            res = self.step()
            results.append(res)
            if not res["converged"]:
                raise RuntimeError(f"training trajectory did not converge at step {i}: {res}")
            if keep:
                samples.append((up, un, tr.U.clone(), ph, self.ngphi.clone(), op))
        mlp = WarmStartMLP(self.device, seed=seed)
        mlp.fit_normalization([s[:3] for s in samples], tr.S, tr.D, tr.k, samples[-1][3],
                              samples[-1][4], ops=[s[5] for s in samples])
        for s in samples:
            mlp.add_pairs([s[:3]], tr.S, tr.ld, tr.D, tr.k, s[3], s[4], ops=[s[5]])
        log = mlp.train(steps=epochs, log_every=100 if verbose else 0)
        if verbose:
            print("mlp training loss", log)
        tr.predictor = mlp
        tr.guess = "learned"
        return results


class GyroidStepPlain:
    """The plain FP64 form of the coupled step: per species FP64 assembly of
    (1/dt + k_s + alpha_s) M + D_s xi K, FP64 RHS with the source, FP64 Jacobi-PCG."""

    def __init__(self, mesh, phi, coef, dt=0.02, rtol=1e-8, max_it=5000, k_orr=2.0,
                 eps_factor=1.5, orr_factor=2.0, rate=0.01, gain=0.5, h=None):
        self.dt, self.inv_dt = float(dt), 1.0 / float(dt)
        self.k_orr, self.orr_factor = float(k_orr), float(orr_factor)
        self.rate, self.gain = float(rate), float(gain)
        ext = float(np.ptp(mesh.coords[:, 0]))
        n_side = round(mesh.n_cells ** (1.0 / 3.0) / 6 ** (1.0 / 3.0))
        self.h = float(h) if h is not None else ext / max(n_side, 1)
        self.eps = float(eps_factor) * self.h
        self.asm = [GPUSparseAssembler(mesh)]
        for _ in range(2):
            self.asm.append(GPUSparseAssembler(ref_asm=self.asm[0]))
        a0 = self.asm[0]
        dev = a0.device
        self.device = dev
        self.dm = a0._dm
        nv, nc = a0.n_dofs, a0.n_cells
        coef_d = to_device(coef, torch.float64, dev)
        self.De = [coef_d * d for d in D_S]
        self.alpha = [torch.full((nc,), k, dtype=torch.float64, device=dev) for k in K_S]
        self.hv_cell = torch.zeros((nc, 1), dtype=torch.float64, device=dev)
        self.solvers = []
        for s in range(3):
            op = CsrOperator(self.asm[s].d_indptr, self.asm[s].d_indices, self.asm[s].d_data)
            self.solvers.append(PersistentCG(op, rtol=rtol, max_it=max_it,
                                             sell=self.solvers[0].sell if s else None))
        self.U = torch.zeros((nv, 4), dtype=torch.float64, device=dev)
        self.f = torch.zeros((nv, 4), dtype=torch.float64, device=dev)
        self.phi = to_device(phi, torch.float64, dev).clone()
        self.grad = torch.zeros((nv, 3), dtype=torch.float64, device=dev)
        self.hv = torch.zeros(nv, dtype=torch.float64, device=dev)
        self.cols = [torch.zeros(nv, dtype=torch.float64, device=dev) for _ in range(3)]

    def set_state(self, U):
        self.U.zero_()
        self.U[:, :3] = to_device(U, torch.float64, self.device)

    def state(self) -> np.ndarray:
        return self.U[:, :3].cpu().numpy()

    def step(self, sync=True):
        st = stream_handle()
        call("tp_nodal_gradient", ctypes.byref(self.dm.tpm), None, ptr(self.phi), ptr(self.grad),
             st)
        call("tp_interface_terms", self.dm.n_verts, ptr(self.phi), ptr(self.grad), self.eps,
             self.k_orr, self.orr_factor, 4, ptr(self.U), O2, OH, ptr(self.f), ptr(self.hv),
             None, st)
        call("tp_cell_average_col", self.dm.n_cells, ptr(self.dm.cells), ptr(self.hv), 1, 0,
             ptr(self.hv_cell), st)
        alpha_o2 = self.alpha[O2] + self.hv_cell.view(-1)
        for s in range(3):
            asm, sol = self.asm[s], self.solvers[s]
            asm.assemble(self.De[s], self.inv_dt, alpha=alpha_o2 if s == O2 else self.alpha[s])
            self.cols[s].copy_(self.U[:, s])
            b = asm.assemble_rhs(self.cols[s], self.inv_dt,
                                 f=self.f[:, s].contiguous() if s == OH else None)
            sol.b.view(-1).copy_(b)
            sol.x.view(-1).copy_(self.cols[s])
            sol.refresh_values()
            sol.run()
        for s in range(3):
            self.U[:, s].copy_(self.solvers[s].x.view(-1))
        call("tp_levelset_advance", self.dm.n_verts, ptr(self.phi), 4, ptr(self.U), CL, self.dt,
             self.rate, self.gain, st)
        return [s.result() for s in self.solvers] if sync else None
