"""Learned warm start: a per-vertex BF16 MLP that predicts the next state as the Krylov
initial guess (kernels in csrc/tp_mlp.cu, C ABI tp_mlp_*).

The network is trained on trajectories the solver itself produces (pairs u^{n-1}, u^n ->
u^{n+1}), by the project's own forward/backward/AdamW kernels.  It predicts the
correction to a base guess (u^n by default, or the linear extrapolation 2 u^n - u^{n-1}),
and the transport guess is the energy-norm projection onto span{u^n - u^{n-1}, that
correction} around u^n (tp_guess_project).  The Krylov solve always
runs to the same tolerance, so the guess only changes how many iterations it takes: the
plain method is both the fallback (no predictor -> previous step) and the measure of the
prediction's error.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np
import torch

from . import _lib
from ._lib import TpMlpInputs, call
from .device import ptr, stream_handle

H, IN = 64, 16
NFEAT = 10  # used inputs: fields 0..6, bias 7, stiffness images 8..9
P = H * IN + H + H * H + H + H + 1
OFF_W1, OFF_B1 = 0, H * IN
OFF_W2, OFF_B2 = OFF_B1 + H, OFF_B1 + H + H * H
OFF_W3, OFF_B3 = OFF_B2 + H, OFF_B2 + 2 * H


def initial_params(seed: int = 3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = np.zeros(P, dtype=np.float32)
    w1 = rng.normal(0, np.sqrt(2.0 / NFEAT), (H, IN))
    w1[:, NFEAT:] = 0.0
    p[OFF_W1:OFF_B1] = w1.reshape(-1)
    p[OFF_W2:OFF_B2] = rng.normal(0, np.sqrt(2.0 / H), H * H)
    p[OFF_W3:OFF_B3] = rng.normal(0, 0.1 / np.sqrt(H), H)
    return p


class WarmStartMLP:
    def __init__(self, device, seed: int = 3, capacity_rows: int = 0, grid: int = 0,
                 base: str = "previous", project: bool = True):
        """base: the guess the network corrects, "previous" (u^n) or "extrapolate"
        (2 u^n - u^{n-1}); the training target is (u^{n+1} - base) / sigma.
        project: the transport guess is u^n + sum_k c_k d_k over the directions
        d = (u^n - u^{n-1}, sigma y, u^{n-1} - u^{n-2}, ..., u^{n-4} - u^{n-5}) (those the
        history has, at most six), c per species from the energy-norm (Galerkin) projection of tp_guess_project,
        never worse than the previous-step guess in that norm; False: base + sigma y."""
        if base not in ("previous", "extrapolate"):
            raise ValueError("base must be 'previous' or 'extrapolate'")
        self.base = base
        self.project = bool(project)
        self._d = None
        self._work = None
        if int(_lib.lib.tp_mlp_param_count()) != P:
            raise RuntimeError("parameter layout mismatch with the library")
        self.device = device
        self.params = torch.from_numpy(initial_params(seed)).to(device)
        self.m = torch.zeros(P, dtype=torch.float32, device=device)
        self.v = torch.zeros(P, dtype=torch.float32, device=device)
        self.step = 0
        self.mean = np.zeros(NFEAT)
        self.istd = np.ones(NFEAT)
        self.sigma = 1.0
        self.grid = grid or 2 * int(_lib.lib.tp_device_sm_count())
        self.ws = torch.empty(int(_lib.lib.tp_mlp_grad_workspace_floats(self.grid)),
                              dtype=torch.float32, device=device)
        self.loss_dev = torch.zeros(1, dtype=torch.float32, device=device)
        # per-call status of the tensor-core inference (1: a bounded wait ran out and the
        # tile's rows kept what they held -- u^n in the solver's x, the previous direction in
        # the projection -- so the solve still starts from a valid guess)
        self.tc_status = torch.zeros(1, dtype=torch.int32, device=device)
        self.X = torch.empty((max(capacity_rows, 1), IN), dtype=torch.bfloat16, device=device)
        self.T = torch.empty(max(capacity_rows, 1), dtype=torch.float32, device=device)
        self.rows = 0
        self.rng = np.random.default_rng(seed)
        # per guess: the stiffness images, the network (+ projection dots, coefficients and
        # update)
        self.launches = 5 if self.project else 2

    # ---- inputs -----------------------------------------------------------------
    def inputs(self, U, Up, S, ld, D, k, phi=None, ngphi=None, ops=None,
               base: int | None = None) -> TpMlpInputs:
        st = TpMlpInputs()
        st.n_verts = int(U.shape[0])
        st.S, st.ld = int(S), int(ld)
        st.U, st.U_prev = ptr(U), ptr(Up)
        st.base = (1 if self.base == "extrapolate" else 0) if base is None else int(base)
        st.phi, st.normgradphi = ptr(phi), ptr(ngphi)
        opU, opDU = ops if ops is not None else (None, None)
        st.opU, st.opDU = ptr(opU), ptr(opDU)
        st.tc_status = ptr(self.tc_status)
        for s in range(S):
            st.logD[s] = math.log(float(D[s]))
            st.k[s] = float(k[s])
        for f in range(NFEAT):
            st.mean[f] = float(self.mean[f])
            st.istd[f] = float(self.istd[f])
        self._keep = (U, Up, phi, ngphi, opU, opDU)
        return st

    def fit_normalization(self, pairs, S, D, k, phi=None, ngphi=None, ops=None):
        """Input/target scales from training pairs [(U_prev, U_n, U_next)] (device) and,
        when given, their stiffness images ops [(opU, opDU)]."""
        up = np.concatenate([p[0][:, :S].cpu().numpy().reshape(-1) for p in pairs])
        un = np.concatenate([p[1][:, :S].cpu().numpy().reshape(-1) for p in pairs])
        nx = np.concatenate([p[2][:, :S].cpu().numpy().reshape(-1) for p in pairs])
        du = un - up
        tg = nx - (2.0 * un - up if self.base == "extrapolate" else un)
        raw = [np.zeros(1) if phi is None else phi.cpu().numpy(),
               np.zeros(1) if ngphi is None else ngphi.cpu().numpy(), un, up, du,
               np.log(np.asarray(D, dtype=np.float64)), np.asarray(k, dtype=np.float64),
               np.zeros(1)]
        for j in range(2):
            raw.append(np.zeros(1) if ops is None else
                       np.concatenate([o[j][:, :S].cpu().numpy().reshape(-1) for o in ops]))
        for f, r in enumerate(raw):
            self.mean[f] = float(np.mean(r))
            sd = float(np.std(r))
            self.istd[f] = 1.0 / sd if sd > 1e-12 else 1.0
        self.mean[7], self.istd[7] = 0.0, 1.0
        self.sigma = float(np.std(tg)) if np.std(tg) > 0 else 1.0

    def add_pairs(self, pairs, S, ld, D, k, phi=None, ngphi=None, ops=None):
        n_new = sum(int(p[1].shape[0]) * S for p in pairs)
        need = self.rows + n_new
        if need > self.X.shape[0]:
            X = torch.empty((need, IN), dtype=torch.bfloat16, device=self.device)
            T = torch.empty(need, dtype=torch.float32, device=self.device)
            if self.rows:
                X[: self.rows].copy_(self.X[: self.rows])
                T[: self.rows].copy_(self.T[: self.rows])
            self.X, self.T = X, T
        st = stream_handle()
        for i, (Up, Un, Unx) in enumerate(pairs):
            V = int(Un.shape[0])
            inp = self.inputs(Un, Up, S, ld, D, k, phi, ngphi,
                              None if ops is None else ops[i])
            r0 = self.rows
            call("tp_mlp_features", ctypes.byref(inp), ptr(self.X) + r0 * IN * 2, st)
            call("tp_mlp_target", V, S, ld, ptr(Un),
                 ptr(Up) if self.base == "extrapolate" else None, ptr(Unx), float(self.sigma),
                 ptr(self.T) + r0 * 4, st)
            self.rows += V * S

    # ---- training ---------------------------------------------------------------
    def train(self, steps=400, batch_rows=65536, lr=2e-3, wd=1e-4, log_every=0):
        losses = []
        st = stream_handle()
        n = self.rows
        b = min(batch_rows, n)
        for i in range(steps):
            self.step += 1
            row0 = int(self.rng.integers(0, max(n - b, 0) + 1))
            lr_i = lr * 0.5 * (1.0 + math.cos(math.pi * i / max(steps, 1)))
            call("tp_mlp_train_step", ptr(self.X), ptr(self.T), row0, b, ptr(self.params),
                 ptr(self.m), ptr(self.v), self.step, float(lr_i), 0.9, 0.999, 1e-8, float(wd),
                 self.grid, ptr(self.ws), None, ptr(self.loss_dev), st)
            if log_every and (i % log_every == 0 or i == steps - 1):
                losses.append((i, float(self.loss_dev.item()) / b))
        return losses

    def gradient(self, row0, nrows):
        """Summed gradient of the mean squared error on rows [row0, row0 + nrows) (no update)."""
        g = torch.empty(P, dtype=torch.float32, device=self.device)
        call("tp_mlp_train_step", ptr(self.X), ptr(self.T), int(row0), int(nrows),
             ptr(self.params), None, None, 1, 0.0, 0.9, 0.999, 1e-8, 0.0, self.grid,
             ptr(self.ws), ptr(g), ptr(self.loss_dev), stream_handle())
        return g, self.loss_dev

    # ---- inference --------------------------------------------------------------
    def predict(self, U, Up, S, ld, D, k, phi=None, ngphi=None, x_out=None, ops=None,
                base: int | None = None):
        """x_out = base + sigma y (base: 0 u^n, 1 2 u^n - u^{n-1}, 2 none; default from
        the constructor), or y itself when x_out is None."""
        inp = self.inputs(U, Up, S, ld, D, k, phi, ngphi, ops, base)
        if x_out is not None:
            call("tp_mlp_predict", ctypes.byref(inp), ptr(self.params), float(self.sigma),
                 ptr(x_out), None, stream_handle())
            return x_out
        y = torch.empty(int(U.shape[0]) * S, dtype=torch.float32, device=self.device)
        call("tp_mlp_predict", ctypes.byref(inp), ptr(self.params), float(self.sigma), None,
             ptr(y), stream_handle())
        return y

    def timed_out(self) -> bool:
        """Whether the last inference gave up on a tensor-core wait (reads the device word)."""
        return bool(int(self.tc_status.item()))

    def predict_into(self, tr, x):
        """The transport driver's hook: guess for tr's next step written into x (tr's
        right-hand side tr.solver.b and diagonal tr.D64 are already assembled)."""
        ops = tr.operator_images()
        phi, ngphi = getattr(tr, "phi", None), getattr(tr, "ngphi", None)
        if not self.project:
            self.predict(tr.U, tr.U_prev, tr.S, tr.ld, tr.D, tr.k, phi, ngphi, x_out=x, ops=ops)
            return
        if self._d is None or self._d.shape != tr.U.shape:
            self._d = torch.zeros_like(tr.U)  # padding columns stay zero
        self.predict(tr.U, tr.U_prev, tr.S, tr.ld, tr.D, tr.k, phi, ngphi, x_out=self._d,
                     ops=ops, base=2)
        # the projection over the increment history plus the network's direction (its
        # stiffness image is gathered; the images of past increments are kept)
        tr.project_history(x, extra=self._d, ops=ops)


def trajectory_pairs(tr, steps):
    """Run `steps` steps of a transport object from its current state, returning the
    (U^{n-1}, U^n, U^{n+1}) triples that have a real history (n >= 1) and the stiffness
    images (D_s K U^n, D_s K (U^n - U^{n-1})) of each."""
    pairs, ops = [], []
    prev = None
    for _ in range(steps):
        cur = tr.U.clone()
        if prev is not None:
            op = tr.operator_images(cur, prev, fresh=True)
        res = tr.step()
        if not res["converged"]:
            raise RuntimeError(f"training trajectory did not converge: {res}")
        if prev is not None:
            pairs.append((prev, cur, tr.U.clone()))
            ops.append(op)
        prev = cur
    return pairs, ops


def attach_trained_predictor(fast, mesh, coef, u_ref, D, K, DT, train_steps=12,
                             epochs=1600, seed=3, verbose=False):
    """Train a WarmStartMLP on a trajectory of the FP64 batched solver started from a
    different random state (seed `seed`) and attach it to `fast` as its guess."""
    from .transport import BatchedTransport

    gen = BatchedTransport(mesh, coef, D, K, DT, rtol=1e-8, inner_fp32=False,
                           guess="previous", asm=fast.asm)
    u_train = np.random.default_rng(seed).uniform(0.0, 1.0, np.asarray(u_ref).shape)
    gen.set_state(u_train)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pairs, ops = trajectory_pairs(gen, train_steps + 1)
    mlp = WarmStartMLP(fast.device, seed=seed)
    mlp.fit_normalization(pairs, fast.S, D, K, ops=ops)
    mlp.add_pairs(pairs, fast.S, fast.ld, D, K, ops=ops)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    log = mlp.train(steps=epochs, log_every=100 if verbose else 0)
    torch.cuda.synchronize()
    # wall time of the trajectory (FP64 solves, features) and of the training steps
    mlp.timings = {"trajectory_s": round(t1 - t0, 4), "train_s": round(time.perf_counter() - t1, 4),
                   "train_steps": epochs, "rows_per_step": min(65536, mlp.rows),
                   "training_rows": int(mlp.rows)}
    if verbose:
        print("mlp training loss", log)
    fast.predictor = mlp
    fast.guess = "learned"
    del gen
    return True
