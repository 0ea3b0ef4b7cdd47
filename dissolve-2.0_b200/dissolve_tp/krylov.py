"""Jacobi-PCG solver objects over the C ABI (tp_cg_*).

A CGSolver owns fixed device buffers b, x (n_rows, ld) and a captured CUDA graph,
the way numerics/solvers.py:311-336 caches one KSP with its Vecs per field name.
Values of the operator and of b/x change between runs; addresses do not.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import TpCgConfig, TpCgResult, TpCsrOp, call
from .device import empty_aligned, ptr, stream_handle

LANE_STATUS = {0: "converged", 6: "max_it", 7: "breakdown", 8: "non-finite", -1: "running"}


class CsrOperator:
    """y[:, s] = dscale[s] (K x)[:, s] + cscale[s] (M x)[:, s] + diag[:, s] x[:, s] on a shared
    CSR pattern; identity rows where bc_mask != 0.  Arrays are referenced, not copied."""

    def __init__(self, indptr, indices, K64, K32=None, M64=None, M32=None, diag64=None,
                 diag32=None, bc_mask=None, dscale=None, cscale=None, S=1, ld=None,
                 n_systems=1, sys_row_ptr=None):
        if ld is None:
            ld = {1: 1, 2: 2, 3: 4, 4: 4}[S]
        self.S, self.ld = int(S), int(ld)
        self.n_rows = int(indptr.numel()) - 1
        self.arrays = dict(indptr=indptr, indices=indices, K64=K64, K32=K32, M64=M64, M32=M32,
                           diag64=diag64, diag32=diag32, bc_mask=bc_mask)
        self.n_systems = int(n_systems)
        self._sys_row_ptr = None
        if sys_row_ptr is not None:
            self._sys_row_ptr = np.ascontiguousarray(np.asarray(sys_row_ptr, dtype=np.int64))
        self.dscale = list(dscale) if dscale is not None else [1.0] * self.S
        self.cscale = list(cscale) if cscale is not None else [0.0] * self.S
        self.struct = self._make()

    def _make(self) -> TpCsrOp:
        a = self.arrays
        op = TpCsrOp()
        op.n_rows = self.n_rows
        op.S, op.ld = self.S, self.ld
        for k in ("indptr", "indices", "K64", "K32", "M64", "M32", "diag64", "diag32", "bc_mask"):
            setattr(op, k, ptr(a[k]))
        for s in range(self.S):
            op.dscale[s] = float(self.dscale[s])
            op.cscale[s] = float(self.cscale[s])
        op.n_systems = self.n_systems
        op.sys_row_ptr = (self._sys_row_ptr.ctypes.data if self._sys_row_ptr is not None
                          else None)
        return op

    def set_scales(self, dscale=None, cscale=None):
        if dscale is not None:
            self.dscale = list(dscale)
        if cscale is not None:
            self.cscale = list(cscale)
        self.struct = self._make()

    def apply(self, x: torch.Tensor, y: torch.Tensor | None = None, fp32: bool = False):
        if y is None:
            y = torch.empty_like(x)
        call("tp_csr_apply", ctypes.byref(self.struct), int(fp32), ptr(x), ptr(y), stream_handle())
        return y


class CGSolver:
    """Jacobi-PCG on every (system, column) lane, FP64 or FP32-inner + FP64 reliable updates."""

    def __init__(self, op: CsrOperator, rtol=1e-8, max_it=1000, inner_fp32=False, delta=0.1,
                 group=4, block=256, rows_per_tile=256, use_graph_loop=True):
        self.op = op
        dev = op.arrays["indptr"].device
        self.device = dev
        self.n_lanes = op.n_systems * op.S
        self.b = torch.zeros((op.n_rows, op.ld), dtype=torch.float64, device=dev)
        self.x = torch.zeros((op.n_rows, op.ld), dtype=torch.float64, device=dev)
        self.rtol = torch.empty(self.n_lanes, dtype=torch.float64, device=dev)
        self.set_rtol(rtol)
        cfg = TpCgConfig()
        cfg.max_it = int(max_it)
        cfg.inner_fp32 = int(bool(inner_fp32))
        cfg.delta = float(delta)
        cfg.group = int(group)
        cfg.block = int(block)
        cfg.rows_per_tile = int(rows_per_tile)
        cfg.use_graph_loop = int(bool(use_graph_loop))
        self.cfg = cfg
        nbytes = _lib.lib.tp_cg_workspace_bytes(ctypes.byref(op.struct), ctypes.byref(cfg))
        if nbytes == 0:
            raise ValueError("invalid solver configuration")
        self._ws_buf, self._ws = empty_aligned(nbytes, dev)
        self._ws_bytes = int(nbytes)
        h = ctypes.c_void_p()
        call("tp_cg_create", ctypes.byref(op.struct), ctypes.byref(cfg), ptr(self.b),
             ptr(self.x), ptr(self.rtol), self._ws, self._ws_bytes, stream_handle(),
             ctypes.byref(h))
        self._h = h

    def set_rtol(self, rtol):
        r = np.broadcast_to(np.asarray(rtol, dtype=np.float64), (self.n_lanes,))
        self.rtol.copy_(torch.from_numpy(np.array(r, dtype=np.float64)))

    def run(self):
        """Enqueue one solve on the current stream (no host synchronisation)."""
        call("tp_cg_run", self._h, stream_handle())

    def result(self) -> dict:
        res = TpCgResult()
        n = self.n_lanes
        it = np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        rn = np.zeros(n, dtype=np.float64)
        bn = np.zeros(n, dtype=np.float64)
        call("tp_cg_result_get", self._h, ctypes.byref(res), it.ctypes.data, st.ctypes.data,
             rn.ctypes.data, bn.ctypes.data, stream_handle())
        return {"status": int(res.status), "converged": int(res.status) == 0,
                "iterations": int(res.iterations), "n_reliable": int(res.n_reliable),
                "lane_iterations": it, "lane_status": st, "rnorm": rn, "bnorm": bn}

    def solve(self) -> dict:
        self.run()
        return self.result()

    def time_spmv(self, reps=20) -> float:
        ms = ctypes.c_float(0)
        call("tp_cg_time_spmv", self._h, int(reps), ctypes.byref(ms), stream_handle())
        return float(ms.value)

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib.tp_cg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
