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


class SellPattern:
    """SELL-32 layout of a CSR pattern (tp_sell_build) plus the CSR->SELL position map."""

    def __init__(self, indptr: torch.Tensor, indices: torch.Tensor):
        from ._lib import _c_i64
        dev = indptr.device
        self.n_rows = int(indptr.numel()) - 1
        ns = (self.n_rows + 31) // 32
        self.slice_ptr = torch.empty(ns + 1, dtype=torch.int32, device=dev)
        ne = _c_i64(0)
        call("tp_sell_build", self.n_rows, ptr(indptr), ptr(indices), ptr(self.slice_ptr), None,
             None, ctypes.byref(ne), stream_handle())
        self.n_entries = int(ne.value)
        self.nnz = int(indices.numel())
        self.sell_col = torch.empty(max(self.n_entries, 1), dtype=torch.int32, device=dev)
        self.csr2sell = torch.empty(max(self.nnz, 1), dtype=torch.int32, device=dev)
        call("tp_sell_build", self.n_rows, ptr(indptr), ptr(indices), ptr(self.slice_ptr),
             ptr(self.sell_col), ptr(self.csr2sell), ctypes.byref(ne), stream_handle())

    def values(self, dtype):
        return torch.zeros(max(self.n_entries, 1), dtype=dtype, device=self.slice_ptr.device)

    def scatter(self, csr_vals64, out32=None, out64=None):
        call("tp_sell_scatter", self.nnz, ptr(self.csr2sell), ptr(csr_vals64), ptr(out32),
             ptr(out64), stream_handle())


class PersistentCG:
    """The same Jacobi-PCG as CGSolver for one system, as one cooperative kernel per solve
    (tp_pcg_*).  The inner operator is read in SELL-32 order: call refresh_values() after the
    CSR values change (it scatters them)."""

    def __init__(self, op: CsrOperator, rtol=1e-8, max_it=1000, inner_fp32=False, delta=0.01,
                 sell: SellPattern | None = None, ctas_per_sm: int = 0):
        from ._lib import TpSell
        if op.n_systems != 1:
            raise ValueError("the persistent engine solves one system")
        self.op = op
        dev = op.arrays["indptr"].device
        self.device = dev
        self.n_lanes = op.S
        self.inner_fp32 = bool(inner_fp32)
        self.sell = sell or SellPattern(op.arrays["indptr"], op.arrays["indices"])
        vdt = torch.float32 if inner_fp32 else torch.float64
        self.sK = self.sell.values(vdt)
        self.sM = self.sell.values(vdt) if op.arrays["M64"] is not None else None
        self.b = torch.zeros((op.n_rows, op.ld), dtype=torch.float64, device=dev)
        self.x = torch.zeros((op.n_rows, op.ld), dtype=torch.float64, device=dev)
        self.rtol = torch.empty(self.n_lanes, dtype=torch.float64, device=dev)
        self.set_rtol(rtol)
        st = TpSell()
        st.n_rows, st.n_entries = self.sell.n_rows, self.sell.n_entries
        st.slice_ptr, st.sell_col = ptr(self.sell.slice_ptr), ptr(self.sell.sell_col)
        if inner_fp32:
            st.sK32, st.sM32 = ptr(self.sK), ptr(self.sM)
        else:
            st.sK64, st.sM64 = ptr(self.sK), ptr(self.sM)
        self._sell_struct = st
        nbytes = _lib.lib.tp_pcg_workspace_bytes(ctypes.byref(op.struct), int(inner_fp32))
        if nbytes == 0:
            raise ValueError("invalid persistent solver configuration")
        self._ws_buf, self._ws = empty_aligned(nbytes, dev)
        h = ctypes.c_void_p()
        call("tp_pcg_create", ctypes.byref(op.struct), ctypes.byref(st), int(max_it),
             int(inner_fp32), float(delta), int(ctas_per_sm), ptr(self.b), ptr(self.x),
             ptr(self.rtol), self._ws, int(nbytes), stream_handle(), ctypes.byref(h))
        self._h = h
        self.refresh_values()

    def set_rtol(self, rtol):
        r = np.broadcast_to(np.asarray(rtol, dtype=np.float64), (self.n_lanes,))
        self.rtol.copy_(torch.from_numpy(np.array(r, dtype=np.float64)))

    def refresh_values(self):
        a = self.op.arrays
        if self.inner_fp32:
            self.sell.scatter(a["K64"], out32=self.sK)
            if self.sM is not None:
                self.sell.scatter(a["M64"], out32=self.sM)
        else:
            self.sell.scatter(a["K64"], out64=self.sK)
            if self.sM is not None:
                self.sell.scatter(a["M64"], out64=self.sM)

    def profile_run(self) -> dict:
        """One solve with per-CTA phase clocks; mean and max over CTAs in microseconds."""
        g, _ = self.grid()
        prof = torch.zeros(g * 8, dtype=torch.int64, device=self.device)
        call("tp_pcg_set_profile", self._h, ptr(prof))
        try:
            res = self.solve()
        finally:
            call("tp_pcg_set_profile", self._h, None)
        p = prof.view(g, 8).double().cpu().numpy() / 1e3
        names = ["A_work", "A_wait", "B_work", "B_wait", "scalars", "reliable", "final", "init"]
        return {"result": res, "mean_us": dict(zip(names, p.mean(0).round(1).tolist())),
                "max_us": dict(zip(names, p.max(0).round(1).tolist())),
                "min_us": dict(zip(names, p.min(0).round(1).tolist()))}

    def set_wait_limit(self, limit_s: float = 0.0, missing_arrivals: int = 0):
        """Bound of every grid-barrier wait of the next solves (0: the 2 s default).
        missing_arrivals > 0 is for tests of the failure path: every barrier then waits for
        that many CTAs that do not exist, so the solve ends with TP_ERR_TIMEOUT after
        limit_s; set it back to 0 for normal solves (the handle stays usable)."""
        call("tp_pcg_set_wait_limit", self._h, int(round(limit_s * 1e9)), int(missing_arrivals))

    def grid(self):
        g, b = ctypes.c_int(0), ctypes.c_int(0)
        call("tp_pcg_grid", self._h, ctypes.byref(g), ctypes.byref(b))
        return int(g.value), int(b.value)

    def engine(self) -> dict:
        """Engine of the handle: shared-memory window (Chronopoulos-Gear; `tmem`: with the
        recurrence vectors in tensor memory; `pipelined`: the one-barrier pipelined form,
        vectors in tensor memory) or streaming."""
        w, sm = ctypes.c_int(0), ctypes.c_size_t(0)
        call("tp_pcg_engine", self._h, ctypes.byref(w), ctypes.byref(sm))
        return {"window": bool(w.value), "tmem": w.value >= 2, "pipelined": w.value == 3,
                "smem_bytes": int(sm.value)}

    def run(self):
        call("tp_pcg_run", self._h, stream_handle())

    def result(self) -> dict:
        res = TpCgResult()
        n = self.n_lanes
        it = np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        rn = np.zeros(n, dtype=np.float64)
        bn = np.zeros(n, dtype=np.float64)
        call("tp_pcg_result_get", self._h, ctypes.byref(res), it.ctypes.data, st.ctypes.data,
             rn.ctypes.data, bn.ctypes.data, stream_handle())
        return {"status": int(res.status), "converged": int(res.status) == 0,
                "iterations": int(res.iterations), "n_reliable": int(res.n_reliable),
                "lane_iterations": it, "lane_status": st, "rnorm": rn, "bnorm": bn}

    def solve(self) -> dict:
        self.run()
        return self.result()

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib.tp_pcg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MatrixFreeCG:
    """Jacobi-PCG whose product is the matrix-free apply (tp_mfcg_solve): the operator of
    tp_matfree_apply -- per column s, sum_e [dscale_s De_e K_e + (inv_dt + alpha_e +
    shift_s) M_e] -- is never assembled; every product recomputes the P1 gradients from the
    coordinates.  The solve of the reference's MatShell branch (numerics/solvers.py:172-203,
    375-404) on the GPU.  b, x: (n_verts, ld) FP64 device arrays; x is the initial guess
    and receives the solution."""

    def __init__(self, dm, S: int = 1, ld: int = 1, rtol=1e-8, max_it: int = 1000,
                 lumped: int = 0, legacy: int = 0):
        from .device import empty_aligned
        self.dm, self.S, self.ld = dm, int(S), int(ld)
        self.max_it, self.lumped, self.legacy = int(max_it), int(lumped), int(legacy)
        self.rtol = np.broadcast_to(np.asarray(rtol, dtype=np.float64), (self.S,)).copy()
        dev = dm.device
        self.b = torch.zeros((dm.n_verts, self.ld), dtype=torch.float64, device=dev)
        self.x = torch.zeros((dm.n_verts, self.ld), dtype=torch.float64, device=dev)
        nb = int(_lib.lib.tp_mfcg_workspace_bytes(dm.n_verts, self.ld))
        self._ws_buf, self._ws = empty_aligned(nb, dev)
        self._nb = nb

    def solve(self, De_cell, inv_dt: float, alpha_cell=None, dscale=None, shift=None,
              bc_mask=None) -> dict:
        from ._lib import TpMfcgResult
        c = ctypes
        res = TpMfcgResult()
        ds = None if dscale is None else (c.c_double * 4)(*(list(dscale) + [0.0] * 4)[:4])
        sh = None if shift is None else (c.c_double * 4)(*(list(shift) + [0.0] * 4)[:4])
        rt = (c.c_double * 4)(*(list(self.rtol) + [0.0] * 4)[:4])
        call("tp_mfcg_solve", c.byref(self.dm.tpm), self.S, self.ld, ptr(De_cell),
             ptr(alpha_cell), ds, sh, float(inv_dt), self.lumped, self.legacy, ptr(bc_mask),
             ptr(self.b), ptr(self.x), rt, self.max_it, self._ws, self._nb, c.byref(res),
             stream_handle())
        S = self.S
        return {"status": int(res.status), "converged": int(res.status) == 0,
                "iterations": int(res.iterations),
                "lane_iterations": np.array(res.lane_iters[:S]),
                "lane_status": np.array(res.lane_status[:S]),
                "rnorm": np.array(res.lane_rnorm[:S]), "bnorm": np.array(res.lane_bnorm[:S])}

    def close(self):
        """Nothing to release beyond the tensors (no handle)."""

