"""Benchmark: 3-species backward-Euler steps/s at 1.57M P1 tets, rtol 1e-8.

Workload (the three-species multi-RHS case): [0,1]^3 with 64^3 cells Kuhn-split
(1,572,864 tets, 274,625 vertices), interior vertices jittered +-0.2h (seed 0);
per-cell diffusivity D_s exp(0.3 xi), xi ~ N(0,1) (seed 1), D_s = (1.0, 1.0, 2.6)
for O2 / Cl- / OH-, reaction k_s = (0.5, 0.0, 0.2), dt = 0.02, u_prev ~ U(0,1) per
vertex and species (seed 2), lumped mass, no Dirichlet rows.  One step = assemble the
operator, assemble the 3 right-hand sides, form the initial guess and solve all three
species to ||b - A x|| <= 1e-8 ||b||.  Synthetic inputs with the configuration's
shapes and distributions; nothing is read from disk.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is the batched, FP32-inner / FP64-refined form with the learned (or, if no
predictor is trained, previous-step) initial guess, inputs resident on the device;
`e2e` is the same step through the host-buffer API (H2D of u_prev, D2H of u_new inside
the timed region).  `forms` reports the plain FP64 GPU form (species one at a time,
full FP64 CSR assembly + FP64 Jacobi-PCG) on the same steps.  Between timed steps a
512 MiB buffer is written to flush the 126 MB L2.  N > 1 runs N independent replicas
(one mesh per GPU, no collective on the data path; weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (REPO, os.path.join(REPO, "dissolve-2.0_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "3-species BE steps/s at 1.57M P1 tets, rtol 1e-8: mixed+learned vs plain FP64"
N_SIDE, JITTER = 64, 0.2
D_S, K_S, DT, RTOL = (1.0, 1.0, 2.6), (0.5, 0.0, 0.2), 0.02, 1e-8
# steps from u_prev after which both GPU forms are compared with the oracle (and the number
# of steps of the CPU baseline sample)
PARITY_STEPS = 3
# relative residual of the oracle's Jacobi-PCG solves that stand in for exact solutions
ORACLE_RTOL = 1e-12
# measured with ncu on this workload (see profiles/); None until captured
# (k_cgw: 2.627 GB over a 258-iteration launch; k_pcgp: 131.4 MB over a 334-iteration launch)
DRAM_BYTES_PER_ITERATION = {"k_cgw": 10.2e6, "k_pcgp": 0.393e6}
WORKLOAD = ("3-species backward-Euler step, 64^3 Kuhn cube (1,572,864 P1 tets, 274,625 "
            "vertices), jitter 0.2h, De = D_s exp(0.3 xi), rtol 1e-8")


def make_inputs(n_side=N_SIDE):
    from dissolve_tp.mesh import kuhn_cube
    m = kuhn_cube(n_side, JITTER, seed=0)
    xi = np.random.default_rng(1).standard_normal(m.n_cells)
    coef = np.exp(0.3 * xi)
    u0 = np.random.default_rng(2).uniform(0.0, 1.0, (m.n_verts, 3))
    return m, coef, u0


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML every 5 ms in a thread while
    the timed region runs (the region is shorter than nvidia-smi's sampling period)."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, gpu_index: int, period_s: float = 0.005):
        self.idx, self.period = gpu_index, period_s
        self.samples, self.reasons, self.max_mhz = [], set(), None

    def _run(self):
        import pynvml
        h = pynvml.nvmlDeviceGetHandleByIndex(self.idx)
        self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        while True:
            self.samples.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
            mask = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
            for nm, bit in self.REASONS.items():
                if mask & bit:
                    self.reasons.add(nm)
            self._ready.set()
            if self._stop.wait(self.period):
                break

    def __enter__(self):
        import threading
        self._stop = threading.Event()
        self._ready = threading.Event()
        self._thr = None
        try:
            import pynvml
            pynvml.nvmlInit()
            dev = os.environ.get("CUDA_VISIBLE_DEVICES")
            if dev and dev.split(",")[0].strip().isdigit():
                self.idx = int(dev.split(",")[self.idx].strip())
            self._thr = threading.Thread(target=self._run, daemon=True)
            self._thr.start()
            # the first sample is taken before the timed region starts (NVML set-up can
            # take longer than the whole region)
            self._ready.wait(timeout=5.0)
        except Exception as e:  # no NVML: report no samples
            self.error = str(e)
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thr is not None:
            self._thr.join(timeout=2)
        return False

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


# ------------------------------------------------------------------ timing helpers
def timed_steps(step_fn, steps, flush, torch):
    """Per-step CUDA-event timing on the current stream, L2 flushed before each step."""
    ms = []
    for _ in range(steps):
        flush()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        step_fn()
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return ms


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from dissolve_tp.transport import BatchedTransport, PlainTransport

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    m, coef, u0 = make_inputs()
    flush_buf = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def flush():
        flush_buf.zero_()

    if args.kernels_only:
        if rank == 0:
            print(json.dumps({"workload": WORKLOAD, "kernels": kernel_table(m, coef, u0, flush)}),
                  flush=True)
        return

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- mixed + batched (+ learned) form
    cg_extra = {"use_graph_loop": not args.host_loop}
    fast = BatchedTransport(m, coef, D_S, K_S, DT, rtol=RTOL, inner_fp32=True, guess="previous",
                            cg=cg_extra)
    if args.roofline_only:
        # W steps with the previous-step guess (W solves), then the roofline solve: the
        # (W+1)-th launch of the solve kernel, a one-launch case for a profiler
        fast.set_state(u0)
        for _ in range(args.warmup):
            fast.step(sync=True)
        if rank == 0:
            print(json.dumps({"workload": WORKLOAD, "cg_launch": fast.cg_config,
                              "roofline": roofline_solve(fast, flush, torch)}), flush=True)
        return
    learned = False
    if args.guess == "learned":
        from dissolve_tp import mlp as mlpmod
        learned = mlpmod.attach_trained_predictor(fast, m, coef, u0, D_S, K_S, DT,
                                                  train_steps=args.train_steps)
    fast.set_state(u0)
    results = []
    for _ in range(args.warmup):
        fast.step(sync=True)
    torch.cuda.synchronize()
    barrier()
    launches = 0
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        barrier()
        step_ms = []
        for _ in range(args.steps):
            flush()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.nvtx.range_push("timed_step")
            e0.record()
            fast.step(sync=False)
            e1.record()
            torch.cuda.nvtx.range_pop()
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            r = fast.solver.result()
            results.append(r)
            launches += fast.launches_per_step(r)
        torch.cuda.synchronize()
        barrier()
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps / (total_ms / 1e3)
    conv = all(r["converged"] for r in results)
    iters = [int(r["iterations"]) for r in results]

    nnz, nv = fast.dm.nnz, fast.dm.n_verts
    roof = roofline_solve(fast, flush, torch)
    # ---- e2e through the host-buffer API
    e2e = None
    if args.e2e:
        fast.set_state(u0)
        u_host = torch.from_numpy(np.ascontiguousarray(u0)).pin_memory()
        out_host = torch.empty_like(u_host).pin_memory()
        # the same trajectory steps as the resident timing: each step's output is the
        # next step's host input
        for _ in range(max(1, args.warmup)):
            fast.step_host(u_host, out_host)
            torch.cuda.synchronize()
            u_host.copy_(out_host)
        torch.cuda.synchronize()
        e_ms = []
        for _ in range(args.steps):
            flush()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fast.step_host(u_host, out_host)
            e1.record()
            e1.synchronize()
            e_ms.append(e0.elapsed_time(e1))
            u_host.copy_(out_host)
        tot = sum(e_ms)
        if world > 1:
            t = torch.tensor([tot], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            tot = float(t.item())
        e2e = {"value": world * args.steps / (tot / 1e3), "unit": "steps/s",
               "h2d_bytes_per_step": int(u_host.numel() * 8),
               "d2h_bytes_per_step": int(out_host.numel() * 8)}

    # ---- the plain FP64 GPU form on the same steps
    forms = {}
    plain = None
    if args.forms:
        plain = PlainTransport(m, coef, D_S, K_S, DT, rtol=RTOL)
        plain.set_state(u0)
        for _ in range(args.warmup):
            plain.step(sync=True)
        p_ms, p_it = [], []
        for _ in range(args.steps):
            flush()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            plain.step(sync=False)
            e1.record()
            e1.synchronize()
            p_ms.append(e0.elapsed_time(e1))
            p_it.append([int(r["iterations"]) for r in (s.result() for s in plain.solvers)])
        # the same steps in the batched form with FP64 inner iterations
        b64 = BatchedTransport(m, coef, D_S, K_S, DT, rtol=RTOL, inner_fp32=False,
                               guess="previous")
        b64.set_state(u0)
        for _ in range(args.warmup):
            b64.step(sync=True)
        q_ms = timed_steps(lambda: b64.step(sync=False), args.steps, flush, torch)
        # agreement of the fast form with the plain FP64 form after W+K steps
        up = plain.state()
        fast.set_state(u0)
        for _ in range(args.warmup + args.steps):
            fast.step(sync=True)
        uf = fast.state()
        rel = float(np.linalg.norm(uf - up) / np.linalg.norm(up))
        forms = {
            "guess_ablation": guess_ablation(fast, u0, args, flush, torch) if learned else None,
            "plain_fp64": {"steps_per_s": args.steps / (sum(p_ms) / 1e3),
                           "ms_per_step": sum(p_ms) / args.steps,
                           "iterations_per_species": p_it[-1]},
            "batched_fp64": {"steps_per_s": args.steps / (sum(q_ms) / 1e3),
                             "ms_per_step": sum(q_ms) / args.steps},
            "fast_vs_plain_speedup": (args.steps / (total_ms / 1e3 / world)) /
                                     (args.steps / (sum(p_ms) / 1e3)),
            "fast_vs_plain_rel_l2": rel,
        }

    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-inner/f64-refined", "data": "synthetic (seeded, config shapes)",
        "config": {"workload": WORKLOAD, "n_tets": m.n_cells, "n_verts": m.n_verts,
                   "nnz": nnz, "species": 3, "form": "batched 3-column CG, FP32 inner + "
                   "FP64 reliable updates, " + ("learned" if learned else "previous-step")
                   + " initial guess", "mass": "lumped", "l2": "flushed (512 MiB write) "
                   "before every timed step", "parallelism": f"replicas x{world}",
                   "cg_launch": fast.cg_config},
        "converged": conv, "cg_iterations": iters,
        "learned_guess_training": getattr(fast.predictor, "timings", None) if learned else None,
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clk.summary(),
        "e2e": e2e,
        "forms": forms,
    }
    # states of both forms after PARITY_STEPS steps from u0, compared with the oracle in the
    # CPU leg below
    gpu_states = {}
    if args.cpu_baseline and world == 1:
        if plain is None:
            plain = PlainTransport(m, coef, D_S, K_S, DT, rtol=RTOL)
        for name, tr in (("fast", fast), ("plain_fp64", plain)):
            tr.set_state(u0)
            for _ in range(PARITY_STEPS):
                tr.step(sync=True)
            gpu_states[name] = tr.state()
    del plain
    if args.kernels and world == 1:
        line["kernels"] = kernel_table(m, coef, u0, flush)
        line["setup"] = setup_times(m)
    parity_inputs = {}
    if args.configs and world == 1:
        line["other_configs"] = other_configs(flush, parity_inputs)
    if rank == 0 and world == 1 and args.cpu_baseline:
        line["cpu_baseline"], line["parity"] = cpu_baseline(
            m, coef, u0, sample_steps=args.cpu_sample_steps, gpu_states=gpu_states,
            gyroid=parity_inputs.get("gyroid_48"))
    if rank == 0:
        print(json.dumps(line), flush=True)


def roofline_solve(fast, flush, torch):
    """Roofline of the dominant kernel: the persistent CG (one launch per solve), timed live
    with CUDA events around its launch on the same stream, on the current state started
    from the previous-step guess (a solve of ~250 iterations at the last timed state: the
    per-iteration rate, not the per-launch set-up and final residual that dominate the
    shortest learned-guess solves)."""
    nnz, nv = fast.dm.nnz, fast.dm.n_verts
    fast.assemble_operator()
    fast.solver.refresh_values()
    fast.assemble_rhs()
    fast.solver.x.copy_(fast.U)
    torch.cuda.synchronize()
    flush()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    fast.solver.run()
    e1.record()
    e1.synchronize()
    solve_ms = e0.elapsed_time(e1)
    rk = fast.solver.result()
    its = max(int(rk["iterations"]), 1)
    form = fast.cg_config.get("form", "")
    window = form.startswith("window")
    if window and "pipelined" in form:
        # pipelined engine, per iteration, counted as for the window engine: the FP32 value
        # per nonzero and 12 passes of (V, 4) FP32 vectors (m into the windows, the update's
        # reads and writes of z, s, p, r, w, xi)
        bytes_it = nnz * 4 + 12 * nv * 16
        kernel = ("k_pcgp<4> (persistent 3-column pipelined Jacobi-PCG, one grid barrier per "
                  "iteration, values and vectors in tensor memory, one cooperative launch "
                  "per solve)")
        engine = "k_pcgp"
    elif window:
        # window engine, per iteration: FP32 value per nonzero (columns stay in shared
        # memory for the whole solve) and 12 passes of (V, 4) FP32: u read once into the
        # windows; P reads p, s, xi, r, D^-1 and writes p, s, xi, r, u; the product reads
        # the row diagonal (w = A u of the own rows stays in shared memory)
        bytes_it = nnz * 4 + 12 * nv * 16
        kernel = ("k_cgw<float,4> (persistent 3-column Jacobi-PCG, Chronopoulos-Gear form, "
                  "shared-memory windows, one cooperative launch per solve)")
        engine = "k_cgt" if "tensor memory" in form else "k_cgw"
    else:
        # streaming engine: int32 column + FP32 value per nonzero and 12 passes of (V, 4)
        # FP32: A reads z, p and writes p, q; B reads p, q, r, xi, D^-1, writes xi, r, z
        bytes_it = nnz * 8 + 12 * nv * 16
        kernel = ("k_pcg<float,4> (persistent 3-column Jacobi-PCG, one cooperative launch "
                  "per solve)")
        engine = "k_pcg"
    # DRAM bytes per iteration of the same kernel on this workload, from an ncu capture
    # (dram__bytes_read.sum + dram__bytes_write.sum of one launch / its iterations)
    per_it = DRAM_BYTES_PER_ITERATION.get(engine)
    traffic = per_it * its if per_it else None
    peaks = _peaks()
    # the driver-measured copy bandwidth of this pool's B200s, else the recipe's fallback
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "of measured" if "hbm_gbs" in peaks else "of fallback: MEASURED_PEAKS.json absent"
    achieved = bytes_it * its / (solve_ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": kernel,
            "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "traffic": traffic,
            "algorithmic_bytes": bytes_it * its, "bytes_per_iteration": bytes_it,
            "iterations": its, "launch_us": solve_ms * 1e3,
            "us_per_iteration": solve_ms * 1e3 / its,
            "note": f"peak = HBM copy bandwidth ({peak_src}); one solve of the current "
                    "state from the previous-step guess; the operator and vectors stay on "
                    "chip (tensor memory, shared memory) and in the 126 MB L2 between "
                    "iterations, so the solve is bound by its grid barrier and on-chip "
                    "latencies, not by DRAM; traffic = ncu DRAM bytes per iteration x "
                    "iterations of this launch"}


def guess_ablation(fast, u0, args, flush, torch):
    """The same W + K steps from u0 with each initial guess of the fast form: the previous
    step u^n (the reference's, numerics/solvers.py:367), linear extrapolation
    2 u^n - u^{n-1}, the energy-norm projection over the last five step increments alone,
    that projection with the network's correction added as one more direction (the
    shipped learned guess) and the network alone (u^n + sigma y).  CG iterations and
    CUDA-event time per step over the K timed steps."""
    pred = fast.predictor
    modes = [("previous", "previous", True), ("extrapolate", "extrapolate", True),
             ("projection_only", "project", True), ("projection_and_network", "learned", True),
             ("network_only", "learned", False)]
    out = {}
    saved = (fast.guess, pred.project, pred.launches)
    try:
        for name, guess, proj in modes:
            fast.guess = guess
            pred.project = proj
            fast.set_state(u0)
            for _ in range(args.warmup):
                fast.step(sync=True)
            its, ms = [], []
            for _ in range(args.steps):
                flush()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                fast.step(sync=False)
                e1.record()
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
                its.append(int(fast.solver.result()["iterations"]))
            out[name] = {"iterations": int(sum(its)), "per_step": its,
                         "ms_per_step": round(sum(ms) / len(ms), 3)}
    finally:
        fast.guess, pred.project, pred.launches = saved
    b = out["projection_only"]["iterations"]
    out["network_gain_over_projection"] = round(1.0 - out["projection_and_network"]["iterations"] / b, 3) if b else None
    return out


# ------------------------------------------------------------------ other kernels / configs
def _event_ms(fn, reps, flush, torch):
    ts = []
    for _ in range(reps + 2):
        flush()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts[2:]))


def kernel_table(m, coef, u0, flush):
    """Assembly, right-hand side and matrix-free apply at this workload: CUDA-event time
    (median of 10, L2 flushed before each) and algorithmic bytes as in the per-unit
    formulas below (per tet and per vertex), against the measured HBM bandwidth."""
    import ctypes

    import torch

    from dissolve_tp import _lib
    from dissolve_tp.assembler import DeviceMesh
    from dissolve_tp.device import ptr, stream_handle
    dev = torch.device("cuda", torch.cuda.current_device())
    dm = DeviceMesh(m.coords, m.cells)
    n, V, nnz = m.n_cells, m.n_verts, dm.nnz
    st = stream_handle()

    class _Tpm:  # the mesh struct as it is at call time (set_tiles replaces it)
        _as_parameter_ = property(lambda self: ctypes.byref(dm.tpm))
    tpm = _Tpm()
    hbm = _peaks().get("hbm_gbs", 6650.0)
    De = torch.from_numpy(coef).to(dev)
    al = torch.full((n,), 0.5, dtype=torch.float64, device=dev)
    o64 = torch.empty(nnz, dtype=torch.float64, device=dev)
    o32 = torch.empty(nnz, dtype=torch.float32, device=dev)
    U = torch.zeros((V, 4), dtype=torch.float64, device=dev)
    U[:, :3] = torch.from_numpy(u0)
    b = torch.empty_like(U)
    x32 = torch.randn((V, 4), dtype=torch.float32, device=dev)
    y32 = torch.empty_like(x32)
    x64, y64 = x32.double(), torch.empty((V, 4), dtype=torch.float64, device=dev)
    ds = (ctypes.c_double * 4)(*D_S, 0.0)
    sh = (ctypes.c_double * 4)(*K_S, 0.0)
    rows = {
        "assemble_full_fp64": (lambda: _lib.call("tp_assemble_csr", tpm, ptr(De), ptr(al), 50.0,
                                                 1, 0, None, ptr(o64), None, st),
                               n * (16 + 64 + 16) + V * 24 + nnz * 8),
        "assemble_stiffness_fp64_fp32": (lambda: _lib.call("tp_assemble_csr", tpm, ptr(De), None,
                                                           0.0, 1, 1, None, ptr(o64), ptr(o32),
                                                           st),
                                         n * (16 + 64 + 8) + V * 24 + nnz * 12),
        "rhs_3col": (lambda: _lib.call("tp_assemble_rhs", tpm, 3, 4, ptr(U), None, 50.0, 1, 0,
                                       None, None, ptr(b), st), n * 24 + V * 64),
        # consistent mass: cell vertices (16 B) and |detJ| (8 B) per cell, u and b per vertex
        "rhs_3col_consistent": (lambda: _lib.call("tp_assemble_rhs", tpm, 3, 4, ptr(U), None, 50.0,
                                                  0, 0, None, None, ptr(b), st), n * 24 + V * 64),
        "matfree_3col_fp64": (lambda: _lib.call("tp_matfree_apply", tpm, 3, 4, 0, ptr(De), None,
                                                ds, sh, 50.0, 0, 0, ptr(x64), ptr(y64), st),
                              n * 40 + V * 72),
        "matfree_3col_fp32": (lambda: _lib.call("tp_matfree_apply", tpm, 3, 4, 1, ptr(De), None,
                                                ds, sh, 50.0, 0, 0, ptr(x32), ptr(y32), st),
                              n * 28 + V * 48),
    }
    out = {}
    # the row walk the tiled kernels replaced (same results), for comparison
    rows_walk = {"assemble_full_fp64_row_walk": rows["assemble_full_fp64"],
                 "assemble_stiffness_fp64_fp32_row_walk": rows["assemble_stiffness_fp64_fp32"],
                 "rhs_3col_consistent_row_walk": rows["rhs_3col_consistent"]}
    tile_rows = dm.tile_rows
    dm.set_tiles(0)
    for name, (fn, nbytes) in rows_walk.items():
        ms = _event_ms(fn, 10, flush, torch)
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[name] = {"us": round(ms * 1e3, 1), "algorithmic_MB": round(nbytes / 1e6, 1),
                     "GB_s": round(gbs, 1), "frac_hbm": round(gbs / hbm, 3)}
    dm.set_tiles(tile_rows)
    out["tiles"] = dm.tiles_info()
    for name, (fn, nbytes) in rows.items():
        ms = _event_ms(fn, 10, flush, torch)
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[name] = {"us": round(ms * 1e3, 1), "algorithmic_MB": round(nbytes / 1e6, 1),
                     "GB_s": round(gbs, 1), "frac_hbm": round(gbs / hbm, 3)}
    out["peak_gbs"] = {"value": hbm, "source": "measured" if "hbm_gbs" in _peaks() else
                       "fallback (MEASURED_PEAKS.json absent)"}
    out["matrix_free_cg_3col_fp64"] = matrix_free_solve(dm, De, U, flush, torch)
    rows["assemble_full_fp64"][0]()  # o64 = the full operator again (the rows reuse it)
    out["reference_assemble_p1_tet"] = reference_kernel_baseline(dm, De, al, o64, flush, hbm)
    return out


def matrix_free_solve(dm, De, U, flush, torch):
    """The three species solved matrix-free (tp_mfcg_solve: Jacobi-PCG whose product is
    the fused matrix-free apply, FP64, lumped mass, rtol 1e-8) from u_prev, for comparison
    with the assembled-operator engines per iteration."""
    import ctypes

    from dissolve_tp import _lib
    from dissolve_tp.device import ptr, stream_handle
    from dissolve_tp.krylov import MatrixFreeCG
    sol = MatrixFreeCG(dm, 3, 4, rtol=RTOL, max_it=5000, lumped=1)
    _lib.call("tp_assemble_rhs", ctypes.byref(dm.tpm), 3, 4, ptr(U), None, 1.0 / DT, 1, 0, None,
              None, ptr(sol.b), stream_handle())
    res = {}

    def run():
        sol.x.copy_(U)
        res.update(sol.solve(De, 1.0 / DT, dscale=D_S, shift=K_S))

    ms = _event_ms(run, 3, flush, torch)
    its = max(int(res["iterations"]), 1)
    return {"ms": round(ms, 3), "iterations": its, "us_per_iteration": round(ms * 1e3 / its, 2),
            "converged": bool(res["converged"]),
            "note": "FP64, 3 lanes, previous-step guess; every product recomputes the "
                    "gradients (tp_matfree_apply), iterations in batches of 8 between host "
                    "checks"}


def reference_kernel_baseline(dm, De, alpha, ours64, flush, hbm):
    """Baseline leg (not the product): the reference's own GPU assembly kernel,
    assemble_p1_tet of gpu/gpu_assembler.py:60-139, compiled from its source string for
    sm_100a into oracle/_ref/ and launched as the reference launches it (:494-508: the CSR
    values zeroed, then one thread per cell, 128 per block, 16 FP64 atomicAdds through the
    scatter map), on the same mesh and coefficients as the full FP64 row above.  Its
    algorithmic bytes are the scope table's n (16 + 64 + 16) + V 24 + nnz 8; what it reads
    is the reference layout (detJ 8 B + Gflat 72 B per cell)."""
    import ctypes

    import torch

    from dissolve_tp.device import ptr, stream_handle
    path = os.path.join(REPO, "oracle", "_ref", "libref_kernels_gpu.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/libref_kernels_gpu.so not built"}
    lib = ctypes.CDLL(path)
    fn = lib.ref_gpu_assemble_p1_tet
    fn.restype = ctypes.c_int
    detJ, G, _ = dm.ref_geometry
    sm = dm.scatter_map
    n, V, nnz = dm.n_cells, dm.n_verts, dm.nnz
    out = torch.empty(nnz, dtype=torch.float64, device=De.device)
    st = stream_handle()
    grid = (n + 127) // 128

    def launch():
        rc = fn(ctypes.c_uint(grid), ctypes.c_uint(128), ctypes.c_void_p(st), ctypes.c_int(n),
                ctypes.c_void_p(ptr(dm.cells)), ctypes.c_void_p(ptr(detJ)),
                ctypes.c_void_p(ptr(G)), ctypes.c_void_p(ptr(De)), ctypes.c_void_p(ptr(alpha)),
                ctypes.c_double(50.0), ctypes.c_int(1), ctypes.c_void_p(ptr(sm)),
                ctypes.c_void_p(ptr(out)))
        if rc != 0:
            raise RuntimeError(f"reference kernel launch failed ({rc})")

    def with_fill():
        out.zero_()
        launch()

    nbytes = n * (16 + 64 + 16) + V * 24 + nnz * 8
    res = {"source": "gpu/gpu_assembler.py:60-139 compiled for sm_100a (oracle/_ref)"}
    for name, fn_ in (("kernel", launch), ("fill_and_kernel", with_fill)):
        ms = _event_ms(fn_, 10, flush, torch)
        gbs = nbytes / (ms * 1e-3) / 1e9
        res[name] = {"us": round(ms * 1e3, 1), "GB_s": round(gbs, 1),
                     "frac_hbm": round(gbs / hbm, 3)}
    with_fill()
    a, b = out.cpu().numpy(), ours64.cpu().numpy()
    # the atomics add in no fixed order: equal up to rounding
    res["max_rel_diff_vs_ours"] = float(np.abs(a - b).max() / np.abs(b).max())
    return res


def setup_times(m):
    """Mesh setup on the GPU at this workload: geometry, incidence, CSR pattern and the
    element-to-nonzero slots (DeviceMesh), the row tiles of the tiled kernels, then the
    reference-layout scatter map on request; host wall time around each (the setup calls
    synchronise).  Beside it, the reference's own setup (GPUSparseAssembler.__init__ of
    gpu/gpu_assembler.py:331-450) timed on the CPU by tests/golden/time_reference_setup.py
    (recorded in tests/golden/ref_setup_timing.json; its Python and numpy work alone)."""
    import torch

    from dissolve_tp.assembler import DeviceMesh
    out = {}
    for rep in range(2):  # the first run pays one-time module loading
        torch.cuda.synchronize()
        t = time.perf_counter()
        dm = DeviceMesh(m.coords, m.cells, tile_rows=0)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        dm.set_tiles(64)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        _ = dm.scatter_map
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        out = {"device_mesh_s": round(t1 - t, 4), "tiles_s": round(t2 - t1, 4),
               "scatter_map_s": round(t3 - t2, 4),
               "includes": "H2D of coords and cells, geometry, incidence, pattern (two "
                           "passes), slots; row tiles (host-built tables); scatter map built "
                           "only on request"}
        del dm
    try:
        ref = json.load(open(os.path.join(REPO, "tests", "golden", "ref_setup_timing.json")))
        out["reference_setup_s"] = ref["setup_64cube_s"]
        out["reference_setup_note"] = ("GPUSparseAssembler.__init__ on this mesh, timed on "
                                       "the CPU of the build container: " + ref["what"])
    except (OSError, KeyError, ValueError):
        pass
    return out


def _peaks():
    try:
        return json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except OSError:
        return {}


def other_configs(flush, parity_inputs):
    """The other workloads at their own shapes, each timed with CUDA events after warm-up:
    256 uneven meshes as one batch vs one mesh at a time; the gyroid coupled step with the
    learned guess trained on 300 steps and evaluated on 100 (N=48) against the
    previous-step guess; the gyroid step at N=96 with the learned guess, eager and
    CUDA-graph captured, against the plain FP64 step.  parity_inputs receives the gyroid
    run's start state and its GPU states after the first evaluated steps (compared with
    the oracle in the CPU leg)."""
    import torch
    out = {}

    def run(name, fn):
        try:
            out[name] = fn()
        except Exception as e:  # reported, not fatal for the headline line
            out[name] = {"error": repr(e)[:300]}

    def batch():
        from dissolve_tp.batch import MeshBatch, MeshBatchPlain, uneven_batch_inputs
        meshes, D, k = uneven_batch_inputs(256)
        mb = MeshBatch(meshes, D, k, 0.02, rtol=1e-8, inner_fp32=True)
        u0 = np.random.default_rng(2).uniform(0, 1, int(mb.vert_ptr[-1]))
        mb.set_state(u0)
        for _ in range(3):
            mb.step()
        ms = _event_ms(lambda: mb.step(sync=False), 3, flush, torch)
        r = mb.solver.result()
        tets = mb.n_cells
        cfg = mb.cg_config
        del mb
        pl = MeshBatchPlain(meshes, D, k, 0.02, rtol=1e-8)
        vp = np.concatenate([[0], np.cumsum([m_.n_verts for m_ in meshes])])
        pl.set_state(u0, vp)
        for _ in range(3):
            pl.step(sync=False)
        ms_p = _event_ms(lambda: pl.step(sync=False), 3, flush, torch)
        return {"workload": "256 Kuhn cubes, N ~ U{8..40}, one species each, rtol 1e-8",
                "tets": int(tets), "batch_ms_per_step": round(ms, 2),
                "batch_tets_per_s": round(tets / (ms * 1e-3), 1),
                "one_at_a_time_plain_fp64_ms_per_step": round(ms_p, 2),
                "speedup": round(ms_p / ms, 2), "max_lane_iterations": int(r["iterations"]),
                "converged": bool(r["converged"]), "cg_launch": cfg}

    def gyroid48():
        from dissolve_tp.coupled import GyroidStep, gyroid_inputs
        mesh, phi, coef, u0 = gyroid_inputs(48, 0.15)
        g = GyroidStep(mesh, phi, coef)
        g.set_state(u0)
        g.train_predictor(300, every=10, epochs=400)
        p = GyroidStep(mesh, phi, coef)
        p.tr.set_state(g.state(), g.tr.U_prev[:, :3].cpu().numpy())
        p.phi.copy_(g.phi)
        # the same start with the increment-history projection alone (no network)
        q = GyroidStep(mesh, phi, coef, guess="project")
        q.tr.set_state(g.state(), g.tr.U_prev[:, :3].cpu().numpy())
        q.phi.copy_(g.phi)
        # the state the evaluation starts from, for the oracle's run of its first steps
        n_or = 10
        start = {"coords": mesh.coords, "cells": mesh.cells, "phi": g.phi.cpu().numpy(),
                 "coef": coef, "U": g.state(), "steps": n_or, "dt": g.dt, "eps": g.eps,
                 "workload": f"gyroid 48^3, the first {n_or} evaluated steps after the 300 "
                             "training steps", "gpu": {}}
        res = {}
        for name, obj in (("learned", g), ("previous", p), ("projection_only", q)):
            its = []
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for i in range(100):
                its.append(obj.step()["iterations"])
                if i == n_or - 1 and name != "projection_only":
                    start["gpu"][name] = obj.state()
            e1.record()
            e1.synchronize()
            res[name] = {"ms_per_step": round(e0.elapsed_time(e1) / 100, 3),
                         "mean_iterations": round(float(np.mean(its)), 1)}
        parity_inputs["gyroid_48"] = start
        a, b_ = g.state(), p.state()
        res["rel_l2_learned_vs_previous"] = float(np.linalg.norm(a - b_) / np.linalg.norm(b_))
        res["workload"] = ("gyroid 48^3 (663,552 tets), k_ORR H_eps interface reaction, 300 "
                           "training steps, 100 evaluated steps, rtol 1e-8")
        return res

    def gyroid96():
        from dissolve_tp.coupled import GyroidStep, GyroidStepPlain, gyroid_inputs
        mesh, phi, coef, u0 = gyroid_inputs(96, 0.2)
        g = GyroidStep(mesh, phi, coef)
        g.set_state(u0)
        g.train_predictor(40, every=5, epochs=300)
        ms_e = _event_ms(lambda: g.step(sync=False), 10, flush, torch)
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(2):
                g.step(sync=False)
        torch.cuda.current_stream().wait_stream(s)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            g.step(sync=False)
        ms_g = _event_ms(graph.replay, 10, flush, torch)
        r = g.tr.solver.result()
        del graph
        p = GyroidStepPlain(mesh, phi, coef)
        p.set_state(u0)
        for _ in range(3):
            p.step(sync=False)
        ms_p = _event_ms(lambda: p.step(sync=False), 10, flush, torch)
        return {"workload": "gyroid 96^3 (5,308,416 tets), coupled step, rtol 1e-8",
                "fast_learned_eager_ms": round(ms_e, 2), "fast_learned_graph_ms": round(ms_g, 2),
                "plain_fp64_ms": round(ms_p, 2), "speedup_graph_vs_plain": round(ms_p / ms_g, 2),
                "iterations": int(r["iterations"]), "converged": bool(r["converged"])}

    run("uneven_batch_256", batch)
    run("gyroid_48_learned", gyroid48)
    run("gyroid_96_coupled", gyroid96)
    return out


# ------------------------------------------------------------------ CPU legs
def cpu_step_runner(m, coef, u0):
    """The reference CPU path restated (oracle): per species FP64 assembly in cell
    order + RHS + GMRES(50) right-preconditioned by block-Jacobi ILU(0), one block per
    host thread, from the previous step, to ||b - A x|| <= rtol ||b||."""
    from oracle import oracle as orc
    nt = orc.num_threads()
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, m.n_verts)
    state = {"U": np.array(u0, dtype=np.float64), "iters": []}
    alphas = [np.full(m.n_cells, k) for k in K_S]

    def step():
        its = []
        for s in range(3):
            A = orc.assemble(detJ, G, D_S[s] * coef, alphas[s], 1.0 / DT, 1, sm, ix.size)
            b = orc.assemble_rhs(m.cells, detJ, state["U"][:, s], None, 1.0 / DT, 1)
            x, it, st, _ = orc.gmres_bjacobi(ip, ix, A, b, state["U"][:, s], RTOL, nblocks=nt)
            state["U"][:, s] = x
            its.append(it)
        state["iters"].append(its)

    return step, nt, state


def cpu_baseline(m, coef, u0, sample_steps=PARITY_STEPS, gpu_states=None, gyroid=None):
    """The timed CPU sample (oracle port of the reference's CPU path: GMRES(50) + block
    Jacobi ILU(0) to rtol 1e-8, one block per host thread), then the parity of the GPU
    forms: the oracle's states after the same steps from u0 with every species solved by
    Jacobi-PCG to ORACLE_RTOL (standing in for the exact solution), against the GPU states
    after those steps; and the gyroid coupled step's first evaluated steps the same way."""
    step, nt, state = cpu_step_runner(m, coef, u0)
    t = time.perf_counter()
    for _ in range(sample_steps):
        step()
    dt = time.perf_counter() - t
    base = {"value": sample_steps / dt, "unit": "steps/s", "cores": nt, "kind": "port",
            "sample": f"{sample_steps} full 3-species steps from u_prev ~ U(0,1) "
                      f"(GMRES iterations per species {state['iters'][-1]})"}
    parity = {}
    if gpu_states:
        from oracle import oracle as orc
        t = time.perf_counter()
        want = orc.transport_steps(m.coords, m.cells, coef, D_S, K_S, DT, u0, PARITY_STEPS,
                                   rtol=ORACLE_RTOL)[-1]
        parity["headline"] = {
            "workload": f"{WORKLOAD}; {PARITY_STEPS} steps from u_prev",
            "oracle": f"per-species FP64 assembly + Jacobi-PCG to {ORACLE_RTOL:g} (CPU port, "
                      f"{nt} threads, {time.perf_counter() - t:.1f} s)",
            "bar": 1e-7}
        for name, U in gpu_states.items():
            parity["headline"][f"rel_l2_vs_oracle_{name}"] = float(
                np.linalg.norm(U - want) / np.linalg.norm(want))
    if gyroid:
        from oracle import oracle as orc
        g = gyroid
        t = time.perf_counter()
        want, _ = orc.gyroid_steps(g["coords"], g["cells"], g["phi"], g["coef"], g["U"],
                                   g["steps"], g["dt"], g["eps"], rtol=ORACLE_RTOL)
        parity["gyroid_48"] = {
            "workload": g["workload"],
            "oracle": f"coupled step, per-species FP64 assembly + Jacobi-PCG to "
                      f"{ORACLE_RTOL:g} (CPU port, {time.perf_counter() - t:.1f} s)",
            "bar": 1e-7}
        for name in ("learned", "previous"):
            U = g["gpu"][name]
            parity["gyroid_48"][f"rel_l2_vs_oracle_{name}"] = float(
                np.linalg.norm(U - want) / np.linalg.norm(want))
    return base, parity


def run_reference(args, rank, world):
    if rank != 0:
        return
    m, coef, u0 = make_inputs()
    step, nt, state = cpu_step_runner(m, coef, u0)
    for _ in range(args.warmup):
        step()
    t = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t
    v = args.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded, config shapes)",
            "config": {"workload": WORKLOAD, "n_tets": m.n_cells, "n_verts": m.n_verts,
                       "parallelism": "host threads"},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": nt, "kind": "port",
                             "sample": f"{args.steps} full 3-species steps after {args.warmup} "
                                       f"warm-up steps; GMRES(50) + block-Jacobi ILU(0), "
                                       f"{nt} blocks"},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "gmres_iterations": state["iters"][-1]}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--guess", default="learned", choices=["learned", "previous"])
    ap.add_argument("--train-steps", type=int, default=12)
    ap.add_argument("--host-loop", action="store_true",
                    help="iterate the CG from the host (plain graphs, one per iteration) "
                         "instead of the device-side while loop; for profilers that cannot "
                         "see kernels inside conditional graphs")
    ap.add_argument("--no-forms", dest="forms", action="store_false")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-sample-steps", type=int, default=3)
    ap.add_argument("--no-kernels", dest="kernels", action="store_false",
                    help="skip the assembly / RHS / apply bandwidth table")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="skip the multi-mesh batch and gyroid coupled-step workloads")
    ap.add_argument("--roofline-only", action="store_true",
                    help="W steps with the previous-step guess, then only the roofline solve "
                         "(the solve kernel's launch W + 1)")
    ap.add_argument("--kernels-only", action="store_true",
                    help="print only the assembly / RHS / apply bandwidth table (no step)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
