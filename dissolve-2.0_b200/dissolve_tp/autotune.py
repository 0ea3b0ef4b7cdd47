"""Project autotuner for the Krylov kernels' launch shape.

Times the inner SpMV+dot kernel (the per-iteration hot kernel) for each candidate
(threads per CSR row, block size, rows per reduction tile) on the real operator with
CUDA events (tp_cg_time_spmv), and keeps the fastest.  Results are cached per
(rows, columns, systems, precision) for the life of the process.
"""
from __future__ import annotations

import itertools

_CACHE: dict = {}

GROUPS = (1, 2, 4, 8)
BLOCKS = (128, 256)
TILE_PASSES = (1, 2)       # rows per tile = passes * block


def candidates():
    for g, b, k in itertools.product(GROUPS, BLOCKS, TILE_PASSES):
        yield {"group": g, "block": b, "rows_per_tile": k * b}


def tune_cg(op, inner_fp32: bool, reps: int = 10, verbose: bool = False) -> dict:
    from .krylov import CGSolver

    key = (op.n_rows, op.S, op.ld, op.n_systems, bool(inner_fp32))
    if key in _CACHE:
        return dict(_CACHE[key])
    best, best_ms, table = None, float("inf"), []
    for cand in candidates():
        sol = CGSolver(op, rtol=1e-8, max_it=1, inner_fp32=inner_fp32, **cand)
        sol.time_spmv(2)
        ms = sol.time_spmv(reps)
        sol.close()
        table.append((ms, cand))
        if ms < best_ms:
            best, best_ms = cand, ms
    if verbose:
        for ms, c in sorted(table, key=lambda t: t[0]):
            print(f"  {ms * 1e3:8.2f} us  {c}")
    _CACHE[key] = dict(best)
    _CACHE[key + ("table",)] = table
    return dict(best)


def last_table(op, inner_fp32: bool):
    return _CACHE.get((op.n_rows, op.S, op.ld, op.n_systems, bool(inner_fp32), "table"))
