"""Project autotuner for the launch shapes of the Krylov and assembly kernels.

tune_cg times the inner SpMV+dot kernel (the per-iteration hot kernel) for each
candidate (threads per CSR row, block size, rows per reduction tile) on the real operator
with CUDA events (tp_cg_time_spmv), and keeps the fastest.  tune_tiles times an assembly
launch for each row-tile size of the tiled kernels (rows per CTA; 0: the row walk, one
thread per row) and keeps the fastest.  Results are cached per shape for the life of the
process.
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


TILE_ROWS = (0, 32, 64, 128)


def tune_tiles(dm, run, reps: int = 10, key=None) -> dict:
    """Rows per tile of the tiled assembly for DeviceMesh `dm`: each candidate is installed
    (dm.set_tiles), run() -- one assembly launch on dm -- is warmed up twice and timed
    `reps` times with CUDA events; the fastest (median) is kept and left installed.
    Returns {"rows_per_tile": R, "us": median us}; the table of every candidate is in
    last_tiles_table(key).  key: the cache key (default: the mesh shape)."""
    import torch

    key = ("tiles",) + (tuple(key) if key is not None else (dm.n_verts, dm.n_cells, dm.nnz))
    if key in _CACHE:
        best = _CACHE[key]
        dm.set_tiles(best["rows_per_tile"])
        return dict(best)
    table = []
    for rows in TILE_ROWS:
        dm.set_tiles(rows)
        for _ in range(2):
            run()
        ts = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            run()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e3)
        table.append((sorted(ts)[len(ts) // 2], rows))
    us, rows = min(table)
    dm.set_tiles(rows)
    _CACHE[key] = {"rows_per_tile": rows, "us": round(us, 2)}
    _CACHE[key + ("table",)] = table
    return dict(_CACHE[key])


def last_tiles_table(key):
    return _CACHE.get(("tiles",) + tuple(key) + ("table",))
