"""Host logic of the launch-shape autotuner (dissolve_tp/autotune.py) on the CPU: every
candidate is timed, the fastest is kept, and the choice is cached per operator shape.
The timing call is a stand-in; the GPU timing itself is covered by the -m gpu tests."""
import types

import dissolve_tp.autotune as at
import dissolve_tp.krylov as kr


class _FakeSolver:
    made = []

    def __init__(self, op, rtol, max_it, inner_fp32, group, block, rows_per_tile):
        self.cand = {"group": group, "block": block, "rows_per_tile": rows_per_tile}
        _FakeSolver.made.append(self.cand)
        self.closed = False

    def time_spmv(self, reps):
        c = self.cand
        # fastest at group 4, block 256, two passes; ties impossible by construction
        return abs(c["group"] - 4) + (c["block"] != 256) * 0.5 + (c["rows_per_tile"] != 512) * 0.25

    def close(self):
        self.closed = True


def _op(n_rows=1000, S=3, ld=4, n_systems=1):
    return types.SimpleNamespace(n_rows=n_rows, S=S, ld=ld, n_systems=n_systems)


def test_candidates_cover_the_grid():
    cands = list(at.candidates())
    assert len(cands) == len(at.GROUPS) * len(at.BLOCKS) * len(at.TILE_PASSES)
    for c in cands:
        assert c["rows_per_tile"] % c["block"] == 0


def test_tune_picks_fastest_and_caches(monkeypatch):
    monkeypatch.setattr(kr, "CGSolver", _FakeSolver)
    monkeypatch.setattr(at, "_CACHE", {})
    _FakeSolver.made = []
    best = at.tune_cg(_op(), inner_fp32=True)
    assert best == {"group": 4, "block": 256, "rows_per_tile": 512}
    n_timed = len(_FakeSolver.made)
    assert n_timed == len(list(at.candidates()))
    # same shape: served from the cache, nothing re-timed; the caller's copy is its own
    best["group"] = 99
    assert at.tune_cg(_op(), inner_fp32=True)["group"] == 4
    assert len(_FakeSolver.made) == n_timed
    table = at.last_table(_op(), inner_fp32=True)
    assert len(table) == n_timed and min(t[0] for t in table) == 0.0
    # another precision or shape is tuned afresh
    at.tune_cg(_op(), inner_fp32=False)
    at.tune_cg(_op(n_systems=5), inner_fp32=True)
    assert len(_FakeSolver.made) == 3 * n_timed


class _FakeMesh:
    def __init__(self):
        self.n_verts, self.n_cells, self.nnz = 100, 500, 1400
        self.tile_rows = 64
        self.installed = []

    def set_tiles(self, rows):
        self.tile_rows = rows
        self.installed.append(rows)


def test_tune_tiles_picks_fastest_installs_and_caches(monkeypatch):
    """Every tile size is installed and timed; the fastest (median of the timed runs) stays
    installed and is cached per mesh shape."""
    import torch

    dm = _FakeMesh()
    cost = {0: 150.0, 32: 120.0, 64: 100.0, 128: 90.0}   # us per launch

    class _Ev:
        def __init__(self, enable_timing=True):
            self.t = 0.0

        def record(self):
            self.t = _Ev.clock
            _Ev.clock += cost[dm.tile_rows] * 1e-3 / 2   # half before, half after the launch

        def synchronize(self):
            pass

        def elapsed_time(self, other):
            return other.t - self.t

    _Ev.clock = 0.0
    monkeypatch.setattr(torch.cuda, "Event", _Ev)
    monkeypatch.setattr(at, "_CACHE", {})
    runs = []
    best = at.tune_tiles(dm, lambda: runs.append(dm.tile_rows), reps=5)
    assert best["rows_per_tile"] == 128 and dm.tile_rows == 128
    assert dm.installed[:len(at.TILE_ROWS)] == list(at.TILE_ROWS)
    assert len(runs) == len(at.TILE_ROWS) * 7          # 2 warm-up + 5 timed each
    table = at.last_tiles_table((dm.n_verts, dm.n_cells, dm.nnz))
    assert sorted(r for _, r in table) == sorted(at.TILE_ROWS)
    # cached: installed again without timing
    dm.set_tiles(0)
    n = len(runs)
    assert at.tune_tiles(dm, lambda: runs.append(dm.tile_rows))["rows_per_tile"] == 128
    assert dm.tile_rows == 128 and len(runs) == n
