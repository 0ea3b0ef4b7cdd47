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
