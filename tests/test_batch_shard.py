"""Multi-mesh batch host logic: LPT sharding and the replica plumbing, on CPU (gloo).

Two ranks each solve their shard of a batch of small meshes with the oracle (CPU) and
rank 0 gathers; the merged result must equal the single-process result exactly, and the
job time is the max over ranks."""
import os
import socket

import numpy as np
import pytest

from oracle import oracle as orc


def test_lpt_partition_properties():
    from dissolve_tp.batch import lpt_partition
    from dissolve_tp.replicas import imbalance
    rng = np.random.default_rng(0)
    w = rng.integers(8, 41, 256) ** 3 * 6
    for k in (1, 2, 3, 4, 8):
        parts = lpt_partition(w, k)
        allidx = sorted(i for p in parts for i in p)
        assert allidx == list(range(256))
        assert parts == lpt_partition(w, k)  # deterministic
        # LPT bound: max load <= 4/3 OPT; with many items it is close to the mean
        assert imbalance(w, parts) < 1.05
    # more parts than items: empty parts allowed, nothing lost
    parts = lpt_partition([5, 3], 4)
    assert sorted(i for p in parts for i in p) == [0, 1]


def _solve_mesh(i):
    from dissolve_tp.mesh import kuhn_cube
    n = 3 + i % 4
    m = kuhn_cube(n, 0.2, seed=100 + i)
    detJ, G, _ = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, m.n_verts)
    D, k = 0.5 + 0.25 * i, 0.1 * (i % 3)
    A = orc.assemble(detJ, G, np.full(m.n_cells, D), np.full(m.n_cells, k), 50.0, 1, sm,
                     ix.size)
    u0 = np.random.default_rng(i).uniform(0, 1, m.n_verts)
    b = orc.assemble_rhs(m.cells, detJ, u0, None, 50.0, 1)
    return float(np.sum(orc.direct_solve(ip, ix, A, b))), m.n_cells


def _worker(rank, world, port, n_items, out):
    import torch.distributed as dist

    from dissolve_tp.replicas import gather_results, max_over_ranks, shard_of
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        weights = [6 * (3 + i % 4) ** 3 for i in range(n_items)]
        mine = shard_of(weights, rank, world)
        local = {i: _solve_mesh(i)[0] for i in mine}
        t = max_over_ranks(float(rank + 1))
        res = gather_results(local, n_items)
        if rank == 0:
            out.put((res, t))
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_match_single_process():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    n_items = 10
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n_items, q)) for r in range(2)]
    for p in procs:
        p.start()
    res, t = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    single = [_solve_mesh(i)[0] for i in range(n_items)]
    assert res == single
    assert t == 2.0


def test_shard_of_rejects_bad_rank():
    from dissolve_tp.replicas import shard_of
    with pytest.raises(ValueError):
        shard_of([1, 2, 3], 2, 2)
