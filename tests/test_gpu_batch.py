"""Multi-mesh batch on the GPU: every mesh a lane of one block-diagonal solve.

Bars: every lane converged; each mesh's solution within 1e-7 relative L2 (FP32 inner,
rtol 1e-8) / 1e-9 (FP64, rtol 1e-10) of the oracle's direct solve of that mesh alone; the
one-at-a-time plain FP64 form agrees with the batch within 1e-7."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _direct(m, D, k, inv_dt, u0):
    detJ, G, _ = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, m.n_verts)
    A = orc.assemble(detJ, G, np.full(m.n_cells, D), np.full(m.n_cells, k), inv_dt, 1, sm,
                     ix.size)
    b = orc.assemble_rhs(m.cells, detJ, u0, None, inv_dt, 1)
    return orc.direct_solve(ip, ix, A, b)


@pytest.mark.parametrize("fp32,rtol,bar", [(True, 1e-8, 1e-7), (False, 1e-10, 1e-9)])
def test_batch_lanes_match_direct_solves(cuda_device, fp32, rtol, bar):
    from dissolve_tp.batch import MeshBatch, uneven_batch_inputs
    meshes, D, k = uneven_batch_inputs(12, 3, 10, seed=5)
    mb = MeshBatch(meshes, D, k, 0.02, rtol=rtol, inner_fp32=fp32)
    vp = mb.vert_ptr
    u0 = np.random.default_rng(1).uniform(0, 1, int(vp[-1]))
    mb.set_state(u0)
    res = mb.step()
    assert res["converged"] and len(res["lane_iterations"]) == 12
    x = mb.state()
    for i, m in enumerate(meshes):
        sl = slice(vp[i], vp[i + 1])
        xd = _direct(m, D[i], k[i], 50.0, u0[sl])
        assert np.linalg.norm(x[sl] - xd) / np.linalg.norm(xd) < bar, i


def test_batch_matches_one_at_a_time_plain(cuda_device):
    from dissolve_tp.batch import MeshBatch, MeshBatchPlain, uneven_batch_inputs
    meshes, D, k = uneven_batch_inputs(8, 4, 12, seed=7)
    mb = MeshBatch(meshes, D, k, 0.02, rtol=1e-8)
    pl = MeshBatchPlain(meshes, D, k, 0.02, rtol=1e-8)
    u0 = np.random.default_rng(2).uniform(0, 1, int(mb.vert_ptr[-1]))
    mb.set_state(u0)
    pl.set_state(u0, mb.vert_ptr)
    for _ in range(3):
        r1 = mb.step()
        r2 = pl.step()
        assert r1["converged"] and all(r["converged"] for r in r2)
    a, b = mb.state(), pl.state()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-7
