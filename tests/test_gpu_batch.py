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


@pytest.mark.gpu
@pytest.mark.parametrize("with_alpha_bc", [False, True])
def test_fused_stiffness_diag_equals_separate_calls(cuda_device, with_alpha_bc):
    """tp_assemble_stiffness_diag = tp_assemble_csr(STIFF) + tp_lumped_diag + the FP32 SELL
    scatter, bit for bit."""
    import ctypes

    import torch

    from dissolve_tp import _lib
    from dissolve_tp.assembler import DeviceMesh
    from dissolve_tp.device import ptr, stream_handle
    from dissolve_tp.krylov import SellPattern
    from dissolve_tp.mesh import face_dofs, kuhn_cube
    m = kuhn_cube(10, 0.2, seed=4)
    rng = np.random.default_rng(9)
    dm = DeviceMesh(m.coords, m.cells)
    dev = torch.device("cuda")
    S, ld, nnz, V = 3, 4, dm.nnz, dm.n_verts
    De = torch.from_numpy(np.exp(0.3 * rng.standard_normal(m.n_cells))).to(dev)
    alpha = bc = None
    if with_alpha_bc:
        alpha = torch.zeros((m.n_cells, ld), dtype=torch.float64, device=dev)
        alpha[:, :S] = torch.from_numpy(rng.uniform(0, 2, (m.n_cells, S)))
        bc = dm.bc_mask(face_dofs(m, 1, "max"))
    shift = (ctypes.c_double * 4)(50.5, 50.0, 50.2, 0.0)
    st = stream_handle()
    K64a, K64b = (torch.zeros(nnz, dtype=torch.float64, device=dev) for _ in range(2))
    K32a, K32b = (torch.zeros(nnz, dtype=torch.float32, device=dev) for _ in range(2))
    D64a, D64b = (torch.zeros((V, ld), dtype=torch.float64, device=dev) for _ in range(2))
    D32a, D32b = (torch.zeros((V, ld), dtype=torch.float32, device=dev) for _ in range(2))
    sell = SellPattern(dm.indptr, dm.indices[:nnz])
    Sa, Sb = sell.values(torch.float32), sell.values(torch.float32)
    _lib.call("tp_assemble_csr", ctypes.byref(dm.tpm), ptr(De), None, 0.0, 1, _lib.TP_ASM_STIFF,
              ptr(bc), ptr(K64a), ptr(K32a), st)
    _lib.call("tp_lumped_diag", ctypes.byref(dm.tpm), S, ld, ptr(alpha), shift, ptr(bc),
              ptr(D64a), ptr(D32a), st)
    sell.scatter(K64a, out32=Sa)
    Sb.fill_(7.0)  # every SELL entry, padding included, must be written
    _lib.call("tp_assemble_stiffness_diag", ctypes.byref(dm.tpm), ptr(De), S, ld, ptr(alpha),
              shift, ptr(bc), ptr(K64b), ptr(K32b), ptr(sell.slice_ptr), ptr(Sb), ptr(D64b),
              ptr(D32b), st)
    for a, b in ((K64a, K64b), (K32a, K32b), (D64a, D64b), (D32a, D32b), (Sa, Sb)):
        assert torch.equal(a, b)


@pytest.mark.gpu
def test_lumped_rhs_matches_cell_order_rhs(cuda_device):
    """tp_lumped_rhs (mass per vertex x (u/dt + f)) against tp_assemble_rhs (cell-order sums),
    with a source and Dirichlet rows: equal to rounding."""
    import ctypes

    import torch

    from dissolve_tp import _lib
    from dissolve_tp.assembler import DeviceMesh
    from dissolve_tp.device import ptr, stream_handle
    from dissolve_tp.mesh import face_dofs, kuhn_cube
    m = kuhn_cube(9, 0.2, seed=2)
    dm = DeviceMesh(m.coords, m.cells)
    rng = np.random.default_rng(4)
    V, S, ld = dm.n_verts, 3, 4
    dev = torch.device("cuda")
    U = torch.zeros((V, ld), dtype=torch.float64, device=dev)
    F = torch.zeros_like(U)
    U[:, :S] = torch.from_numpy(rng.uniform(0, 1, (V, S)))
    F[:, :S] = torch.from_numpy(rng.normal(0, 1, (V, S)))
    bc = torch.from_numpy(face_dofs(m, 2, "min")).to(dev)
    bcv = (ctypes.c_double * 4)(1.0, 0.5, 0.25, 0.0)
    st = stream_handle()
    mass = torch.zeros(V, dtype=torch.float64, device=dev)
    _lib.call("tp_lumped_diag", ctypes.byref(dm.tpm), 1, 1, None, (ctypes.c_double * 4)(1.0), None,
              ptr(mass), None, st)
    b1, b2 = torch.zeros_like(U), torch.full_like(U, 7.0)
    _lib.call("tp_assemble_rhs", ctypes.byref(dm.tpm), S, ld, ptr(U), ptr(F), 50.0, 1,
              int(bc.numel()), ptr(bc), bcv, ptr(b1), st)
    _lib.call("tp_lumped_rhs", V, S, ld, ptr(mass), ptr(U), ptr(F), 50.0, int(bc.numel()),
              ptr(bc), bcv, ptr(b2), st)
    assert (b1 - b2).abs().max().item() <= 1e-14 * b1.abs().max().item()
    assert torch.equal(b1[bc.long()], b2[bc.long()])
    assert torch.equal(b2[:, S:], torch.zeros_like(b2[:, S:]))
