"""GPU parity: the CUDA path against the reference's golden vectors and the CPU oracle.

Bars: integer/index arrays (pattern, scatter map) bit-exact; assembly / RHS / nodal
gradient bit-exact when fed the reference's own geometry (the kernels replay the
reference's operation order, cell by cell); with GPU-computed geometry FP64 values
within 1e-12 relative (max-norm, relative to the largest entry); FP32 values within
1e-6 relative; solves within the stated relative L2 of the direct FP64 solution.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import golden_cases, load_golden
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

CASES = golden_cases()


@pytest.fixture(scope="module")
def tp(cuda_device):
    import torch  # noqa: F401

    from dissolve_tp import _lib, assembler, krylov
    return _lib, assembler, krylov


@pytest.fixture(params=CASES, ids=[os.path.basename(c)[:-4] for c in CASES], scope="module")
def g(request):
    return load_golden(request.param)


def _np(t):
    return t.detach().cpu().numpy()


def relmax(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_pattern_bit_exact(tp, g):
    _, A, _ = tp
    dm = A.DeviceMesh(g["coords"], g["cells"])
    assert dm.nnz == g["indices"].size
    assert np.array_equal(_np(dm.indptr), g["indptr"])
    assert np.array_equal(_np(dm.indices)[: dm.nnz], g["indices"])
    assert np.array_equal(_np(dm.scatter_map), g["scatter_map"])


def test_geometry_close(tp, g):
    _, A, _ = tp
    dm = A.DeviceMesh(g["coords"], g["cells"])
    detJ, G, JT = (_np(t) for t in dm.ref_geometry)
    assert relmax(detJ, g["detJ"]) < 1e-13
    assert relmax(G, g["Gflat"]) < 1e-12
    assert relmax(JT, g["JinvT"]) < 1e-12


@pytest.mark.parametrize("lumped", [1, 0])
def test_assembly_bit_exact_on_reference_geometry(tp, g, lumped, monkeypatch):
    _, A, _ = tp
    monkeypatch.setattr(A, "LUMP_MASS", lumped)
    tag = "lumped" if lumped else "cons"
    asm = A.GPUSparseAssembler((g["coords"], g["cells"]))
    asm._dm.use_reference_geometry(g["detJ"], g["Gflat"])
    asm.assemble(g["De_vert"], float(g["inv_dt"]), alpha=g["alpha_cell"])
    assert np.array_equal(_np(asm.d_data), g[f"A_{tag}"])
    asm.assemble(g["De_cell"], float(g["inv_dt"]), alpha=g["alpha_vert"], bc_dofs=g["bc_dofs"])
    assert np.array_equal(_np(asm.d_data), g[f"A_{tag}_bc"])
    asm.assemble(g["De_cell"], float(g["inv_dt"]))
    assert np.array_equal(_np(asm.d_data), g[f"A_{tag}_noalpha"])
    b = asm.assemble_rhs(g["u_old"], float(g["inv_dt"]), f=g["f_vert"])
    assert np.array_equal(_np(b), g[f"b_{tag}"])
    b = asm.assemble_rhs(g["u_old"], float(g["inv_dt"]), f=g["f_vert"], bc_dofs=g["bc_dofs"],
                         bc_value=float(g["bc_value"]))
    assert np.array_equal(_np(b), g[f"b_{tag}_bc"])
    b = asm.assemble_rhs(g["u_old"], float(g["inv_dt"]))
    assert np.array_equal(_np(b), g[f"b_{tag}_nof"])
    # borrower shares geometry and pattern (gpu_assembler.py:346-367)
    asm2 = A.GPUSparseAssembler(ref_asm=asm)
    asm2.assemble(g["De_cell"], float(g["inv_dt"]), alpha=g["alpha_cell"], bc_dofs=g["bc_dofs"])
    if lumped:
        assert np.array_equal(_np(asm2.d_data), g["A_lumped_bc_borrow"])


def test_assembly_on_gpu_geometry(tp, g):
    _, A, _ = tp
    asm = A.GPUSparseAssembler((g["coords"], g["cells"]))
    asm.assemble(g["De_vert"], float(g["inv_dt"]), alpha=g["alpha_cell"])
    assert relmax(_np(asm.d_data), g["A_lumped"]) < 1e-12
    assert relmax(_np(asm.nodal_gradient(g["u_old"])), g["grad_u"]) < 1e-12
    v = asm.scaffold_volume(g["phi"], float(g["eps"]))
    assert abs(v - float(g["scaffold_volume"])) <= 1e-13 * abs(float(g["scaffold_volume"]))


def test_nodal_gradient_bit_exact_with_reference_jinvt(tp, g):
    _lib, A, _ = tp
    import torch

    from dissolve_tp.device import ptr, stream_handle
    dm = A.DeviceMesh(g["coords"], g["cells"])
    dm.use_reference_geometry(g["detJ"], g["Gflat"])
    JT = torch.from_numpy(g["JinvT"]).cuda()
    for key, u in (("grad_u", g["u_old"]), ("grad_phi", g["phi"])):
        d = torch.from_numpy(np.ascontiguousarray(u)).cuda()
        out = torch.empty((dm.n_verts, 3), dtype=torch.float64, device="cuda")
        _lib.call("tp_nodal_gradient", ctypes.byref(dm.tpm), ptr(JT), ptr(d), ptr(out),
                  stream_handle())
        assert np.array_equal(_np(out), g[key])


def test_length_mismatch_errors(tp, g):
    _, A, _ = tp
    asm = A.GPUSparseAssembler((g["coords"], g["cells"]))
    nv = g["coords"].shape[0]
    with pytest.raises(ValueError) as e:
        asm.assemble(np.ones(nv + 1), 1.0)
    assert str(e.value) == str(g["err_len"])
    with pytest.raises(ValueError):
        asm.assemble_rhs(np.ones(nv + 2), 1.0)
    with pytest.raises(ValueError):
        asm.assemble_rhs(np.ones(nv), 1.0, f=np.ones(nv + 3))


# --------------------------------------------------------------------- larger meshes
@pytest.fixture(scope="module")
def mesh16():
    from dissolve_tp.mesh import kuhn_cube
    return kuhn_cube(16, 0.15, seed=0)


def test_setup_and_assembly_n16(tp, mesh16):
    _, A, _ = tp
    m = mesh16
    asm = A.GPUSparseAssembler(m)
    ip, ix, sm = orc.csr_pattern(m.cells, m.n_verts)
    assert np.array_equal(_np(asm.d_indptr), ip) and np.array_equal(_np(asm.d_indices), ix)
    assert np.array_equal(_np(asm.d_scatter_map), sm)
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    rng = np.random.default_rng(1)
    De = np.exp(0.3 * rng.standard_normal(m.n_cells))
    al = rng.uniform(0, 1, m.n_cells)
    for lumped in (1, 0):
        A.LUMP_MASS = lumped
        asm.assemble(De, 20.0, alpha=al)
        ref = orc.assemble(detJ, G, De, al, 20.0, lumped, sm, ix.size)
        assert relmax(_np(asm.d_data), ref) < 1e-12
    A.LUMP_MASS = 1


def test_fp32_values_are_rounded_fp64(tp, mesh16):
    _lib, A, _ = tp
    import torch

    from dissolve_tp.device import ptr, stream_handle
    dm = A.DeviceMesh(mesh16.coords, mesh16.cells)
    De = torch.ones(dm.n_cells, dtype=torch.float64, device="cuda")
    v64 = torch.empty(dm.nnz, dtype=torch.float64, device="cuda")
    v32 = torch.empty(dm.nnz, dtype=torch.float32, device="cuda")
    _lib.call("tp_assemble_csr", ctypes.byref(dm.tpm), ptr(De), None, 20.0, 1, _lib.TP_ASM_STIFF,
              None, ptr(v64), ptr(v32), stream_handle())
    assert torch.equal(v64.float(), v32)


def test_matfree_apply_matches_oracle(tp, mesh16):
    _lib, A, _ = tp
    import torch

    from dissolve_tp.device import ptr, stream_handle
    m = mesh16
    dm = A.DeviceMesh(m.coords, m.cells)
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    rng = np.random.default_rng(7)
    De = np.exp(0.3 * rng.standard_normal(m.n_cells))
    al = rng.uniform(0, 1, m.n_cells)
    for S, ld in ((1, 1), (3, 4)):
        x = rng.standard_normal((m.n_verts, S))
        ds = np.array([1.0, 1.0, 2.6, 1.0])[:S]
        sh = np.array([0.5, 0.0, 0.2, 0.0])[:S]
        for lumped in (0, 1):
            for legacy in (0, 1):
                ref = orc.matfree_apply(m.cells, detJ, G, De, x, 50.0, alpha_cell=al,
                                        lumped=lumped, legacy=legacy, diff_scale=ds, shift=sh)
                xd = np.zeros((m.n_verts, ld))
                xd[:, :S] = x
                for fp32, tol in ((0, 1e-12), (1, 2e-5)):
                    dt = torch.float32 if fp32 else torch.float64
                    X = torch.from_numpy(xd).to("cuda", dt)
                    Y = torch.empty_like(X)
                    Dd = torch.from_numpy(De).cuda()
                    Ad = torch.from_numpy(al).cuda()
                    dsc = (ctypes.c_double * 4)(*ds)
                    shf = (ctypes.c_double * 4)(*sh)
                    _lib.call("tp_matfree_apply", ctypes.byref(dm.tpm), S, ld, fp32, ptr(Dd),
                              ptr(Ad), dsc, shf, 50.0, lumped, legacy, ptr(X), ptr(Y),
                              stream_handle())
                    got = _np(Y.double())[:, :S]
                    assert relmax(got, ref) < tol, (S, lumped, legacy, fp32)


# --------------------------------------------------------------------- Krylov
def _config1(A):
    """small plain-method case: 16^3 cube, D=1, k=0.5, dt=0.05, u=1 on x=0."""
    from dissolve_tp.mesh import face_dofs, kuhn_cube
    m = kuhn_cube(16, 0.15, seed=0)
    bc = face_dofs(m, 0, "min")
    u0 = np.random.default_rng(2).uniform(0, 1, m.n_verts)
    asm = A.GPUSparseAssembler(m)
    asm.assemble(np.ones(m.n_cells), 20.0, alpha=np.full(m.n_cells, 0.5), bc_dofs=bc)
    b = asm.assemble_rhs(u0, 20.0, bc_dofs=bc, bc_value=1.0)
    return m, bc, u0, asm, b


@pytest.mark.parametrize("graph_loop", [0, 1])
def test_cg_fp64_config1(tp, graph_loop):
    _, A, K = tp
    m, bc, u0, asm, b = _config1(A)
    mask = asm._dm.bc_mask(bc)
    op = K.CsrOperator(asm.d_indptr, asm.d_indices, asm.d_data, bc_mask=mask)
    sol = K.CGSolver(op, rtol=1e-10, max_it=2000, use_graph_loop=graph_loop)
    sol.b[:, 0].copy_(b)
    sol.x[:, 0].copy_(__import__("torch").from_numpy(u0))
    res = sol.solve()
    assert res["converged"], res
    x = _np(sol.x[:, 0])
    ip, ix, A_ = (t for t in asm.mat.getValuesCSR())
    xd = orc.direct_solve(ip, ix, A_, _np(b))
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-9
    assert res["rnorm"][0] <= 1e-10 * res["bnorm"][0]
    x0 = u0.copy()
    x0[bc] = 1.0
    xo, it_o, st_o, _ = orc.pcg_jacobi(ip, ix, A_, _np(b), x0, 1e-10, bc_dofs=bc)
    assert st_o == 0 and abs(res["iterations"] - it_o) <= 3, (res["iterations"], it_o)


def test_gpu_manufactured_solution_converges_second_order(tp):
    """The drop-in assembler (c M + K, Dirichlet rows), its RHS (M f) and the persistent CG
    on the manufactured problem u = sin(pi x) sin(pi y) sin(pi z), -div grad u + c u = f:
    the mass-weighted nodal error falls by about 4x per halving of h, and each solution
    matches the oracle's direct solve of the oracle's system."""
    _, A, K = tp
    import torch

    from test_oracle_golden import _manufactured_case
    c = 2.0
    errs = []
    for n in (8, 16, 32):
        m, ue, f, bnd = _manufactured_case(n, c)
        asm = A.GPUSparseAssembler(m)
        asm.assemble(np.ones(m.n_cells), c, bc_dofs=bnd)
        b = asm.assemble_rhs(np.zeros(m.n_verts), c, f=f, bc_dofs=bnd, bc_value=0.0)
        mask = asm._dm.bc_mask(bnd)
        op = K.CsrOperator(asm.d_indptr, asm.d_indices, asm.d_data, bc_mask=mask)
        sol = K.CGSolver(op, rtol=1e-12, max_it=5000)
        sol.b[:, 0].copy_(b)
        sol.x[:, 0].zero_()
        res = sol.solve()
        assert res["converged"], res
        uh = _np(sol.x[:, 0])
        if n <= 16:
            ip, ix, A_ = (t for t in asm.mat.getValuesCSR())
            ud = orc.direct_solve(ip, ix, A_, _np(b))
            assert np.linalg.norm(uh - ud) / np.linalg.norm(ud) < 1e-10
        detJ, _, _ = orc.geometry(m.coords, m.cells)
        ml = orc.lumped_mass(m.cells, detJ, m.n_verts)
        errs.append(float(np.sqrt(np.sum(ml * (uh - ue) ** 2))))
        del sol, op, asm
        torch.cuda.synchronize()
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(len(errs) - 1)]
    # the coarsest pair is pre-asymptotic; the finest is second order
    assert all(1.6 < r < 2.3 for r in rates) and 1.85 < rates[-1] < 2.3, (errs, rates)


def test_cg_mixed_and_multi_rhs(tp):
    _, A, K = tp
    import torch

    from dissolve_tp.mesh import kuhn_cube
    m = kuhn_cube(16, 0.2, seed=0)
    asm = A.GPUSparseAssembler(m)
    rng = np.random.default_rng(1)
    xi = np.exp(0.3 * rng.standard_normal(m.n_cells))
    Ds, ks, inv_dt = [1.0, 1.0, 2.6], [0.5, 0.0, 0.2], 50.0
    dm = asm._dm
    from dissolve_tp.device import ptr, stream_handle
    from dissolve_tp import _lib
    K64 = torch.empty(dm.nnz, dtype=torch.float64, device="cuda")
    K32 = torch.empty(dm.nnz, dtype=torch.float32, device="cuda")
    _lib.call("tp_assemble_csr", ctypes.byref(dm.tpm), ptr(torch.from_numpy(xi).cuda()), None,
              0.0, 1, _lib.TP_ASM_STIFF, None, ptr(K64), ptr(K32), stream_handle())
    D64 = torch.empty((m.n_verts, 4), dtype=torch.float64, device="cuda")
    D32 = torch.empty((m.n_verts, 4), dtype=torch.float32, device="cuda")
    shift = (ctypes.c_double * 4)(*[inv_dt + k for k in ks], 0.0)
    _lib.call("tp_lumped_diag", ctypes.byref(dm.tpm), 3, 4, None, shift, None, ptr(D64), ptr(D32),
              stream_handle())
    u0 = rng.uniform(0, 1, (m.n_verts, 3))
    U = torch.zeros((m.n_verts, 4), dtype=torch.float64, device="cuda")
    U[:, :3] = torch.from_numpy(u0)
    B = torch.zeros_like(U)
    _lib.call("tp_assemble_rhs", ctypes.byref(dm.tpm), 3, 4, ptr(U), None, inv_dt, 1, 0, None,
              None, ptr(B), stream_handle())
    # oracle: per species FP64 assembled matrix and direct solve
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, m.n_verts)
    xref = []
    for s in range(3):
        As = orc.assemble(detJ, G, Ds[s] * xi, np.full(m.n_cells, ks[s]), inv_dt, 1, sm, ix.size)
        bs = orc.assemble_rhs(m.cells, detJ, u0[:, s], None, inv_dt, 1)
        assert relmax(_np(B[:, s]), bs) < 1e-13
        xref.append(orc.direct_solve(ip, ix, As, bs))
    for fp32 in (0, 1):
        op = K.CsrOperator(dm.indptr, dm.indices, K64, K32=K32 if fp32 else None, diag64=D64,
                           diag32=D32 if fp32 else None, dscale=Ds, S=3)
        sol = K.CGSolver(op, rtol=1e-8, max_it=2000, inner_fp32=bool(fp32))
        sol.b.copy_(B)
        sol.x.copy_(U)
        res = sol.solve()
        assert res["converged"], res
        for s in range(3):
            x = _np(sol.x[:, s])
            err = np.linalg.norm(x - xref[s]) / np.linalg.norm(xref[s])
            assert err < 1e-7, (fp32, s, err)
            assert res["rnorm"][s] <= 1e-8 * res["bnorm"][s]
        assert np.all(_np(sol.x[:, 3]) == 0.0)


def test_cg_batched_systems(tp):
    """independent meshes as one block-diagonal system: each lane matches its own solve"""
    _, A, K = tp
    import torch

    from dissolve_tp.mesh import concat_meshes, kuhn_cube
    meshes = [kuhn_cube(n, 0.2, seed=10 + n) for n in (4, 9, 6)]
    U, vp, cp = concat_meshes(meshes)
    asm = A.GPUSparseAssembler(U)
    rng = np.random.default_rng(3)
    D = np.repeat([0.3, 2.0, 7.0], [m.n_cells for m in meshes])
    k = np.repeat([0.1, 0.9, 0.5], [m.n_cells for m in meshes])
    asm.assemble(D, 50.0, alpha=k)
    u0 = rng.uniform(0, 1, U.n_verts)
    b = asm.assemble_rhs(u0, 50.0)
    op = K.CsrOperator(asm.d_indptr, asm.d_indices, asm.d_data, n_systems=3, sys_row_ptr=vp)
    sol = K.CGSolver(op, rtol=[1e-8, 1e-9, 1e-10], max_it=2000, rows_per_tile=256)
    sol.b[:, 0].copy_(b)
    sol.x[:, 0].copy_(torch.from_numpy(u0))
    res = sol.solve()
    assert res["converged"] and len(res["lane_iterations"]) == 3
    ip, ix, A_ = asm.mat.getValuesCSR()
    xd = orc.direct_solve(ip, ix, A_, _np(b))
    x = _np(sol.x[:, 0])
    for i, rt in enumerate((1e-8, 1e-9, 1e-10)):
        sl = slice(vp[i], vp[i + 1])
        assert res["rnorm"][i] <= rt * res["bnorm"][i]
        assert np.linalg.norm(x[sl] - xd[sl]) / np.linalg.norm(xd[sl]) < 100 * rt


def test_cg_reports_breakdown_without_raising(tp):
    _, A, K = tp
    import torch
    m, bc, u0, asm, b = _config1(A)
    neg = -asm.d_data  # negative definite: p.Ap < 0 at the first step
    op = K.CsrOperator(asm.d_indptr, asm.d_indices, neg)
    sol = K.CGSolver(op, rtol=1e-10, max_it=50)
    sol.b[:, 0].copy_(b)
    sol.x[:, 0].zero_()
    res = sol.solve()
    assert not res["converged"] and res["status"] == 7
    assert torch.isfinite(sol.x).all()


def test_bad_mesh_inputs_raise(tp):
    _, A, _ = tp
    coords = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)
    with pytest.raises(ValueError, match="index"):
        A.DeviceMesh(coords, np.array([[0, 1, 2, 7]], dtype=np.int32))
    flat = coords.copy()
    flat[3] = [1, 1, 0]
    with pytest.raises(ValueError, match="degenerate"):
        A.DeviceMesh(flat, np.array([[0, 1, 2, 3]], dtype=np.int32))
    asm = A.GPUSparseAssembler((coords, np.array([[0, 1, 2, 3]], dtype=np.int32)))
    with pytest.raises(ValueError, match="index"):
        asm.assemble(np.ones(1), 1.0, bc_dofs=np.array([9], dtype=np.int32))


def test_zero_size_inputs_are_no_ops(tp):
    """Entry points given zero rows / cells / values return TP_OK and write nothing (a
    sentinel buffer stays as it was)."""
    _lib, _, _ = tp
    import torch

    from dissolve_tp.device import ptr, stream_handle
    st = stream_handle()
    a = torch.full((8,), 7.0, dtype=torch.float64, device="cuda")
    b = torch.full((8,), 7.0, dtype=torch.float64, device="cuda")
    c = torch.full((8,), 7.0, dtype=torch.float64, device="cuda")
    d = torch.full((8,), 7.0, dtype=torch.float64, device="cuda")
    cells = torch.zeros((2, 4), dtype=torch.int32, device="cuda")
    one = (ctypes.c_double * 4)(1.0, 1.0, 1.0, 1.0)
    calls = [
        ("tp_cell_average", 0, ptr(cells), ptr(a), ptr(b), st),
        ("tp_axpby", 0, 2.0, ptr(a), 3.0, ptr(b), st),
        ("tp_advance_state", 0, ptr(a), ptr(b), ptr(c), ptr(d), st),
        ("tp_pack_columns", 0, 3, 4, ptr(a), ptr(b), st),
        ("tp_unpack_columns", 0, 3, 4, ptr(a), ptr(b), st),
        ("tp_o2_alpha", 0, ptr(a), ptr(b), 0.1, 2.0, ptr(c), st),
        ("tp_lumped_rhs", 0, 3, 4, ptr(a), ptr(b), None, 50.0, 0, None, one, ptr(c), st),
    ]
    for name, *args in calls:
        assert _lib.call(name, *args) == 0, name
    torch.cuda.synchronize()
    for t in (a, b, c, d):
        assert torch.all(t == 7.0)
