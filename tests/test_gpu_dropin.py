"""The reference-facing modules on the GPU, called the way dissolve.py and solvers.py
call them (dissolve.py:780-954; solvers.py:206-372; ceed_operators.py:247-353).

Bars: solutions within 1e-9 relative L2 of the oracle's direct solve of the oracle CSR
(rtol 1e-10), under-relaxation exact to 1e-14, matrix-free apply within 1e-12 relative
(max-norm) of the oracle in both the intended and the reference-QFunction semantics."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(cuda_device):
    from dissolve_tp import fem
    from dissolve_tp.mesh import face_dofs, kuhn_cube
    m = kuhn_cube(12, 0.15, seed=0)
    mesh = fem.mesh_from(m)
    V = fem.FunctionSpace(mesh)
    return m, mesh, V, face_dofs(m, 0, "min")


def _oracle_step(m, De, alpha, inv_dt, u_old, f=None, bc=None, bc_value=0.0, lumped=1):
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, m.n_verts)
    De_c = orc.to_cell_avg(De, m.n_cells, m.n_verts, m.cells)
    al_c = orc.to_cell_avg(alpha, m.n_cells, m.n_verts, m.cells)
    A = orc.assemble(detJ, G, De_c, al_c, inv_dt, lumped, sm, ix.size, bc_dofs=bc, indptr=ip,
                     indices=ix)
    b = orc.assemble_rhs(m.cells, detJ, u_old, f, inv_dt, lumped, bc_dofs=bc, bc_value=bc_value)
    return orc.direct_solve(ip, ix, A, b)


def test_solve_transport_o2_like_call(case):
    """O2 call site: alpha field, Dirichlet dofs on de_field, bc_value, under_relax 0.3"""
    import solvers
    from dissolve_tp import fem
    m, mesh, V, bc = case
    rng = np.random.default_rng(3)
    De = fem.Function(V, np.exp(0.3 * rng.standard_normal(m.n_verts)))
    De._solver_inv_dt = 1.0 / 0.05
    De._solver_bc_dofs = bc
    u = fem.Function(V, rng.uniform(0, 1, m.n_verts))
    u_before = u.x.array.copy()
    alpha = rng.uniform(0, 2, m.n_verts)
    res = solvers.solve_transport("O2", None, None, u, rtol=1e-10, max_it=2000,
                                  under_relax=0.3, use_gpu=True, de_field=De,
                                  alpha_field=alpha, u_old=np.zeros(m.n_verts), bc_value=0.8)
    assert res["converged"] and res["iterations"] > 0 and res["time_s"] >= 0
    # with under_relax the pre-solve u is the RHS's u_old (solvers.py:246-247)
    x = _oracle_step(m, De.x.array, alpha, 20.0, u_before, bc=bc, bc_value=0.8)
    want = 0.3 * x + 0.7 * u_before
    assert np.linalg.norm(u.x.array - want) / np.linalg.norm(want) < 1e-9
    solvers._destroy_gpu_cache()


def test_solve_transport_oh_like_call_and_cache(case):
    """OH call site: source field, no Dirichlet; a second call reuses the cached solver"""
    import solvers
    from dissolve_tp import fem
    m, mesh, V, bc = case
    rng = np.random.default_rng(4)
    De = fem.Function(V, np.full(m.n_verts, 2.6))
    De._solver_inv_dt = 1.0 / 0.02
    u_old = rng.uniform(0, 1, m.n_verts)
    u = fem.Function(V, u_old.copy())
    f = rng.uniform(0, 0.1, m.n_verts)
    for _ in range(2):
        res = solvers.solve_transport("OH", None, None, u, rtol=1e-10, use_gpu=True,
                                      de_field=De, u_old=u_old, source_field=f)
        assert res["converged"]
        x = _oracle_step(m, De.x.array, np.zeros(m.n_verts), 50.0, u_old, f=f)
        assert np.linalg.norm(u.x.array - x) / np.linalg.norm(x) < 1e-9
        u_old = u.x.array.copy()
    assert len(solvers._GPU_ASM_CACHE) == 1
    solvers._destroy_gpu_cache()


def test_lump_mass_switch_through_shim(case):
    import gpu_assembler
    m, mesh, V, bc = case
    rng = np.random.default_rng(5)
    De, al = np.exp(rng.standard_normal(m.n_cells)), rng.uniform(0, 1, m.n_cells)
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, m.n_verts)
    old = gpu_assembler.LUMP_MASS
    try:
        for lm in (0, 1):
            gpu_assembler.LUMP_MASS = lm
            asm = gpu_assembler.GPUSparseAssembler(mesh, V)
            asm.assemble(De, 7.0, alpha=al)
            ref = orc.assemble(detJ, G, De, al, 7.0, lm, sm, ix.size)
            got = asm.d_data.cpu().numpy()
            assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    finally:
        gpu_assembler.LUMP_MASS = old


@pytest.mark.parametrize("legacy", [False, True])
def test_ceed_operator_apply(case, legacy):
    import torch

    import ceed_operators as co
    m, mesh, V, bc = case
    rng = np.random.default_rng(6)
    ceed, name = co.make_ceed(True)
    md = co.extract_ceed_mesh_data(mesh, V)
    De_v = np.exp(0.3 * rng.standard_normal(m.n_verts))
    op = co.CeedDiffusionMassOp(ceed, md, De_v, 20.0, legacy_stiffness=legacy)
    x = rng.standard_normal(m.n_verts)
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    De_c = orc.to_cell_avg(De_v, m.n_cells, m.n_verts, m.cells)
    ref = orc.matfree_apply(m.cells, detJ, G, De_c, x, 20.0, lumped=False, legacy=legacy)
    y = op.apply(x)
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()
    # device in / device out, and update_coeffs
    op.update_coeffs(2.0 * De_v, 10.0)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    op.apply(xd, yd)
    ref2 = orc.matfree_apply(m.cells, detJ, G, 2.0 * De_c, x, 10.0, legacy=legacy)
    assert np.abs(yd.cpu().numpy() - ref2).max() <= 1e-12 * np.abs(ref2).max()


def test_compute_geometric_factors_layout(case):
    import ceed_operators as co
    m, mesh, V, bc = case
    md = co.extract_ceed_mesh_data(mesh, V)
    geom = co.compute_geometric_factors(md["coords"], md["elem_nodes"], md["q_wts"])
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    g = geom.reshape(m.n_cells, 4, 10)
    assert np.allclose(g[:, 2, 0], md["q_wts"][2] * detJ, rtol=1e-13)
    assert np.allclose(g[:, 1, 1:], G, rtol=1e-11, atol=1e-14 * np.abs(G).max())
