"""The matrix-free Krylov solve (tp_mfcg_solve, the GPU form of the reference's MatShell
branch numerics/solvers.py:172-203, 375-404) against the oracle's direct solve of the
assembled operator, through the C ABI and through solve_transport(ceed_op=...).

Bars: rtol 1e-11 on the FP64 true residual; solutions within 1e-8 relative L2 of the
direct solution; Dirichlet rows exact."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mesh(cuda_device):
    from dissolve_tp.mesh import face_dofs, kuhn_cube
    m = kuhn_cube(10, 0.2, seed=5)
    return m, face_dofs(m, 0, "min")


def _direct(m, De_c, al_c, inv_dt, lumped, b, bc=None):
    detJ, G, _ = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, m.n_verts)
    A = orc.assemble(detJ, G, De_c, al_c, inv_dt, lumped, sm, ix.size, bc_dofs=bc, indptr=ip,
                     indices=ix)
    return orc.direct_solve(ip, ix, A, b)


@pytest.mark.parametrize("lumped", [0, 1])
def test_matrix_free_solve_one_column_with_dirichlet(mesh, lumped):
    import torch

    from dissolve_tp.assembler import DeviceMesh
    from dissolve_tp.krylov import MatrixFreeCG
    m, bc = mesh
    rng = np.random.default_rng(1)
    De = np.exp(0.3 * rng.standard_normal(m.n_cells))
    al = rng.uniform(0, 1, m.n_cells)
    u_old = rng.uniform(0, 1, m.n_verts)
    detJ, _, _ = orc.geometry(m.coords, m.cells)
    b = orc.assemble_rhs(m.cells, detJ, u_old, None, 20.0, lumped, bc_dofs=bc, bc_value=1.0)
    want = _direct(m, De, al, 20.0, lumped, b, bc)
    dm = DeviceMesh(m.coords, m.cells)
    sol = MatrixFreeCG(dm, 1, 1, rtol=1e-11, max_it=3000, lumped=lumped)
    sol.b[:, 0] = torch.from_numpy(b)
    sol.x[:, 0] = torch.from_numpy(u_old)
    dev = dm.device
    res = sol.solve(torch.from_numpy(De).to(dev), 20.0, alpha_cell=torch.from_numpy(al).to(dev),
                    bc_mask=dm.bc_mask(bc))
    assert res["converged"], res
    assert res["rnorm"][0] <= 1e-11 * res["bnorm"][0]
    x = sol.x[:, 0].cpu().numpy()
    assert np.all(x[bc] == 1.0)
    assert np.linalg.norm(x - want) / np.linalg.norm(want) < 1e-8


def test_matrix_free_solve_three_species_columns(mesh):
    """The benchmarked step's three operators (D_s scaling of the stiffness, k_s shift of
    the lumped reaction) as three lanes of one matrix-free solve."""
    import torch

    from dissolve_tp.assembler import DeviceMesh
    from dissolve_tp.krylov import MatrixFreeCG
    m, _ = mesh
    rng = np.random.default_rng(2)
    coef = np.exp(0.3 * rng.standard_normal(m.n_cells))
    D, kk, inv_dt = (1.0, 1.0, 2.6), (0.5, 0.0, 0.2), 50.0
    U = rng.uniform(0, 1, (m.n_verts, 3))
    detJ, _, _ = orc.geometry(m.coords, m.cells)
    dm = DeviceMesh(m.coords, m.cells)
    sol = MatrixFreeCG(dm, 3, 4, rtol=1e-11, max_it=3000, lumped=1)
    wants = []
    for s in range(3):
        b = orc.assemble_rhs(m.cells, detJ, U[:, s], None, inv_dt, 1)
        sol.b[:, s] = torch.from_numpy(b)
        wants.append(_direct(m, D[s] * coef, np.full(m.n_cells, kk[s]), inv_dt, 1, b))
    sol.x[:, :3] = torch.from_numpy(U)
    res = sol.solve(torch.from_numpy(coef).to(dm.device), inv_dt, dscale=D, shift=kk)
    assert res["converged"], res
    X = sol.x[:, :3].cpu().numpy()
    for s in range(3):
        assert np.linalg.norm(X[:, s] - wants[s]) / np.linalg.norm(wants[s]) < 1e-8, s
    assert np.all(sol.x[:, 3].cpu().numpy() == 0.0)


def test_solve_transport_matrix_free_branch(cuda_device):
    """solve_transport(ceed_op=...) the way the driver calls the MatShell branch: the
    CeedDiffusionMassOp's operator (consistent mass + De K), the right-hand side from u_old,
    Dirichlet dofs on de_field, warm start from u."""
    import ceed_operators as co
    import solvers
    from dissolve_tp import fem
    from dissolve_tp.mesh import face_dofs, kuhn_cube
    m = kuhn_cube(9, 0.15, seed=3)
    mesh = fem.mesh_from(m)
    V = fem.FunctionSpace(mesh)
    bc = face_dofs(m, 0, "min")
    rng = np.random.default_rng(4)
    De_v = np.exp(0.3 * rng.standard_normal(m.n_verts))
    op = co.CeedDiffusionMassOp(co.make_ceed(True)[0], co.extract_ceed_mesh_data(mesh, V), De_v,
                                20.0)
    De = fem.Function(V, De_v)
    De._solver_bc_dofs = bc
    u_old = rng.uniform(0, 1, m.n_verts)
    u = fem.Function(V, u_old.copy())
    res = solvers.solve_transport("Cl", None, None, u, rtol=1e-11, max_it=3000,
                                  ceed_op=solvers.MatrixFreeOperator(op, m.n_verts),
                                  use_gpu=True, de_field=De, u_old=u_old, bc_value=0.5)
    assert res["converged"] and res["iterations"] > 0
    detJ, _, _ = orc.geometry(m.coords, m.cells)
    De_c = orc.to_cell_avg(De_v, m.n_cells, m.n_verts, m.cells)
    b = orc.assemble_rhs(m.cells, detJ, u_old, None, 20.0, 0, bc_dofs=bc, bc_value=0.5)
    want = _direct(m, De_c, np.zeros(m.n_cells), 20.0, 0, b, bc)
    assert np.linalg.norm(u.x.array - want) / np.linalg.norm(want) < 1e-8
    solvers._destroy_gpu_cache()
