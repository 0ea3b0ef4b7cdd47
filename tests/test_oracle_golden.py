"""Pin the CPU oracle to the reference: golden vectors made by the reference's own
gpu_assembler.py (tests/golden/make_golden.py) and known-answer P1 identities."""
import os

import numpy as np
import pytest

from conftest import golden_cases, load_golden
from oracle import oracle as orc

CASES = golden_cases()


@pytest.fixture(params=CASES, ids=[os.path.basename(c)[:-4] for c in CASES], scope="module")
def g(request):
    return load_golden(request.param)


def test_golden_fixtures_present():
    assert len(CASES) >= 4


def test_geometry_bit_exact(g):
    detJ, G, JT = orc.geometry(g["coords"], g["cells"])
    assert np.array_equal(detJ, g["detJ"])
    assert np.array_equal(G.ravel(), g["Gflat"])
    assert np.array_equal(JT.ravel(), g["JinvT"])


def test_pattern_and_scatter_map_bit_exact(g):
    indptr, indices, sm = orc.csr_pattern(g["cells"], g["coords"].shape[0])
    assert np.array_equal(indptr, g["indptr"])
    assert np.array_equal(indices, g["indices"])
    assert np.array_equal(sm, g["scatter_map"])
    assert np.array_equal(g["elem_nodes"], g["cells"].ravel())
    # PETSc COO preallocation order is CSR order (gpu_assembler.py:447-449)
    rows = np.repeat(np.arange(indptr.size - 1), np.diff(indptr))
    assert np.array_equal(rows, g["coo_rows"]) and np.array_equal(indices, g["coo_cols"])


@pytest.mark.parametrize("lumped", [1, 0])
def test_assembly_bit_exact(g, lumped):
    tag = "lumped" if lumped else "cons"
    nc, nv = g["cells"].shape[0], g["coords"].shape[0]
    G = g["Gflat"].reshape(nc, 9)
    nnz = g["indices"].size
    De = orc.to_cell_avg(g["De_vert"], nc, nv, g["cells"])
    A = orc.assemble(g["detJ"], G, De, g["alpha_cell"], float(g["inv_dt"]), lumped,
                     g["scatter_map"], nnz)
    assert np.array_equal(A, g[f"A_{tag}"])
    al = orc.to_cell_avg(g["alpha_vert"], nc, nv, g["cells"])
    A = orc.assemble(g["detJ"], G, g["De_cell"], al, float(g["inv_dt"]), lumped,
                     g["scatter_map"], nnz, bc_dofs=g["bc_dofs"], indptr=g["indptr"],
                     indices=g["indices"])
    assert np.array_equal(A, g[f"A_{tag}_bc"])
    A = orc.assemble(g["detJ"], G, g["De_cell"], np.zeros(nc), float(g["inv_dt"]), lumped,
                     g["scatter_map"], nnz)
    assert np.array_equal(A, g[f"A_{tag}_noalpha"])


def test_borrowed_geometry_matches_owner(g):
    assert np.array_equal(g["A_lumped_bc_borrow"].size, g["A_lumped_bc"].size)
    nc = g["cells"].shape[0]
    A = orc.assemble(g["detJ"], g["Gflat"].reshape(nc, 9), g["De_cell"], g["alpha_cell"],
                     float(g["inv_dt"]), 1, g["scatter_map"], g["indices"].size,
                     bc_dofs=g["bc_dofs"], indptr=g["indptr"], indices=g["indices"])
    assert np.array_equal(A, g["A_lumped_bc_borrow"])


@pytest.mark.parametrize("lumped", [1, 0])
def test_rhs_bit_exact(g, lumped):
    tag = "lumped" if lumped else "cons"
    args = (g["cells"], g["detJ"], g["u_old"])
    b = orc.assemble_rhs(*args, g["f_vert"], float(g["inv_dt"]), lumped)
    assert np.array_equal(b, g[f"b_{tag}"])
    b = orc.assemble_rhs(*args, g["f_vert"], float(g["inv_dt"]), lumped,
                         bc_dofs=g["bc_dofs"], bc_value=float(g["bc_value"]))
    assert np.array_equal(b, g[f"b_{tag}_bc"])
    b = orc.assemble_rhs(*args, None, float(g["inv_dt"]), lumped)
    assert np.array_equal(b, g[f"b_{tag}_nof"])


def test_nodal_gradient_and_scaffold_volume_bit_exact(g):
    nc = g["cells"].shape[0]
    for key, u in (("grad_u", g["u_old"]), ("grad_phi", g["phi"])):
        gr = orc.nodal_gradient(g["cells"], g["detJ"], g["JinvT"].reshape(nc, 9), u)
        assert np.array_equal(gr, g[key])
    v = orc.scaffold_volume(g["detJ"], g["cells"], g["phi"], float(g["eps"]))
    assert v == float(g["scaffold_volume"])


def test_length_mismatch_error_text(g):
    nc, nv = g["cells"].shape[0], g["coords"].shape[0]
    with pytest.raises(ValueError) as e:
        orc.to_cell_avg(np.ones(nv + 1), nc, nv, g["cells"])
    assert str(e.value) == str(g["err_len"])


# --------------------------------------------------------------- known answers
def _unit_tet():
    coords = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)
    cells = np.array([[0, 1, 2, 3]], dtype=np.int32)
    return coords, cells


def test_unit_tet_known_answers():
    coords, cells = _unit_tet()
    detJ, G, JT = orc.geometry(coords, cells)
    ip, ix, sm = orc.csr_pattern(cells, 4)
    M = orc.assemble(detJ, G, np.zeros(1), np.zeros(1), 1.0, 0, sm, 16).reshape(4, 4)
    assert np.allclose(M, (np.ones((4, 4)) + np.eye(4)) / 120.0, rtol=0, atol=1e-17)
    assert np.isclose(M.sum(), 1.0 / 6.0)
    ML = orc.assemble(detJ, G, np.zeros(1), np.zeros(1), 1.0, 1, sm, 16).reshape(4, 4)
    assert np.allclose(ML, np.eye(4) / 24.0, atol=1e-17)
    K = orc.assemble(detJ, G, np.ones(1), np.zeros(1), 0.0, 1, sm, 16).reshape(4, 4)
    Kexp = np.array([[3, -1, -1, -1], [-1, 1, 0, 0], [-1, 0, 1, 0], [-1, 0, 0, 1]]) / 6.0
    assert np.allclose(K, Kexp, atol=1e-16)


def test_mesh_identities():
    from dissolve_tp.mesh import kuhn_cube

    m = kuhn_cube(6, 0.2, seed=3)
    nc, nv = m.n_cells, m.n_verts
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, nv)
    K = orc.assemble(detJ, G, np.ones(nc), np.zeros(nc), 0.0, 1, sm, ix.size)
    M = orc.assemble(detJ, G, np.zeros(nc), np.zeros(nc), 1.0, 0, sm, ix.size)
    # K 1 = 0, sum(M) = volume, lumped mass = row sums of consistent mass
    assert np.abs(orc.spmv(ip, ix, K, np.ones(nv))).max() < 1e-12
    assert np.isclose(M.sum(), 1.0, rtol=1e-13)
    ml = orc.lumped_mass(m.cells, detJ, nv)
    assert np.allclose(orc.spmv(ip, ix, M, np.ones(nv)), ml, rtol=1e-13)
    # patch test: K x_linear vanishes on interior rows
    xl = 0.3 * m.coords[:, 0] - 1.2 * m.coords[:, 1] + 0.7 * m.coords[:, 2] + 0.1
    r = orc.spmv(ip, ix, K, xl)
    interior = np.all((m.coords > 1e-12) & (m.coords < 1 - 1e-12), axis=1)
    assert np.abs(r[interior]).max() < 1e-12


def test_matfree_matches_assembled():
    from dissolve_tp.mesh import kuhn_cube

    m = kuhn_cube(5, 0.2, seed=4)
    nc, nv = m.n_cells, m.n_verts
    rng = np.random.default_rng(0)
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, nv)
    De, al = np.exp(rng.standard_normal(nc)), rng.uniform(0, 1, nc)
    x = rng.standard_normal(nv)
    for lumped in (0, 1):
        A = orc.assemble(detJ, G, De, al, 7.0, lumped, sm, ix.size)
        y = orc.matfree_apply(m.cells, detJ, G, De, x, 7.0, alpha_cell=al, lumped=lumped)
        assert np.allclose(y, orc.spmv(ip, ix, A, x), rtol=1e-12, atol=1e-14)
    # legacy QFunction: stiffness weighted by 4 instead of |detJ|/6
    y0 = orc.matfree_apply(m.cells, detJ, G, De * (24.0 / detJ), x, 7.0)
    y1 = orc.matfree_apply(m.cells, detJ, G, De, x, 7.0, legacy=True)
    assert np.allclose(y0, y1, rtol=1e-11, atol=1e-12)


def test_oracle_solvers_agree_with_direct():
    from dissolve_tp.mesh import kuhn_cube, face_dofs

    m = kuhn_cube(8, 0.15, seed=0)
    nc, nv = m.n_cells, m.n_verts
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, nv)
    bc = face_dofs(m, 0, "min")
    A = orc.assemble(detJ, G, np.ones(nc), np.full(nc, 0.5), 20.0, 1, sm, ix.size,
                     bc_dofs=bc, indptr=ip, indices=ix)
    u0 = np.random.default_rng(2).uniform(0, 1, nv)
    b = orc.assemble_rhs(m.cells, detJ, u0, None, 20.0, 1, bc_dofs=bc, bc_value=1.0)
    xd = orc.direct_solve(ip, ix, A, b)
    x0 = u0.copy()
    x0[bc] = 1.0
    x, it, st, rn = orc.pcg_jacobi(ip, ix, A, b, x0, 1e-10, bc_dofs=bc)
    assert st == 0 and np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-9
    for nb in (1, 4):
        x, it, st, rn = orc.gmres_bjacobi(ip, ix, A, b, u0, 1e-10, nblocks=nb)
        assert st == 0 and np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-9


def test_reference_kernels_compiled_here_match_oracle():
    """oracle/_ref/libref_kernels_cpu.so (the reference kernel strings built by g++)
    against the C restatement on a larger mesh than the fixtures."""
    import ctypes

    from oracle import ref_recipe

    so = os.path.join(ref_recipe.OUT, "libref_kernels_cpu.so")
    if not os.path.exists(so):
        pytest.skip("oracle/_ref not built (reference not mounted)")
    from dissolve_tp.mesh import kuhn_cube

    lib = ctypes.CDLL(so)
    m = kuhn_cube(12, 0.2, seed=9)
    nc, nv = m.n_cells, m.n_verts
    rng = np.random.default_rng(5)
    detJ, G, JT = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, nv)
    De, al = np.exp(rng.standard_normal(nc)), rng.uniform(0, 1, nc)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    for lumped in (0, 1):
        data = np.zeros(ix.size)
        lib.ref_cpu_assemble_p1_tet(ctypes.c_uint((nc + 127) // 128), ctypes.c_uint(128),
                                    ctypes.c_int(nc), p(m.cells), p(detJ), p(G), p(De), p(al),
                                    ctypes.c_double(13.0), ctypes.c_int(lumped), p(sm), p(data))
        assert np.array_equal(data, orc.assemble(detJ, G, De, al, 13.0, lumped, sm, ix.size))


def _manufactured_case(n, c):
    """Unit cube, n cells per side: u = sin(pi x) sin(pi y) sin(pi z) solves
    -div grad u + c u = f with f = (3 pi^2 + c) u and u = 0 on the boundary."""
    from dissolve_tp.mesh import kuhn_cube

    m = kuhn_cube(n)
    x, y, z = m.coords.T
    ue = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
    f = (3.0 * np.pi ** 2 + c) * ue
    bnd = np.flatnonzero(np.any((m.coords < 1e-12) | (m.coords > 1.0 - 1e-12), axis=1))
    return m, ue, f, bnd.astype(np.int32)


@pytest.mark.parametrize("lumped", [0, 1])
def test_manufactured_solution_converges_second_order(lumped):
    """c M + K assembled by the oracle, b = M f, Dirichlet rows on the boundary, solved by
    the oracle's Jacobi-PCG: the mass-weighted nodal error against the exact solution
    falls by about 4x per halving of h (P1, second order), for both mass forms."""
    c = 2.0
    errs = []
    for n in (4, 8, 16):
        m, ue, f, bnd = _manufactured_case(n, c)
        detJ, G, JT = orc.geometry(m.coords, m.cells)
        ip, ix, sm = orc.csr_pattern(m.cells, m.n_verts)
        A = orc.assemble(detJ, G, np.ones(m.n_cells), np.zeros(m.n_cells), c, lumped, sm,
                         ix.size, bc_dofs=bnd, indptr=ip, indices=ix)
        b = orc.assemble_rhs(m.cells, detJ, np.zeros(m.n_verts), f, c, lumped, bc_dofs=bnd)
        uh, it, st, _ = orc.pcg_jacobi(ip, ix, A, b, np.zeros(m.n_verts), 1e-12,
                                       bc_dofs=bnd)
        assert st == 0
        e = uh - ue
        ml = orc.lumped_mass(m.cells, detJ, m.n_verts)
        errs.append(float(np.sqrt(np.sum(ml * e * e))))
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(len(errs) - 1)]
    # the coarsest pair is pre-asymptotic; the finest is second order
    assert all(1.6 < r < 2.3 for r in rates) and 1.85 < rates[-1] < 2.3, (errs, rates)
