"""Drop-in modules: import paths, pure-host helpers and the error behaviour of the
branches this build does not provide (no GPU needed)."""
import numpy as np
import pytest


def test_gpu_assembler_module_is_the_implementation():
    import gpu_assembler
    from dissolve_tp import assembler
    assert gpu_assembler is assembler
    assert hasattr(gpu_assembler, "GPUSparseAssembler") and gpu_assembler.LUMP_MASS in (0, 1)


def test_ceed_helpers_without_gpu():
    import ceed_operators as co
    from dissolve_tp.mesh import kuhn_cube
    m = kuhn_cube(3, 0.1)
    md = co.extract_ceed_mesh_data(m)
    assert md["num_cells"] == 162 and md["num_dofs"] == 64 and md["num_qpts"] == 4
    assert np.isclose(md["q_wts"].sum(), 1.0 / 6.0)
    basis, nq = co.build_simplex_basis(None)
    assert nq == 4 and np.allclose(basis["interp"].sum(1), 1.0)
    # degree-2 rule integrates x^2 on the reference tet exactly: 1/60
    assert np.isclose((co.Q_PTS[:, 0] ** 2 * co.Q_WTS).sum(), 1.0 / 60.0)
    er = co.build_elem_restriction(None, m.cells, m.n_verts)
    assert er["l_size"] == m.n_verts and er["offsets"].size == 4 * m.n_cells
    assert co.libceed_available()


def test_unsupported_branches_raise():
    import solvers
    with pytest.raises(NotImplementedError):
        solvers.solve_transport("Cl", None, None, None, use_gpu=False)
    with pytest.raises(NotImplementedError):
        solvers.solve_transport("Cl", None, None, None, ceed_op=object(), use_gpu=True)
    with pytest.raises(NotImplementedError):
        solvers.solve_transport("Cl", None, None, None, use_gpu=True, de_field=object(),
                                pc_type="hypre")
