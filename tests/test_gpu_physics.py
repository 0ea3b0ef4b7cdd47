"""Builders around the transport step on the GPU against the oracle: effective film
diffusivity (interface_velocity.py:90-155), Zn transport coefficients and the Zn solve with
the scaffold as its Dirichlet set (dissolve.py:740-778, through the solvers drop-in),
Sussman redistancing (mesh_utils.py:450-542) and the mean cell diameter.

Bars: element-wise builders exact to 1e-15 relative; h_avg to 1e-13; redistancing within
1e-12 absolute after 5 steps; the Zn solve within 1e-9 relative L2 of the oracle's direct
solve (rtol 1e-10)."""
import math

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _gyroid(n=8, jitter=0.15):
    from dissolve_tp.coupled import gyroid_inputs
    return gyroid_inputs(n, jitter)


def test_effective_diffusion_and_bounds(cuda_device):
    from dissolve_tp import physics
    m, phi, _, _ = _gyroid()
    F = np.random.default_rng(1).uniform(0, 2.0, m.n_verts)
    out = physics.effective_diffusion(phi, F, 1.5)
    ref = orc.effective_diffusion(phi, F, 1.5, physics.film_floor(), (2.72, 7.78, 20.16, 9.36))
    for a, b in zip(out, ref):
        assert np.allclose(a.cpu().numpy(), b, rtol=1e-15, atol=0)
    with pytest.raises(RuntimeError):
        physics.effective_diffusion(phi, np.full(m.n_verts, np.nan), 1.5)
    with pytest.raises(RuntimeError):
        physics.effective_diffusion(phi, F, 1.5, D0=(-1.0, 1.0, 1.0, 1.0))


def test_zn_solve_with_scaffold_dirichlet(cuda_device):
    import solvers
    from dissolve_tp import fem, physics
    m, phi, _, _ = _gyroid()
    rng = np.random.default_rng(2)
    F = rng.uniform(0, 1, m.n_verts)
    Cl = rng.uniform(0, 1, m.n_verts)
    alpha, src, scaffold = physics.zn_coefficients(phi, F, Cl, 0.3, 0.05, 1.5)
    a_ref, s_ref = orc.zn_coefficients(phi, F, Cl, 0.3, 0.05, 1.5)
    assert np.allclose(alpha.cpu().numpy(), a_ref, rtol=1e-15, atol=0)
    assert np.allclose(src.cpu().numpy(), s_ref, rtol=1e-15, atol=0)
    assert np.array_equal(scaffold, np.nonzero(phi > 0)[0]) and scaffold.size > m.n_verts // 10
    mesh = fem.mesh_from(m)
    V = fem.FunctionSpace(mesh)
    De = fem.Function(V, np.full(m.n_verts, 2.72))
    De._solver_inv_dt = 1.0 / 0.05
    De._solver_bc_dofs = scaffold
    zn_old = rng.uniform(0, 1e-8, m.n_verts)
    zn = fem.Function(V, zn_old.copy())
    res = solvers.solve_transport("Zn", None, None, zn, rtol=1e-10, max_it=2000, use_gpu=True,
                                  de_field=De, alpha_field=alpha.cpu().numpy(), u_old=zn_old,
                                  source_field=src.cpu().numpy(), bc_value=1e-8)
    assert res["converged"]
    detJ, G, _ = orc.geometry(m.coords, m.cells)
    ip, ix, sm = orc.csr_pattern(m.cells, m.n_verts)
    De_c = orc.to_cell_avg(np.full(m.n_verts, 2.72), m.n_cells, m.n_verts, m.cells)
    al_c = orc.to_cell_avg(a_ref, m.n_cells, m.n_verts, m.cells)
    A = orc.assemble(detJ, G, De_c, al_c, 20.0, 1, sm, ix.size, bc_dofs=scaffold, indptr=ip,
                     indices=ix)
    b = orc.assemble_rhs(m.cells, detJ, zn_old, s_ref, 20.0, 1, bc_dofs=scaffold, bc_value=1e-8)
    x = orc.direct_solve(ip, ix, A, b)
    assert np.linalg.norm(zn.x.array - x) / np.linalg.norm(x) < 1e-9
    assert np.all(zn.x.array[scaffold] == 1e-8)
    solvers._destroy_gpu_cache()


def test_redistance_and_h_avg(cuda_device):
    import torch

    from dissolve_tp import physics
    from dissolve_tp.assembler import DeviceMesh
    m, phi, _, _ = _gyroid(10, 0.2)
    dm = DeviceMesh(m.coords, m.cells)
    h = physics.mean_cell_diameter(dm)
    assert abs(h - orc.mean_cell_diameter(m.coords, m.cells)) <= 1e-13 * h
    # a level set with |grad| far from 1: 3 x the gyroid
    p = torch.from_numpy(3.0 * phi).to(cuda_device)
    physics.redistance(dm, p, num_iters=5, h_avg=h)
    detJ, _, JT = orc.geometry(m.coords, m.cells)
    ref = orc.redistance(m.cells, detJ, JT, 3.0 * phi, 5, h)
    assert np.abs(p.cpu().numpy() - ref).max() < 1e-12
    assert not np.array_equal(ref, 3.0 * phi)
    # the frozen band keeps the interface nodes
    band = np.abs(3.0 * phi) < 3.0 * h
    assert np.array_equal(p.cpu().numpy()[band], (3.0 * phi)[band])
