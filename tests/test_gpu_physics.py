"""Builders around the transport step on the GPU against the oracle: the O2 reaction and
OH- source coefficients (dissolve.py:866-875, 923-936), effective film
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


def _species_fields(n=20000, eps=0.1):
    """phi spread over the band |phi| < eps, its edges, both sides of it and exact zeros."""
    rng = np.random.default_rng(11)
    phi = np.concatenate([rng.uniform(-eps, eps, n // 2), rng.uniform(-1.0, 1.0, n // 2)])
    phi[:8] = [0.0, eps, -eps, np.nextafter(eps, 0.0), -np.nextafter(eps, 0.0), 1e-300,
               -1e-300, 0.5 * eps]
    ng = np.abs(rng.normal(1.0, 0.3, n))
    F, Cl, O2 = rng.uniform(0, 2, n), rng.uniform(0, 1, n), rng.uniform(0, 1, n)
    return phi, ng, F, Cl, O2


def _close(got, want, rel=1e-14):
    """Within rel of each value, or of the largest value where 1 + cos(pi phi / eps)
    cancels near the band edges (there one ulp of cos is a large relative change)."""
    return np.all(np.abs(got - want) <= rel * (np.abs(want) + 0.1 * np.abs(want).max()))


def test_o2_alpha_matches_oracle(cuda_device):
    from dissolve_tp import physics
    eps, k_orr = 0.1, 2.0
    phi, ng, _, _, _ = _species_fields(eps=eps)
    got = physics.o2_alpha(phi, ng, eps, k_orr).cpu().numpy()
    want = orc.o2_alpha(phi, ng, eps, k_orr)
    inside = np.abs(phi) < eps
    assert inside.sum() > 1000 and (~inside).sum() > 1000
    assert np.all(got[~inside] == 0.0) and np.all(want[~inside] == 0.0)
    # just inside the band edges 1 + cos(pi phi / eps) rounds to 0: non-negative, and
    # positive almost everywhere
    assert np.all(got[inside] >= 0.0) and (got[inside] > 0.0).mean() > 0.99
    assert _close(got, want)


def test_oh_source_matches_oracle(cuda_device):
    from dissolve_tp import physics
    eps, kd, k_orr = 0.1, 0.05, 2.0
    phi, ng, F, Cl, O2 = _species_fields(eps=eps)
    for fac in (4.0, 2.0):
        got = physics.oh_source(phi, ng, F, Cl, O2, eps, kd, k_orr, fac).cpu().numpy()
        want = orc.oh_source(phi, ng, F, Cl, O2, eps, kd, k_orr, fac)
        assert _close(got, want)
    # outside the band and outside the medium (phi > eps) nothing is produced
    dry = phi >= eps
    assert dry.sum() > 1000 and np.all(got[dry] == 0.0)
    # inside the medium and outside the band: the film term alone
    wet = phi <= -eps
    assert np.allclose(got[wet], kd * F[wet] * Cl[wet] ** 2, rtol=1e-15, atol=0)


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
