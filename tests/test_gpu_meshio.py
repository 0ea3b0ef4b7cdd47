"""An ingested mesh on the GPU: the level set from cell regions (tp_phi_from_regions,
domain/mesh_utils.py:367-449) against the oracle's KD-tree restatement, and the assembly
of the ingested mesh against the oracle.

Bars: the level set equal to the oracle's within 1e-15 absolute (the same FP64 distances,
each rounded once, and an exact minimum); FP64 assembly within 1e-12 relative."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def test_phi_from_regions_and_assembly_of_an_ingested_mesh(cuda_device, tmp_path):
    from dissolve_tp import meshio, physics
    from dissolve_tp.assembler import DeviceMesh, GPUSparseAssembler
    from dissolve_tp.mesh import kuhn_cube
    m = kuhn_cube(10, 0.15, seed=3)
    c = m.coords[m.cells].mean(axis=1) * 2 * np.pi
    g = (np.sin(c[:, 0]) * np.cos(c[:, 1]) + np.sin(c[:, 1]) * np.cos(c[:, 2]) +
         np.sin(c[:, 2]) * np.cos(c[:, 0]))
    reg = np.where(g > 0.3, 1, 2).astype(np.int32)
    medit = str(tmp_path / "scaffold.mesh")
    meshio.write_medit_mesh(medit, m.coords, m.cells, reg)
    mesh, tags = meshio.load_mesh(meshio.convert_mesh_to_xdmf(medit))
    assert np.array_equal(tags, reg)
    dm = DeviceMesh(mesh.coords, mesh.cells)
    want = orc.phi_from_regions(mesh.coords, mesh.cells, tags, 1)
    got = physics.phi_from_regions(dm, tags, 1).cpu().numpy()
    assert np.abs(got - want).max() <= 1e-15
    # every cell in the scaffold: no interface vertex, +0.5 everywhere
    half = physics.phi_from_regions(dm, np.ones_like(tags), 1).cpu().numpy()
    assert np.array_equal(half, np.full(mesh.n_verts, 0.5))
    # the ingested mesh assembles as the oracle does
    asm = GPUSparseAssembler(mesh)
    De = np.exp(0.3 * np.random.default_rng(1).standard_normal(mesh.n_cells))
    asm.assemble(De, 20.0, alpha=np.full(mesh.n_cells, 0.5))
    detJ, G, JT = orc.geometry(mesh.coords, mesh.cells)
    ip, ix, sm = orc.csr_pattern(mesh.cells, mesh.n_verts)
    A = orc.assemble(detJ, G, De, np.full(mesh.n_cells, 0.5), 20.0, 1, sm, ix.size)
    got_a = asm.d_data.cpu().numpy()
    assert np.abs(got_a - A).max() <= 1e-12 * np.abs(A).max()
