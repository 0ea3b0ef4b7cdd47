"""Mesh ingest on the CPU: Medit .mesh and XDMF (XML and raw-binary DataItems) readers
against the arrays they were written from, the reference's cell-tag check, the error for
HDF5 DataItems, and the oracle's level set from cell regions against a brute-force
nearest-interface search (domain/mesh_utils.py:81-267, 367-449)."""
import os

import numpy as np
import pytest

from oracle import oracle as orc


def _regioned(n=6):
    from dissolve_tp.mesh import kuhn_cube
    m = kuhn_cube(n, 0.15, seed=3)
    c = m.coords[m.cells].mean(axis=1) * 2 * np.pi
    g = (np.sin(c[:, 0]) * np.cos(c[:, 1]) + np.sin(c[:, 1]) * np.cos(c[:, 2]) +
         np.sin(c[:, 2]) * np.cos(c[:, 0]))
    return m, np.where(g > 0.3, 1, 2).astype(np.int32)


def test_medit_round_trip(tmp_path):
    from dissolve_tp import meshio
    m, reg = _regioned()
    path = str(tmp_path / "scaffold.mesh")
    meshio.write_medit_mesh(path, m.coords, m.cells, reg)
    pts, cells, regions = meshio.read_medit_mesh(path)
    assert np.array_equal(pts, m.coords)
    assert np.array_equal(cells, m.cells.astype(np.int64))
    assert np.array_equal(regions, reg)


def test_xdmf_binary_round_trip_and_tags(tmp_path):
    from dissolve_tp import meshio
    m, reg = _regioned()
    medit = str(tmp_path / "scaffold.mesh")
    meshio.write_medit_mesh(medit, m.coords, m.cells, reg)
    xdmf = meshio.convert_mesh_to_xdmf(medit)
    assert xdmf == str(tmp_path / "scaffold.xdmf") and os.path.exists(xdmf)
    mesh, tags = meshio.load_mesh(xdmf)
    assert np.array_equal(mesh.coords, m.coords)
    assert np.array_equal(mesh.cells, m.cells)
    assert mesh.cells.dtype == np.int32 and np.array_equal(tags, reg)
    # a single label fails the reference's check: no tags
    meshio.write_xdmf(str(tmp_path / "one.xdmf"), m.coords, m.cells, np.ones_like(reg))
    assert meshio.load_mesh(str(tmp_path / "one.xdmf"))[1] is None


def test_xdmf_inline_xml(tmp_path):
    from dissolve_tp import meshio
    xml = """<?xml version="1.0"?>
<Xdmf Version="3.0"><Domain><Grid Name="Grid" GridType="Uniform">
  <Topology TopologyType="Tetrahedron" NumberOfElements="2">
    <DataItem DataType="Int" Dimensions="2 4" Format="XML">0 1 2 3  1 2 3 4</DataItem>
  </Topology>
  <Geometry GeometryType="XYZ">
    <DataItem DataType="Float" Dimensions="5 3" Format="XML" Precision="8">
      0 0 0  1 0 0  0 1 0  0 0 1  1 1 1
    </DataItem>
  </Geometry>
  <Attribute Name="region" AttributeType="Scalar" Center="Cell">
    <DataItem DataType="Int" Dimensions="2" Format="XML">1 2</DataItem>
  </Attribute>
</Grid></Domain></Xdmf>"""
    p = tmp_path / "tiny.xdmf"
    p.write_text(xml)
    mesh, tags = meshio.load_mesh(str(p))
    assert mesh.cells.tolist() == [[0, 1, 2, 3], [1, 2, 3, 4]]
    assert mesh.coords[4].tolist() == [1.0, 1.0, 1.0] and tags.tolist() == [1, 2]
    bad = xml.replace("1 2 3 4</DataItem>", "1 2 3 9</DataItem>")
    p.write_text(bad)
    with pytest.raises(meshio.MeshFormatError, match="outside the geometry"):
        meshio.load_mesh(str(p))


def test_hdf5_dataitem_is_named_in_the_error(tmp_path):
    """The reference's own layout (mesh_utils.py:172-193): HDF DataItems with an .h5
    companion, which this build cannot read."""
    from dissolve_tp import meshio
    xml = """<?xml version="1.0"?>
<Xdmf Version="3.0"><Domain><Grid Name="Grid" GridType="Uniform">
  <Topology TopologyType="Tetrahedron" NumberOfElements="802365">
    <DataItem DataType="Int" Dimensions="802365 4" Format="HDF">m.h5:/mesh/cells</DataItem>
  </Topology>
  <Geometry GeometryType="XYZ">
    <DataItem DataType="Float" Dimensions="135075 3" Format="HDF" Precision="8">m.h5:/mesh/points</DataItem>
  </Geometry>
</Grid></Domain></Xdmf>"""
    p = tmp_path / "m.xdmf"
    p.write_text(xml)
    with pytest.raises(meshio.MeshFormatError, match=r"m\.h5:/mesh/cells.*missing"):
        meshio.load_mesh(str(p))


def test_oracle_phi_from_regions_matches_brute_force():
    m, reg = _regioned(5)
    phi = orc.phi_from_regions(m.coords, m.cells, reg, 1)
    scaf = reg == 1
    in_s = np.zeros(m.n_verts, bool)
    in_f = np.zeros(m.n_verts, bool)
    in_s[m.cells[scaf].ravel()] = True
    in_f[m.cells[~scaf].ravel()] = True
    iface = np.nonzero(in_s & in_f)[0]
    assert 0 < iface.size < m.n_verts
    d = np.sqrt(((m.coords[:, None, :] - m.coords[None, iface, :]) ** 2).sum(-1)).min(1)
    sign = np.where(in_s, 1.0, -1.0)
    assert np.allclose(phi, sign * d, rtol=0, atol=1e-15)
    assert np.all(phi[iface] == 0.0)
    # no interface: +-0.5
    assert np.array_equal(orc.phi_from_regions(m.coords, m.cells, np.ones_like(reg), 1),
                          np.full(m.n_verts, 0.5))
