"""Mesh ingest: Medit .mesh files and XDMF mesh descriptions (host side).

Reference: domain/mesh_utils.py -- _read_medit_mesh (:111-153), _write_xdmf (:156-197),
convert_mesh_to_xdmf (:81-108) and load_mesh (:200-267).  The reference converts a Medit
mesh into XDMF with an HDF5 companion and loads it through DOLFINx.  Here:

  read_medit_mesh(path)              -> (points, cells, regions), as the reference's reader
  write_xdmf(xdmf_path, points, cells, regions)
                                     the reference's XDMF structure (one Grid with a
                                     Tetrahedron Topology, XYZ Geometry and a cell
                                     Attribute "region"), with the data in raw little-endian
                                     binary companions (Format="Binary") instead of HDF5
  convert_mesh_to_xdmf(mesh_path, output_dir=None) -> xdmf path
  load_mesh(xdmf_path)               -> (TetMesh, cell_tags or None)

load_mesh reads DataItems in XML (inline) and Binary form.  An HDF DataItem needs an
HDF5 reader, which this build does not have: it raises MeshFormatError naming the dataset.
The reference's own shipped description (mesh_adaptive_800k.xdmf) points to an .h5
companion that is not shipped with it.  The P1 dofs are the vertices in file order: DOLFINx
renumbers dofs when it builds a function space, and that order is not reproduced here.
Cell tags follow the reference's check (:218-228): they must contain the scaffold label
1 and at least one other label, else they are None.
"""
from __future__ import annotations

import os
import xml.etree.ElementTree as ET

import numpy as np

from .mesh import TetMesh


class MeshFormatError(ValueError):
    """A mesh file this reader cannot read (unsupported form, missing data)."""


# ----------------------------------------------------------------- Medit
def read_medit_mesh(path: str):
    """Parse a Medit .mesh file (mesh_utils.py:111-153): the Vertices and Tetrahedra
    sections.  Returns (points (nv, 3) float64, cells (nc, 4) int64 with 0-based vertex
    ids, regions (nc,) int32 from each tetrahedron's reference number, 0 when absent)."""
    points, cells, regions = [], [], []
    with open(path) as f:
        lines = f.readlines()
    i, n = 0, len(lines)
    while i < n:
        key = lines[i].strip()
        if key == "Vertices":
            nv = int(lines[i + 1].strip())
            for j in range(nv):
                p = lines[i + 2 + j].split()
                points.append([float(p[0]), float(p[1]), float(p[2])])
            i += 2 + nv
        elif key == "Tetrahedra":
            nt = int(lines[i + 1].strip())
            for j in range(nt):
                p = lines[i + 2 + j].split()
                cells.append([int(p[0]) - 1, int(p[1]) - 1, int(p[2]) - 1, int(p[3]) - 1])
                regions.append(int(p[4]) if len(p) > 4 else 0)
            i += 2 + nt
        else:
            i += 1
    return (np.array(points, dtype=np.float64).reshape(-1, 3),
            np.array(cells, dtype=np.int64).reshape(-1, 4),
            np.array(regions, dtype=np.int32))


def write_medit_mesh(path: str, points, cells, regions=None):
    """Write a Medit .mesh file (MeshVersionFormatted 1, dimension 3) with the vertices and
    tetrahedra (1-based ids, the region as reference number)."""
    points = np.asarray(points, dtype=np.float64)
    cells = np.asarray(cells, dtype=np.int64)
    regions = np.zeros(len(cells), np.int32) if regions is None else np.asarray(regions)
    with open(path, "w") as f:
        f.write("MeshVersionFormatted 1\nDimension 3\nVertices\n%d\n" % len(points))
        for p in points:
            f.write("%.17g %.17g %.17g 0\n" % (p[0], p[1], p[2]))
        f.write("Tetrahedra\n%d\n" % len(cells))
        for c, r in zip(cells, regions):
            f.write("%d %d %d %d %d\n" % (c[0] + 1, c[1] + 1, c[2] + 1, c[3] + 1, r))
        f.write("End\n")


# ----------------------------------------------------------------- XDMF
_XDMF = """<?xml version="1.0"?>
<Xdmf Version="3.0">
  <Domain>
    <Grid Name="Grid" GridType="Uniform">
      <Topology TopologyType="Tetrahedron" NumberOfElements="{nc}">
        <DataItem DataType="Int" Dimensions="{nc} 4" Format="Binary" Precision="8" Endian="Little">
          {base}.cells.bin
        </DataItem>
      </Topology>
      <Geometry GeometryType="XYZ">
        <DataItem DataType="Float" Dimensions="{nv} 3" Format="Binary" Precision="8" Endian="Little">
          {base}.points.bin
        </DataItem>
      </Geometry>
      <Attribute Name="region" AttributeType="Scalar" Center="Cell">
        <DataItem DataType="Int" Dimensions="{nc}" Format="Binary" Precision="4" Endian="Little">
          {base}.regions.bin
        </DataItem>
      </Attribute>
    </Grid>
  </Domain>
</Xdmf>
"""


def write_xdmf(xdmf_path: str, points, cells, regions=None) -> str:
    """The reference's XDMF layout (mesh_utils.py:156-197) with raw little-endian binary
    companions next to it: <base>.points.bin (float64), <base>.cells.bin (int64),
    <base>.regions.bin (int32)."""
    d = os.path.dirname(os.path.abspath(xdmf_path))
    base = os.path.splitext(os.path.basename(xdmf_path))[0]
    points = np.ascontiguousarray(points, dtype="<f8")
    cells = np.ascontiguousarray(cells, dtype="<i8")
    regions = np.zeros(len(cells), "<i4") if regions is None else \
        np.ascontiguousarray(regions, dtype="<i4")
    points.tofile(os.path.join(d, base + ".points.bin"))
    cells.tofile(os.path.join(d, base + ".cells.bin"))
    regions.tofile(os.path.join(d, base + ".regions.bin"))
    with open(xdmf_path, "w") as f:
        f.write(_XDMF.format(nc=len(cells), nv=len(points), base=base))
    return xdmf_path


def convert_mesh_to_xdmf(mesh_path: str, output_dir: str | None = None) -> str:
    """Medit .mesh -> XDMF (mesh_utils.py:81-108): <base>.xdmf in output_dir (default: the
    mesh's directory), kept when it exists already."""
    out = output_dir or os.path.dirname(mesh_path) or "."
    base = os.path.splitext(os.path.basename(mesh_path))[0]
    xdmf_path = os.path.join(out, base + ".xdmf")
    if not os.path.exists(xdmf_path):
        points, cells, regions = read_medit_mesh(mesh_path)
        write_xdmf(xdmf_path, points, cells, regions)
    return xdmf_path


_TYPES = {("int", 4): "i4", ("int", 8): "i8", ("uint", 4): "u4", ("uint", 8): "u8",
          ("float", 4): "f4", ("float", 8): "f8", ("char", 1): "i1", ("uchar", 1): "u1"}


def _data_item(item, base_dir: str) -> np.ndarray:
    """One XDMF DataItem as an array of its Dimensions (XML and Binary forms)."""
    dims = [int(x) for x in item.get("Dimensions", "").split()]
    fmt = item.get("Format", "XML").lower()
    dtype = item.get("DataType", item.get("NumberType", "Float")).lower()
    prec = int(item.get("Precision", "8" if dtype == "float" else "4"))
    if (dtype, prec) not in _TYPES:
        raise MeshFormatError(f"unsupported XDMF DataType {dtype} Precision {prec}")
    text = (item.text or "").strip()
    count = int(np.prod(dims)) if dims else 0
    if fmt == "xml":
        arr = np.array(text.split(), dtype=_TYPES[(dtype, prec)])
    elif fmt == "binary":
        endian = "<" if item.get("Endian", "Native").lower() in ("little", "native") else ">"
        path = text if os.path.isabs(text) else os.path.join(base_dir, text)
        if not os.path.exists(path):
            raise MeshFormatError(f"XDMF binary data file {path} does not exist")
        arr = np.fromfile(path, dtype=endian + _TYPES[(dtype, prec)], count=count,
                          offset=int(item.get("Seek", "0")))
    elif fmt == "hdf":
        h5 = text.split(":")[0]
        where = "present" if os.path.exists(os.path.join(base_dir, h5)) else "missing"
        raise MeshFormatError(f"XDMF DataItem {text} is HDF5 data (companion {h5}: {where}); "
                              "this build reads XML and Binary DataItems only")
    else:
        raise MeshFormatError(f"unsupported XDMF DataItem Format {item.get('Format')}")
    if arr.size != count:
        raise MeshFormatError(f"XDMF DataItem holds {arr.size} values, Dimensions say {count}")
    return arr.reshape(dims)


def load_mesh(xdmf_path: str, comm=None):
    """The Grid of an XDMF file as (TetMesh, cell_tags) (mesh_utils.py:200-267).
    cell_tags is the cell Attribute (int32 per cell) when it holds the scaffold label 1
    and at least one other label, else None (the reference's check, :218-228).  comm is
    accepted for the reference's signature; the mesh is read whole."""
    base_dir = os.path.dirname(os.path.abspath(xdmf_path))
    root = ET.parse(xdmf_path).getroot()
    grid = root.find(".//Grid")
    if grid is None:
        raise MeshFormatError(f"{xdmf_path}: no Grid")
    topo, geom = grid.find("Topology"), grid.find("Geometry")
    if topo is None or geom is None:
        raise MeshFormatError(f"{xdmf_path}: the Grid needs a Topology and a Geometry")
    if topo.get("TopologyType", "").lower() != "tetrahedron":
        raise MeshFormatError(f"topology {topo.get('TopologyType')}: tetrahedra only")
    if geom.get("GeometryType", "XYZ").upper() != "XYZ":
        raise MeshFormatError(f"geometry {geom.get('GeometryType')}: XYZ only")
    cells = _data_item(topo.find("DataItem"), base_dir).reshape(-1, 4)
    points = _data_item(geom.find("DataItem"), base_dir).reshape(-1, 3).astype(np.float64)
    if cells.size and (cells.min() < 0 or cells.max() >= len(points)):
        raise MeshFormatError("topology references a vertex outside the geometry")
    mesh = TetMesh(coords=np.ascontiguousarray(points),
                   cells=np.ascontiguousarray(cells.astype(np.int32)))
    tags = None
    for att in grid.findall("Attribute"):
        if att.get("Center", "").lower() == "cell":
            vals = _data_item(att.find("DataItem"), base_dir).reshape(-1).astype(np.int32)
            if vals.size == len(cells):
                u = set(np.unique(vals).tolist())
                tags = vals if (1 in u and len(u) >= 2) else None
            break
    return mesh, tags
