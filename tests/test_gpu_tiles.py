"""Tiled kernels (row tiles of tp_tiles_create) against the row-walk kernels they replace,
through the C ABI.

Bar: bit-identical outputs -- both sum every row's cells in ascending cell order with the
same rounding -- for every assembly mode, lumped and consistent mass, Dirichlet rows, the
FP32 copies, the SELL-32 values and lumped diagonals of the batched step, the lumped and
consistent right-hand sides, on a jittered
Kuhn cube and on the same mesh with its vertices and cells renumbered at random, for
tiles of 32, 64 and 128 rows."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _meshes():
    from dissolve_tp.mesh import TetMesh, kuhn_cube
    m = kuhn_cube(10, 0.2, seed=4)  # 1331 rows: the last SELL slice is partial
    rng = np.random.default_rng(7)
    pv = rng.permutation(m.n_verts)
    inv = np.empty_like(pv)
    inv[pv] = np.arange(m.n_verts)
    cells = inv[m.cells][rng.permutation(m.n_cells)]
    shuffled = TetMesh(coords=np.ascontiguousarray(m.coords[pv]),
                       cells=np.ascontiguousarray(cells.astype(np.int32)))
    return {"kuhn": m, "renumbered": shuffled}


@pytest.fixture(scope="module", params=["kuhn", "renumbered"])
def mesh(request, cuda_device):
    return _meshes()[request.param]


def _assemble(dm, mode, lumped, bc, De, al, tiles):
    import torch

    from dissolve_tp import _lib
    from dissolve_tp.device import ptr, stream_handle
    dm.set_tiles(tiles)
    o64 = torch.full((dm.nnz,), -7.0, dtype=torch.float64, device=De.device)
    o32 = torch.full((dm.nnz,), -7.0, dtype=torch.float32, device=De.device)
    _lib.call("tp_assemble_csr", ctypes.byref(dm.tpm), ptr(De), ptr(al), 20.0, lumped, mode,
              ptr(bc), ptr(o64), ptr(o32), stream_handle())
    return o64.cpu().numpy(), o32.cpu().numpy()


@pytest.mark.parametrize("tiles", [32, 64, 128])
def test_tiled_assembly_equals_row_walk(mesh, tiles):
    import torch

    from dissolve_tp import _lib
    from dissolve_tp.assembler import DeviceMesh
    from dissolve_tp.mesh import face_dofs
    dev = torch.device("cuda")
    dm = DeviceMesh(mesh.coords, mesh.cells, tile_rows=0)
    rng = np.random.default_rng(3)
    De = torch.from_numpy(np.exp(0.3 * rng.standard_normal(dm.n_cells))).to(dev)
    al = torch.from_numpy(rng.uniform(0, 1, dm.n_cells)).to(dev)
    bc = dm.bc_mask(np.nonzero(np.abs(mesh.coords[:, 0]) < 1e-12)[0].astype(np.int32))
    for mode in (_lib.TP_ASM_FULL, _lib.TP_ASM_STIFF, _lib.TP_ASM_MASS):
        for lumped in (1, 0):
            for mask in (None, bc):
                want = _assemble(dm, mode, lumped, mask, De, al, 0)
                got = _assemble(dm, mode, lumped, mask, De, al, tiles)
                assert np.array_equal(got[0], want[0]), (mode, lumped, mask is None)
                assert np.array_equal(got[1], want[1]), (mode, lumped, mask is None)
    info = dm.tiles_info()
    # bisection at multiples of the tile size leaves one partial tile at most
    assert info["rows_per_tile"] == tiles and info["n_tiles"] == -(-dm.n_verts // tiles)


@pytest.mark.parametrize("with_alpha", [True, False])
@pytest.mark.parametrize("S", [1, 3])
def test_tiled_stiffness_diag_equals_row_walk(mesh, S, with_alpha):
    """Without per-cell alpha the tiles keep 88-byte cell slots (the lumped factor alone)."""
    import torch

    from dissolve_tp.assembler import DeviceMesh
    from dissolve_tp.device import ptr, stream_handle
    from dissolve_tp.krylov import SellPattern
    from dissolve_tp import _lib
    dev = torch.device("cuda")
    dm = DeviceMesh(mesh.coords, mesh.cells, tile_rows=0)
    rng = np.random.default_rng(5)
    ld = {1: 1, 3: 4}[S]
    De = torch.from_numpy(np.exp(0.3 * rng.standard_normal(dm.n_cells))).to(dev)
    alpha = torch.from_numpy(rng.uniform(0, 1, (dm.n_cells, ld))).to(dev)
    shift = (ctypes.c_double * 4)(50.5, 50.0, 50.2, 0.0)
    bc = dm.bc_mask(np.arange(0, dm.n_verts, 17, dtype=np.int32))
    sell = SellPattern(dm.indptr, dm.indices)
    outs = []
    for tiles in (0, 64):
        dm.set_tiles(tiles)
        o64 = torch.full((dm.nnz,), -7.0, dtype=torch.float64, device=dev)
        o32 = torch.full((dm.nnz,), -7.0, dtype=torch.float32, device=dev)
        s32 = torch.full((sell.n_entries,), -7.0, dtype=torch.float32, device=dev)
        d64 = torch.full((dm.n_verts, ld), -7.0, dtype=torch.float64, device=dev)
        d32 = torch.full((dm.n_verts, ld), -7.0, dtype=torch.float32, device=dev)
        _lib.call("tp_assemble_stiffness_diag", ctypes.byref(dm.tpm), ptr(De), S, ld,
                  ptr(alpha) if with_alpha else None,
                  shift, ptr(bc), ptr(o64), ptr(o32), ptr(sell.slice_ptr), ptr(s32), ptr(d64),
                  ptr(d32), stream_handle())
        outs.append([t.cpu().numpy() for t in (o64, o32, s32, d64, d32)])
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("lumped", [1, 0])
@pytest.mark.parametrize("S,ld,with_f", [(1, 1, False), (3, 4, True), (2, 2, True),
                                         (3, 4, False)])
def test_tiled_rhs_equals_row_walk(mesh, S, ld, with_f, lumped):
    import torch

    from dissolve_tp import _lib
    from dissolve_tp.assembler import DeviceMesh
    from dissolve_tp.device import ptr, stream_handle
    dev = torch.device("cuda")
    dm = DeviceMesh(mesh.coords, mesh.cells, tile_rows=0)
    rng = np.random.default_rng(6)
    u = torch.from_numpy(rng.uniform(0, 1, (dm.n_verts, ld))).to(dev)
    f = torch.from_numpy(rng.normal(0, 1, (dm.n_verts, ld))).to(dev) if with_f else None
    bc = np.arange(0, dm.n_verts, 13, dtype=np.int32)
    bcd = torch.from_numpy(bc).to(dev)
    vals = (ctypes.c_double * 4)(0.5, 1.5, 2.5, 3.5)
    outs = []
    for tiles in (0, 64):
        dm.set_tiles(tiles)
        b = torch.full((dm.n_verts, ld), -7.0, dtype=torch.float64, device=dev)
        _lib.call("tp_assemble_rhs", ctypes.byref(dm.tpm), S, ld, ptr(u), ptr(f), 50.0, lumped,
                  bc.size, ptr(bcd), vals, ptr(b), stream_handle())
        outs.append(b.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
