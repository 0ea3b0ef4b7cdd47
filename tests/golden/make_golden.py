"""Generate golden vectors by running the reference's own gpu_assembler.py on the CPU.

    python tests/golden/make_golden.py <reference checkout>    # writes *.npz here
    (or DISSOLVE_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden.py)

The reference module (gpu/gpu_assembler.py) imports cupy, petsc4py and mpi4py,
none of which exist in this image.  This script imports the module UNMODIFIED
with stand-ins injected into sys.modules:

  cupy      numpy under the cupy names the module uses, plus
            `RawModule(code=...)`, which compiles the CUDA C string it is handed
            with g++ through oracle/cuda_cpu_shim.h and runs each launch thread by
            thread (atomicAdd -> plain add, so accumulation is in thread order);
  petsc4py  a Mat that records what setPreallocationCOO / setValuesCOO receive;
  mpi4py    COMM_WORLD.

`GPUSparseAssembler(domain, V)` then runs its own setup code (elem_nodes, numpy
geometry, Python-set sparsity pattern, dict scatter map) on duck-typed DOLFINx
mesh/function-space objects, and `assemble`, `assemble_rhs`, `nodal_gradient`
and `scaffold_volume` run the reference kernels.  Every output is saved with its
inputs.  The fixtures are small (meshes of 2-8 cells per side).
"""
from __future__ import annotations

import ctypes
import importlib.util
import os
import subprocess
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "dissolve-2.0_b200"))

from oracle import ref_recipe  # noqa: E402
from dissolve_tp.mesh import kuhn_cube, face_dofs  # noqa: E402

REF_GPU_ASSEMBLER = None  # set by main() from the command line or DISSOLVE_REFERENCE_ROOT


# ----------------------------------------------------------------------------- stand-ins
class _CpuKernel:
    def __init__(self, fn, params):
        self.fn = fn
        self.params = params

    def __call__(self, grid, block, args):
        conv = []
        for (typ, _), a in zip(self.params, args):
            if isinstance(a, np.ndarray):
                assert a.flags.c_contiguous
                conv.append(ctypes.c_void_p(a.ctypes.data))
            elif "double" in typ:
                conv.append(ctypes.c_double(float(a)))
            else:
                conv.append(ctypes.c_int(int(a)))
        self.fn(ctypes.c_uint(int(grid[0])), ctypes.c_uint(int(block[0])), *conv)


class RawModule:
    _count = 0

    def __init__(self, code, options=()):
        RawModule._count += 1
        self.kernels = dict(ref_recipe.parse_kernels(code))
        d = tempfile.mkdtemp(prefix="refk_")
        src = os.path.join(d, "k.cpp")
        with open(src, "w") as f:
            f.write('#include "cuda_cpu_shim.h"\n' + code + "\n")
            for name, params in self.kernels.items():
                f.write(ref_recipe._wrapper(name, params, gpu=False))
        so = os.path.join(d, f"k{RawModule._count}.so")
        subprocess.check_call(["g++", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
                               "-I", os.path.join(REPO, "oracle"), "-o", so, src])
        self.lib = ctypes.CDLL(so)

    def get_function(self, name):
        return _CpuKernel(getattr(self.lib, f"ref_cpu_{name}"), self.kernels[name])


def _fake_cupy():
    m = types.ModuleType("cupy")

    def __getattr__(name):
        return getattr(np, name)

    m.__getattr__ = __getattr__
    m.RawModule = RawModule
    m.asnumpy = lambda a: np.array(a)
    m.cuda = types.SimpleNamespace(runtime=types.SimpleNamespace(deviceSynchronize=lambda: None))
    return m


class _Mat:
    def create(self, comm=None):
        return self

    def setType(self, t):
        self.type = t

    def setSizes(self, s):
        self.sizes = s

    def setPreallocationCOO(self, rows, cols):
        self.coo_rows = np.array(rows)
        self.coo_cols = np.array(cols)

    def zeroEntries(self):
        pass

    def assemble(self):
        pass

    def setValuesCOO(self, data, mode=None):
        self.values = np.array(data, copy=True)


def _fake_petsc():
    pkg = types.ModuleType("petsc4py")
    petsc = types.ModuleType("petsc4py.PETSc")
    petsc.Mat = _Mat
    petsc.InsertMode = types.SimpleNamespace(INSERT=1, ADD=2)
    pkg.PETSc = petsc
    return pkg, petsc


def _fake_mpi():
    pkg = types.ModuleType("mpi4py")
    mpi = types.ModuleType("mpi4py.MPI")
    mpi.COMM_WORLD = types.SimpleNamespace(rank=0, size=1)
    pkg.MPI = mpi
    return pkg, mpi


def load_reference_assembler():
    pk, pe = _fake_petsc()
    mk, mp = _fake_mpi()
    # the stand-ins stay installed: GPUSparseAssembler.__init__ imports mpi4py at call time
    sys.modules.update({"cupy": _fake_cupy(), "petsc4py": pk, "petsc4py.PETSc": pe,
                        "mpi4py": mk, "mpi4py.MPI": mp})
    spec = importlib.util.spec_from_file_location("ref_gpu_assembler", REF_GPU_ASSEMBLER)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# duck-typed DOLFINx objects (only what GPUSparseAssembler.__init__ reads)
class _IndexMap:
    def __init__(self, n):
        self.size_local = n


def fake_domain_and_space(coords, cells):
    n, nv = cells.shape[0], coords.shape[0]
    topo = types.SimpleNamespace(dim=3, index_map=lambda d: _IndexMap(n))
    geom = types.SimpleNamespace(x=np.ascontiguousarray(coords))
    domain = types.SimpleNamespace(topology=topo, geometry=geom)
    dofmap = types.SimpleNamespace(index_map=_IndexMap(nv), cell_dofs=lambda i: cells[i])
    V = types.SimpleNamespace(dofmap=dofmap)
    return domain, V


# ----------------------------------------------------------------------------- cases
CASES = [
    # name, cells per side, jitter, mesh seed
    ("n2_j015", 2, 0.15, 0),
    ("n3_j020", 3, 0.20, 5),
    ("n4_j020", 4, 0.20, 7),
    ("n8_j015", 8, 0.15, 11),
]


def run_case(mod, name, n, jitter, seed):
    mesh = kuhn_cube(n, jitter, seed)
    coords, cells = mesh.coords, mesh.cells
    nc, nv = cells.shape[0], coords.shape[0]
    rng = np.random.default_rng(1000 + seed)
    De_vert = np.exp(0.3 * rng.standard_normal(nv))          # per-vertex -> cell average
    De_cell = np.exp(0.3 * rng.standard_normal(nc))          # per-cell pass-through
    alpha_cell = rng.uniform(0.0, 2.0, nc)
    alpha_vert = rng.uniform(0.0, 2.0, nv)
    u_old = rng.uniform(0.0, 1.0, nv)
    f_vert = rng.uniform(-0.5, 0.5, nv)
    phi = np.sin(3.0 * coords[:, 0]) * np.cos(2.0 * coords[:, 1]) + coords[:, 2] - 0.4
    eps = 1.5 / n
    inv_dt = 1.0 / 0.05
    bc = face_dofs(mesh, 0, "min")

    domain, V = fake_domain_and_space(coords, cells)
    out = dict(coords=coords, cells=cells, De_vert=De_vert, De_cell=De_cell,
               alpha_cell=alpha_cell, alpha_vert=alpha_vert, u_old=u_old, f_vert=f_vert,
               phi=phi, eps=np.float64(eps), inv_dt=np.float64(inv_dt), bc_dofs=bc,
               bc_value=np.float64(1.0))
    asm = mod.GPUSparseAssembler(domain, V)
    out.update(detJ=asm.d_detJ.copy(), Gflat=asm.d_Gflat.copy(), JinvT=asm.d_JinvT.copy(),
               indptr=asm.d_indptr.copy(), indices=asm.d_indices.copy(),
               scatter_map=asm.d_scatter_map.copy(), elem_nodes=asm.d_elem_nodes.copy(),
               coo_rows=asm.mat.coo_rows, coo_cols=asm.mat.coo_cols)
    for lumped in (1, 0):
        mod.LUMP_MASS = lumped
        tag = "lumped" if lumped else "cons"
        asm.assemble(De_vert, inv_dt, alpha=alpha_cell)
        out[f"A_{tag}"] = asm.mat.values.copy()
        asm.assemble(De_cell, inv_dt, alpha=alpha_vert, bc_dofs=bc)
        out[f"A_{tag}_bc"] = asm.mat.values.copy()
        asm.assemble(De_cell, inv_dt)
        out[f"A_{tag}_noalpha"] = asm.mat.values.copy()
        out[f"b_{tag}"] = asm.assemble_rhs(u_old, inv_dt, f=f_vert).copy()
        out[f"b_{tag}_bc"] = asm.assemble_rhs(u_old, inv_dt, f=f_vert, bc_dofs=bc,
                                              bc_value=1.0).copy()
        out[f"b_{tag}_nof"] = asm.assemble_rhs(u_old, inv_dt).copy()
    mod.LUMP_MASS = 1
    out["grad_u"] = np.array(asm.nodal_gradient(u_old))
    out["grad_phi"] = np.array(asm.nodal_gradient(phi))
    out["scaffold_volume"] = np.float64(asm.scaffold_volume(phi, eps))
    # length-mismatch error text (gpu_assembler.py:467-470)
    try:
        asm.assemble(np.ones(nv + 1), inv_dt)
    except ValueError as e:
        out["err_len"] = np.array(str(e))
    # shared-geometry borrower (gpu_assembler.py:346-367) must agree with the owner
    asm2 = mod.GPUSparseAssembler(domain, V, ref_asm=asm)
    asm2.assemble(De_cell, inv_dt, alpha=alpha_cell, bc_dofs=bc)
    out["A_lumped_bc_borrow"] = asm2.mat.values.copy()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return out


def main():
    global REF_GPU_ASSEMBLER
    REF_GPU_ASSEMBLER = ref_recipe.ref_file(sys.argv[1] if len(sys.argv) > 1 else None)
    if not os.path.exists(REF_GPU_ASSEMBLER):
        raise SystemExit(f"no reference gpu_assembler.py at {REF_GPU_ASSEMBLER}")
    mod = load_reference_assembler()
    for case in CASES:
        o = run_case(mod, *case)
        print(case[0], "cells", o["cells"].shape[0], "nnz", o["indices"].size)


if __name__ == "__main__":
    main()
