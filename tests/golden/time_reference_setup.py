"""Time the reference's own setup, GPUSparseAssembler.__init__, on the CPU.

    python tests/golden/time_reference_setup.py <reference checkout>
    (or DISSOLVE_REFERENCE_ROOT=<reference checkout> python tests/golden/time_reference_setup.py)

The reference module runs unmodified with the stand-ins of make_golden.py: numpy for
cupy, a recording Mat for petsc4py, and duck-typed DOLFINx objects. Its setup
(gpu/gpu_assembler.py:331-450) computes numpy geometry, builds the CSR pattern from
per-row Python sets and the element-to-nonzero scatter map from a Python dict, and uploads
the result. The stand-ins make the upload a numpy copy and preallocation a record, so
the time measured is the Python and numpy work of the setup alone, a lower bound for the
reference's setup on a GPU host.

Jittered Kuhn cubes of N = 8 .. 64 cells per side (the benchmark mesh's family, up to
the 64^3 benchmark mesh itself) are timed, best of 3 runs (one at N = 64). The result is
tests/golden/ref_setup_timing.json, which bench.py reports beside its own GPU setup
time.
"""
from __future__ import annotations

import json
import os
import platform
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_golden  # noqa: E402  (stand-ins and the reference loader)
from make_golden import fake_domain_and_space, kuhn_cube, ref_recipe  # noqa: E402

SIZES = (8, 16, 32, 64)


def main():
    make_golden.REF_GPU_ASSEMBLER = ref_recipe.ref_file(sys.argv[1] if len(sys.argv) > 1
                                                        else None)
    mod = make_golden.load_reference_assembler()
    rows = []
    for n in SIZES:
        mesh = kuhn_cube(n, 0.2, 0)
        domain, V = fake_domain_and_space(mesh.coords, mesh.cells)
        best = float("inf")
        for _ in range(1 if n >= 64 else 3):
            t = time.perf_counter()
            mod.GPUSparseAssembler(domain, V)
            best = min(best, time.perf_counter() - t)
        rows.append({"cells_per_side": n, "cells": int(mesh.n_cells), "vertices": int(mesh.n_verts),
                     "setup_s": round(best, 4)})
        print(rows[-1], flush=True)
    out = {
        "what": "GPUSparseAssembler.__init__ of gpu/gpu_assembler.py:331-450, unmodified, with "
                "numpy standing in for cupy and a recording Mat for petsc4py (a lower bound: "
                "no device transfers, no PETSc preallocation)",
        "host": platform.processor() or platform.machine(),
        "python": platform.python_version(),
        "runs": rows,
        "setup_64cube_s": rows[-1]["setup_s"],
    }
    with open(os.path.join(HERE, "ref_setup_timing.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps({"setup_64cube_s": out["setup_64cube_s"]}))


if __name__ == "__main__":
    main()
