"""Compile the reference's own CUDA kernel sources into oracle/_ref/ (test infrastructure).

The reference keeps its kernels as CUDA C string literals in gpu/gpu_assembler.py
(`_ASSEMBLE_KERNEL` :60-139, `_BC_KERNEL_SRC` :147-165, `_RHS_KERNEL_SRC` :176-221,
`_RHS_BC_KERNEL_SRC` :228-239, `_GRAD_KERNEL_SRC` :251-304) and compiles them at
import with CuPy NVRTC.  This recipe reads those literals with `ast` from the
mounted reference (never copying them into the repository), writes them under
a temporary directory and builds two libraries from them into oracle/_ref/:

  libref_kernels_cpu.so  the kernels compiled by g++ through cuda_cpu_shim.h, each
                         wrapped in `ref_cpu_<name>(grid, block, args...)`, which
                         runs every (block, thread) in order -- atomicAdd becomes a
                         plain add, so accumulation follows thread order;
  libref_kernels_gpu.so  the same kernels compiled by nvcc for sm_100a, each wrapped
                         in `ref_gpu_<name>(grid, block, stream, args...)` -- the
                         reference's own GPU kernels, timed on the B200 as a bar.

oracle/_ref/ is git-ignored; the built libraries travel with the working tree.
"""
from __future__ import annotations

import ast
import os
import re
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: an argument of build() / the command line, else this variable
REF_ROOT = os.environ.get("DISSOLVE_REFERENCE_ROOT")
OUT = os.path.join(HERE, "_ref")
KERNEL_VARS = ("_ASSEMBLE_KERNEL", "_BC_KERNEL_SRC", "_RHS_KERNEL_SRC",
               "_RHS_BC_KERNEL_SRC", "_GRAD_KERNEL_SRC")


def ref_file(ref_root: str | None = None) -> str:
    root = ref_root or REF_ROOT
    if not root:
        raise RuntimeError("the reference checkout is not given: pass its root or set "
                           "DISSOLVE_REFERENCE_ROOT")
    return os.path.join(root, "gpu", "gpu_assembler.py")


def reference_present(ref_root: str | None = None) -> bool:
    root = ref_root or REF_ROOT
    return bool(root) and os.path.exists(ref_file(root))


def extract_sources(path: str) -> dict[str, str]:
    tree = ast.parse(open(path).read())
    found = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and len(node.targets) == 1:
            t = node.targets[0]
            if isinstance(t, ast.Name) and t.id in KERNEL_VARS:
                found[t.id] = ast.literal_eval(node.value)
    missing = set(KERNEL_VARS) - set(found)
    if missing:
        raise RuntimeError(f"kernel literals not found in {path}: {sorted(missing)}")
    return found


_SIG = re.compile(r'extern\s+"C"\s+__global__\s+void\s+(\w+)\s*\((.*?)\)\s*\{', re.S)


def parse_kernels(src: str):
    """[(name, [(type, argname), ...])] of each extern "C" __global__ kernel in src."""
    nocomment = re.sub(r"//[^\n]*", "", src)
    out = []
    for m in _SIG.finditer(nocomment):
        params = []
        for p in m.group(2).split(","):
            p = " ".join(p.split())
            if not p:
                continue
            name = re.findall(r"(\w+)\s*$", p)[0]
            typ = p[: p.rfind(name)].strip()
            params.append((typ, name))
        out.append((m.group(1), params))
    return out


def _wrapper(name, params, gpu: bool) -> str:
    decl = ", ".join(f"{t} {n}" for t, n in params)
    call = ", ".join(n for _, n in params)
    if gpu:
        return (f'extern "C" int ref_gpu_{name}(unsigned shim_grid_, unsigned shim_block_, '
                f'void* shim_stream_, {decl}) {{\n'
                f"  {name}<<<shim_grid_, shim_block_, 0, (cudaStream_t)shim_stream_>>>({call});\n"
                f"  return (int)cudaGetLastError();\n}}\n")
    return (f'extern "C" void ref_cpu_{name}(unsigned shim_grid_, unsigned shim_block_, {decl}) {{\n'
            f"  blockDim.x = shim_block_; gridDim.x = shim_grid_;\n"
            f"  for (unsigned shim_b_ = 0; shim_b_ < shim_grid_; shim_b_++)\n"
            f"    for (unsigned shim_t_ = 0; shim_t_ < shim_block_; shim_t_++) {{\n"
            f"      blockIdx.x = shim_b_; threadIdx.x = shim_t_; {name}({call});\n"
            f"    }}\n}}\n")


def write_sources(workdir: str, ref_root: str | None = None) -> tuple[str, str, list]:
    srcs = extract_sources(ref_file(ref_root))
    body = "\n".join(srcs[k] for k in KERNEL_VARS)
    kernels = parse_kernels(body)
    cpu = os.path.join(workdir, "ref_kernels_cpu.cpp")
    gpu = os.path.join(workdir, "ref_kernels_gpu.cu")
    with open(cpu, "w") as f:
        f.write('#include "cuda_cpu_shim.h"\n')
        f.write(body)
        f.write("\n")
        for name, params in kernels:
            f.write(_wrapper(name, params, gpu=False))
    with open(gpu, "w") as f:
        f.write("#include <cuda_runtime.h>\n")
        f.write(body)
        f.write("\n")
        for name, params in kernels:
            f.write(_wrapper(name, params, gpu=True))
    return cpu, gpu, kernels


def build(ref_root: str | None = None, verbose: bool = False, gpu: bool = True) -> dict:
    """Compile the kernels of the reference checkout at ref_root (else
    DISSOLVE_REFERENCE_ROOT) in a temporary directory; only the two libraries land in
    oracle/_ref/."""
    import tempfile

    os.makedirs(OUT, exist_ok=True)
    with tempfile.TemporaryDirectory(prefix="ref_recipe_") as work:
        return _build_in(work, ref_root, verbose, gpu)


def _build_in(work: str, ref_root: str | None, verbose: bool, gpu: bool) -> dict:
    cpu_src, gpu_src, kernels = write_sources(work, ref_root)
    outs = {}
    cpu_so = os.path.join(OUT, "libref_kernels_cpu.so")
    cmd = ["g++", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-I", HERE,
           "-o", cpu_so, cpu_src]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    outs["cpu"] = cpu_so
    if gpu and shutil.which("nvcc"):
        gpu_so = os.path.join(OUT, "libref_kernels_gpu.so")
        cmd = ["nvcc", "-O3", "-std=c++14", "-gencode", "arch=compute_100a,code=sm_100a",
               "-Xcompiler", "-fPIC", "-shared", "-o", gpu_so, gpu_src]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        outs["gpu"] = gpu_so
    outs["kernels"] = kernels
    return outs


if __name__ == "__main__":
    import sys

    # python -m oracle.ref_recipe <reference checkout>   (or DISSOLVE_REFERENCE_ROOT)
    r = build(sys.argv[1] if len(sys.argv) > 1 else None, verbose=True)
    print({k: v for k, v in r.items() if k != "kernels"})
    for name, params in r["kernels"]:
        print(name, [n for _, n in params])
