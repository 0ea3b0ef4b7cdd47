"""Build recipe for the CPU oracle (test infrastructure).

    python -m oracle.build          # from the repository root

Compiles tp_oracle.c into oracle/build/libtp_oracle.so with gcc, OpenMP on and
floating-point contraction off (so every multiply and add rounds separately, as
the source is written).  When the reference project is mounted, also runs
oracle/ref_recipe.py, which compiles the reference's own kernel sources into
oracle/_ref/.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build_oracle(verbose: bool = False) -> str:
    out_dir = os.path.join(HERE, "build")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "libtp_oracle.so")
    src = os.path.join(HERE, "tp_oracle.c")
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-fvisibility=hidden", "-o", out + ".tmp", src, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(out + ".tmp", out)
    return out


# where the reference checkout is mounted when it is (this build recipe reads its kernel
# sources there); DISSOLVE_REFERENCE_ROOT names another checkout
REFERENCE_MOUNT = os.environ.get("DISSOLVE_REFERENCE_ROOT", "/root/reference")


def build_all(verbose: bool = False):
    build_oracle(verbose)
    from oracle import ref_recipe

    if ref_recipe.reference_present(REFERENCE_MOUNT):
        ref_recipe.build(REFERENCE_MOUNT, verbose=verbose)


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(HERE))
    build_all(verbose=True)
