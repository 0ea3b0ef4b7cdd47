"""The shipped package never reaches the oracle: no module under dissolve-2.0_b200/ imports,
loads or names a file of oracle/, so every result it returns comes from the CUDA
library."""
import ast
import glob
import os

from conftest import PKG


def _sources():
    return sorted(glob.glob(os.path.join(PKG, "**", "*.py"), recursive=True))


def test_package_imports_nothing_from_the_oracle():
    assert _sources()
    for path in _sources():
        tree = ast.parse(open(path).read(), filename=path)
        for node in ast.walk(tree):
            if isinstance(node, ast.Import):
                names = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom):
                names = [node.module or ""]
            else:
                continue
            for name in names:
                assert not name.split(".")[0] == "oracle", f"{path}: imports {name}"


def test_package_loads_no_oracle_library():
    for path in _sources() + glob.glob(os.path.join(PKG, "csrc", "*")):
        text = open(path, errors="replace").read()
        for token in ("libtp_oracle", "oracle/_ref", "oracle/build", "ref_kernels"):
            assert token not in text, f"{path}: names {token}"
