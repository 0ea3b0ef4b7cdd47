"""tp_scaffold_volume_static (fixed scratch compiled into the library, no allocation)
against tp_scaffold_volume (caller scratch), through the C ABI.

Bar: two calls in a row each within 1e-13 relative of the caller-scratch result (the two
entry points launch the same kernels, so equality is expected), on a mesh whose launch
uses fewer than the 1024 block partials and on one that uses all of them."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [9, 40])
def test_static_scratch_matches_caller_scratch(cuda_device, n):
    import torch

    from dissolve_tp import _lib
    from dissolve_tp.assembler import DeviceMesh
    from dissolve_tp.device import ptr, stream_handle
    from dissolve_tp.mesh import kuhn_cube
    m = kuhn_cube(n, 0.15, seed=2)
    dm = DeviceMesh(m.coords, m.cells)
    rng = np.random.default_rng(n)
    x = m.coords
    phi = torch.from_numpy(np.linalg.norm(x - 0.5, axis=1) - 0.3
                           + 0.01 * rng.standard_normal(m.n_verts)).to(cuda_device)
    eps = 0.05
    ref = torch.zeros(1, dtype=torch.float64, device=cuda_device)
    _lib.call("tp_scaffold_volume", ctypes.byref(dm.tpm), ptr(phi), eps, ptr(ref), ptr(dm.scratch),
              stream_handle())
    want = float(ref.item())
    assert 0.0 < want < 1.0
    for _ in range(2):
        out = torch.full((1,), -1.0, dtype=torch.float64, device=cuda_device)
        _lib.call("tp_scaffold_volume_static", ctypes.byref(dm.tpm), ptr(phi), eps, ptr(out),
                  stream_handle())
        got = float(out.item())
        assert abs(got - want) <= 1e-13 * abs(want), (got, want)


def test_static_scratch_rejects_bad_arguments(cuda_device):
    import torch

    from dissolve_tp import _lib
    from dissolve_tp.assembler import DeviceMesh
    from dissolve_tp.device import ptr, stream_handle
    from dissolve_tp.mesh import kuhn_cube
    m = kuhn_cube(3, 0.1)
    dm = DeviceMesh(m.coords, m.cells)
    phi = torch.zeros(m.n_verts, dtype=torch.float64, device=cuda_device)
    out = torch.zeros(1, dtype=torch.float64, device=cuda_device)
    rc = _lib.lib.tp_scaffold_volume_static(ctypes.byref(dm.tpm), ptr(phi), 0.0, ptr(out),
                                            stream_handle())
    assert rc == 1
    rc = _lib.lib.tp_scaffold_volume_static(ctypes.byref(dm.tpm), ptr(phi), 0.1, None,
                                            stream_handle())
    assert rc == 1
