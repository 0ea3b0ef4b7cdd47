"""Per-vertex builders around the transport step, on the GPU (the CuPy/numpy element-wise
code of the reference's time loop): the O2 reaction and OH- source coefficients, effective
film diffusivity, Zn transport coefficients, Sussman redistancing of the level set and the
mean cell diameter."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import call
from .device import ptr, stream_handle, to_device


def film_floor(porosity: float = 0.25, constrictivity: float = 1.0,
               tortuosity: float = 2.0) -> float:
    """eps delta / tau^2 (physics/interface_velocity.py:118-127; parameters.py:119-121)."""
    return porosity * constrictivity / (tortuosity * tortuosity)


def o2_alpha(phi, normgradphi, epsilon, k_orr):
    """alpha_O2 = delta_eps(phi) |grad phi| k_ORR per vertex (dissolve.py:866-875, with
    delta_eps of physics/weak_forms.py:18-24): the O2 consumption at the interface band."""
    phi_d = to_device(phi, torch.float64, torch.device("cuda"))
    dev = phi_d.device
    ng_d = to_device(normgradphi, torch.float64, dev)
    out = torch.empty_like(phi_d)
    call("tp_o2_alpha", int(phi_d.numel()), ptr(phi_d), ptr(ng_d), float(epsilon), float(k_orr),
         ptr(out), stream_handle())
    return out


def oh_source(phi, normgradphi, F, Cl, O2, epsilon, kd, k_orr, orr_factor=4.0):
    """f_OH = [phi <= 0] kd F Cl^2 + orr_factor delta_eps(phi) |grad phi| k_ORR O2 per vertex
    (dissolve.py:923-936): film dissolution plus the ORR production of OH-."""
    phi_d = to_device(phi, torch.float64, torch.device("cuda"))
    dev = phi_d.device
    ins = [to_device(a, torch.float64, dev) for a in (normgradphi, F, Cl, O2)]
    out = torch.empty_like(phi_d)
    call("tp_oh_source", int(phi_d.numel()), ptr(phi_d), *(ptr(a) for a in ins),
         float(epsilon), float(kd), float(k_orr), float(orr_factor), ptr(out), stream_handle())
    return out


def effective_diffusion(phi, F, Fmax, D0=(2.72, 7.78, 20.16, 9.36), floor=None):
    """(De_Zn, De_Cl, De_OH, De_O2) per vertex (compute_effective_diffusion,
    interface_velocity.py:90-155); raises like the reference on NaN/Inf or negatives."""
    phi_d = to_device(phi, torch.float64, torch.device("cuda"))
    dev = phi_d.device
    F_d = to_device(F, torch.float64, dev)
    n = int(phi_d.numel())
    out = [torch.empty(n, dtype=torch.float64, device=dev) for _ in range(4)]
    flags = torch.zeros(1, dtype=torch.int32, device=dev)
    d0 = (ctypes.c_double * 4)(*[float(v) for v in D0])
    fl = film_floor() if floor is None else float(floor)
    rc = _lib.lib.tp_effective_diffusion(n, ptr(phi_d), ptr(F_d), float(Fmax), fl, d0,
                                         *(ptr(o) for o in out), ptr(flags), stream_handle())
    if rc != _lib.TP_OK:
        raise RuntimeError(f"[bounds] {_lib.last_error()}")
    return tuple(out)


def zn_coefficients(phi, F, Cl, kf, kd, Fmax):
    """(alpha, source) of the Zn transport (dissolve.py:746-755) and the scaffold
    Dirichlet dofs phi > 0 (dissolve.py:745) as an int32 numpy array."""
    phi_d = to_device(phi, torch.float64, torch.device("cuda"))
    dev = phi_d.device
    n = int(phi_d.numel())
    alpha = torch.empty(n, dtype=torch.float64, device=dev)
    src = torch.empty(n, dtype=torch.float64, device=dev)
    # keep the device copies referenced until the kernel has been enqueued
    F_d, Cl_d = to_device(F, torch.float64, dev), to_device(Cl, torch.float64, dev)
    call("tp_zn_coefficients", n, ptr(phi_d), ptr(F_d), ptr(Cl_d), float(kf), float(kd),
         float(Fmax), ptr(alpha), ptr(src), stream_handle())
    scaffold = np.nonzero(phi_d.cpu().numpy() > 0.0)[0].astype(np.int32)
    return alpha, src, scaffold


def mean_cell_diameter(dm) -> float:
    """h_avg of a DeviceMesh (domain/mesh_utils.py:559-575)."""
    out = torch.zeros(1, dtype=torch.float64, device=dm.device)
    scratch = torch.empty(1024, dtype=torch.float64, device=dm.device)
    call("tp_mean_cell_diameter", ctypes.byref(dm.tpm), ptr(out), ptr(scratch), stream_handle())
    return float(out.item()) / dm.n_cells


def redistance(dm, phi: torch.Tensor, num_iters: int = 8, h_avg: float | None = None,
               band_factor: float = 3.0, eps_factor: float = 1.5) -> torch.Tensor:
    """Sussman redistancing of phi (device, in place) on a DeviceMesh
    (domain/mesh_utils.py:450-542, GPU branch)."""
    h = mean_cell_diameter(dm) if h_avg is None else float(h_avg)
    scratch = torch.empty(int(_lib.lib.tp_redistance_scratch_bytes(dm.n_verts)) // 8,
                          dtype=torch.float64, device=dm.device)
    call("tp_redistance", ctypes.byref(dm.tpm), ptr(phi), int(num_iters), h, float(band_factor),
         float(eps_factor), ptr(scratch), stream_handle())
    return phi


def phi_from_regions(dm, regions, scaffold_label: int = 1) -> torch.Tensor:
    """Level set from cell region labels (domain/mesh_utils.py:367-449): + inside the
    scaffold cells' vertices, - elsewhere, magnitude the distance to the nearest vertex
    shared by a scaffold cell and another cell (0.5 when there is none).  regions: one
    int label per cell (load_mesh's cell tags)."""
    reg = to_device(np.asarray(regions, dtype=np.int32) if not isinstance(regions, torch.Tensor)
                    else regions, torch.int32, dm.device)
    phi = torch.empty(dm.n_verts, dtype=torch.float64, device=dm.device)
    nb = int(_lib.lib.tp_phi_from_regions_scratch_bytes(dm.n_verts))
    scratch = torch.empty(max(nb, 8) // 8 + 1, dtype=torch.float64, device=dm.device)
    call("tp_phi_from_regions", ctypes.byref(dm.tpm), ptr(reg), int(scaffold_label), ptr(phi),
         ptr(scratch), stream_handle())
    return phi
