"""CPU oracle for the P1-tet transport path (TEST INFRASTRUCTURE ONLY).

Only tests/, `__graft_entry__.smoke()` and bench.py's CPU-baseline legs import this
module, as the checker or the timed CPU baseline.  The product package never does.

The numpy parts restate the reference line by line:
  geometry           gpu/gpu_assembler.py:380-386   (same numpy calls: det, inv, matmul)
  csr_pattern        gpu/gpu_assembler.py:396-410   (row = sorted set of cell-mates)
  scatter_map        gpu/gpu_assembler.py:423-438   ((row, col) -> CSR position)
  to_cell_avg        gpu/gpu_assembler.py:452-470
  scaffold_volume    gpu/gpu_assembler.py:605-644
  species coefficients  dissolve.py:866-875 (O2 alpha), :923-936 (OH source),
                        physics/weak_forms.py:18-38 (delta_eps, coarea factor)
  under_relax        numerics/solvers.py:278-279
The sequential C parts live in tp_oracle.c (built by oracle/build.py).

Parity pin: tests/golden/ holds vectors produced by running the reference's own
gpu_assembler.py (kernel source strings compiled for the CPU) on small meshes, and
tests/test_oracle_golden.py checks this oracle against them.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


def lib_path() -> str:
    return os.path.join(_HERE, "build", "libtp_oracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = lib_path()
        if not os.path.exists(path):
            from oracle.build import build_oracle  # noqa: local import

            build_oracle()
        _LIB = ctypes.CDLL(path)
    return _LIB


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ---------------------------------------------------------------- geometry / pattern
def geometry(coords: np.ndarray, cells: np.ndarray):
    """(detJ, Gflat (n,9), JinvT (n,9)) exactly as gpu_assembler.py:380-386."""
    x = coords[:, :3]
    edges = x[cells][:, 1:, :] - x[cells][:, 0:1, :]
    J = edges.transpose(0, 2, 1)
    detJ = np.abs(np.linalg.det(J))
    Jinv = np.linalg.inv(J)
    G = Jinv @ Jinv.transpose(0, 2, 1)
    JinvT = Jinv.transpose(0, 2, 1)
    n = cells.shape[0]
    return (np.ascontiguousarray(detJ), np.ascontiguousarray(G.reshape(n, 9)),
            np.ascontiguousarray(JinvT.reshape(n, 9)))


def csr_pattern(cells: np.ndarray, n_dofs: int):
    """(indptr int32, indices int32, scatter_map int32) of gpu_assembler.py:396-438.

    Row r holds the sorted set of every vertex sharing a cell with r (itself
    included); scatter_map[c*16 + i*4 + j] is the CSR position of
    (cells[c,i], cells[c,j])."""
    c = cells.astype(np.int64)
    rows = np.repeat(c, 4, axis=1).ravel()
    cols = np.tile(c, (1, 4)).ravel()
    key = rows * n_dofs + cols
    ukey, inv = np.unique(key, return_inverse=True)
    urow = ukey // n_dofs
    indices = (ukey % n_dofs).astype(np.int32)
    counts = np.bincount(urow, minlength=n_dofs)
    indptr = np.zeros(n_dofs + 1, dtype=np.int64)
    np.cumsum(counts, out=indptr[1:])
    return indptr.astype(np.int32), indices, inv.astype(np.int32).ravel()


def to_cell_avg(arr, n_cells: int, n_dofs: int, cells: np.ndarray):
    """gpu_assembler.py:452-470."""
    if arr is None:
        return np.zeros(n_cells, dtype=np.float64)
    n = int(arr.shape[0])
    if n == n_cells:
        return np.asarray(arr, dtype=np.float64)
    if n == n_dofs:
        d = np.asarray(arr, dtype=np.float64)
        return d[cells.ravel()].reshape(n_cells, 4).mean(axis=1)
    raise ValueError(f"array length {n} matches neither n_cells={n_cells} "
                     f"nor n_dofs={n_dofs}")


# ---------------------------------------------------------------- assembly (C)
def assemble(detJ, Gflat, De_cell, alpha_cell, inv_dt, lumped, scatter_map, nnz,
             bc_dofs=None, indptr=None, indices=None):
    data = np.zeros(nnz, dtype=np.float64)
    n = detJ.shape[0]
    sm = _c32(scatter_map)
    lib().or_assemble(ctypes.c_int64(n), _p(_c64(detJ)), _p(_c64(Gflat)), _p(_c64(De_cell)),
                      _p(_c64(alpha_cell)), ctypes.c_double(inv_dt), ctypes.c_int(int(lumped)),
                      _p(sm), ctypes.c_int64(nnz), _p(data))
    if bc_dofs is not None and len(bc_dofs) > 0:
        bc = _c32(bc_dofs)
        lib().or_dirichlet_rows(ctypes.c_int64(bc.size), _p(bc), _p(_c32(indptr)),
                                _p(_c32(indices)), _p(data))
    return data


def assemble_rhs(cells, detJ, u_old, f, inv_dt, lumped, bc_dofs=None, bc_value=0.0):
    n, nd = cells.shape[0], u_old.shape[0]
    b = np.zeros(nd, dtype=np.float64)
    f = np.zeros(nd) if f is None else f
    lib().or_assemble_rhs(ctypes.c_int64(n), ctypes.c_int64(nd), _p(_c32(cells)), _p(_c64(detJ)),
                          _p(_c64(u_old)), _p(_c64(f)), ctypes.c_double(inv_dt),
                          ctypes.c_int(int(lumped)), _p(b))
    if bc_dofs is not None and len(bc_dofs) > 0:
        bc = _c32(bc_dofs)
        lib().or_dirichlet_rhs(ctypes.c_int64(bc.size), _p(bc), ctypes.c_double(bc_value), _p(b))
    return b


def nodal_gradient(cells, detJ, JinvT, u):
    n, nd = cells.shape[0], u.shape[0]
    g = np.zeros((nd, 3), dtype=np.float64)
    w = np.zeros(nd, dtype=np.float64)
    lib().or_nodal_gradient(ctypes.c_int64(n), ctypes.c_int64(nd), _p(_c32(cells)),
                            _p(_c64(detJ)), _p(_c64(JinvT)), _p(_c64(u)), _p(g), _p(w))
    return g


def lumped_mass(cells, detJ, n_dofs):
    m = np.zeros(n_dofs, dtype=np.float64)
    lib().or_lumped_mass(ctypes.c_int64(cells.shape[0]), ctypes.c_int64(n_dofs),
                         _p(_c32(cells)), _p(_c64(detJ)), _p(m))
    return m


def matfree_apply(cells, detJ, Gflat, De_cell, x, inv_dt, alpha_cell=None, lumped=False,
                  legacy=False, diff_scale=None, shift=None):
    """y = sum_e [De_e K_e + (inv_dt + alpha_e + shift_s) M_e] x  for x of shape (V,) or (V,S)."""
    x2 = x.reshape(x.shape[0], -1)
    S = x2.shape[1]
    y = np.zeros_like(x2, dtype=np.float64)
    xs = _c64(x2)
    ds = None if diff_scale is None else _c64(diff_scale)
    sh = None if shift is None else _c64(shift)
    al = None if alpha_cell is None else _c64(alpha_cell)
    lib().or_matfree_apply(ctypes.c_int64(cells.shape[0]), ctypes.c_int64(x2.shape[0]),
                           ctypes.c_int(S), _p(_c32(cells)), _p(_c64(detJ)), _p(_c64(Gflat)),
                           _p(_c64(De_cell)), _p(al) if al is not None else None,
                           _p(ds) if ds is not None else None, _p(sh) if sh is not None else None,
                           ctypes.c_double(inv_dt), ctypes.c_int(int(lumped)),
                           ctypes.c_int(int(legacy)), _p(xs), _p(y))
    return y.reshape(x.shape)


def spmv(indptr, indices, data, x):
    y = np.empty(indptr.shape[0] - 1, dtype=np.float64)
    lib().or_spmv(ctypes.c_int64(y.size), _p(_c32(indptr)), _p(_c32(indices)), _p(_c64(data)),
                  _p(_c64(x)), _p(y))
    return y


def pcg_jacobi(indptr, indices, data, b, x0, rtol, max_it=10000, bc_dofs=None):
    n = b.shape[0]
    x = _c64(x0).copy()
    mask = np.zeros(n, dtype=np.uint8)
    if bc_dofs is not None:
        mask[np.asarray(bc_dofs)] = 1
    st = ctypes.c_int(0)
    rn = ctypes.c_double(0.0)
    it = lib().or_pcg_jacobi(ctypes.c_int64(n), _p(_c32(indptr)), _p(_c32(indices)),
                             _p(_c64(data)), _p(mask), _p(_c64(b)), _p(x), ctypes.c_double(rtol),
                             ctypes.c_int(max_it), ctypes.byref(st), ctypes.byref(rn))
    return x, int(it), int(st.value), float(rn.value)


def gmres_bjacobi(indptr, indices, data, b, x0, rtol, max_it=10000, restart=50, nblocks=1):
    n = b.shape[0]
    x = _c64(x0).copy()
    st = ctypes.c_int(0)
    rn = ctypes.c_double(0.0)
    it = lib().or_gmres_bjacobi(ctypes.c_int64(n), _p(_c32(indptr)), _p(_c32(indices)),
                                _p(_c64(data)), _p(_c64(b)), _p(x), ctypes.c_double(rtol),
                                ctypes.c_int(max_it), ctypes.c_int(restart),
                                ctypes.c_int(nblocks), ctypes.byref(st), ctypes.byref(rn))
    return x, int(it), int(st.value), float(rn.value)


def set_threads(n: int):
    lib().or_set_threads(ctypes.c_int(n))


def num_threads() -> int:
    return int(lib().or_num_threads())


# ---------------------------------------------------------------- numpy restatements
def scaffold_volume(detJ, cells, phi, epsilon):
    """gpu_assembler.py:605-644: 4-point degree-2 rule, smoothed Heaviside."""
    alpha = (5.0 + 3.0 * math.sqrt(5.0)) / 20.0
    beta = (5.0 - math.sqrt(5.0)) / 20.0
    f = np.asarray(phi, dtype=np.float64)
    n = cells.shape[0]
    phi_nodes = f[cells.ravel()].reshape(n, 4)
    phi_sum = phi_nodes.sum(axis=1, keepdims=True)
    phi_q = (alpha - beta) * phi_nodes + beta * phi_sum
    H_q = np.where(phi_q < -epsilon, 0.0,
                   np.where(phi_q > epsilon, 1.0,
                            0.5 * (1.0 + phi_q / epsilon + np.sin(np.pi * phi_q / epsilon) / np.pi)))
    cell_H = H_q.mean(axis=1)
    return float(np.sum(cell_H * (detJ / 6.0)))


def delta_eps(phi, epsilon):
    """physics/weak_forms.py:18-24 / dissolve.py:869-872."""
    return np.where(np.abs(phi) < epsilon,
                    (1.0 / (2.0 * epsilon)) * (1.0 + np.cos(np.pi * phi / epsilon)), 0.0)


def o2_alpha(phi, normgradphi, epsilon, k_orr):
    """dissolve.py:866-875: alpha_O2 = delta_eps(phi) |grad phi| k_ORR."""
    return delta_eps(phi, epsilon) * normgradphi * k_orr


def oh_source(phi, normgradphi, F, Cl, O2, epsilon, kd, k_orr, orr_factor=4.0):
    """dissolve.py:923-936: medium kd F Cl^2 + 4 delta_eps |grad phi| k_ORR O2."""
    medium = np.where(phi <= 0.0, 1.0, 0.0)
    return medium * kd * F * Cl ** 2 + orr_factor * delta_eps(phi, epsilon) * normgradphi * k_orr * O2



def heaviside_eps(phi, epsilon):
    """Smoothed Heaviside of gpu_assembler.py:605-644 (scaffold_volume's integrand)."""
    phi = np.asarray(phi, dtype=np.float64)
    mid = 0.5 * (1.0 + phi / epsilon + np.sin(np.pi * phi / epsilon) / np.pi)
    return np.where(phi < -epsilon, 0.0, np.where(phi > epsilon, 1.0, mid))


def interface_terms(phi, grad, epsilon, k_orr, orr_factor, U, col_o2=0, col_oh=2):
    """Gyroid-step interface reaction: hv = k_orr H_eps(phi), |grad phi|, and the explicit
    OH- source f[:, col_oh] = orr_factor hv U[:, col_o2] (zero elsewhere)."""
    hv = k_orr * heaviside_eps(phi, epsilon)
    ng = None if grad is None else np.sqrt((np.asarray(grad) ** 2).sum(axis=1))
    f = np.zeros_like(np.asarray(U, dtype=np.float64))
    f[:, col_oh] = orr_factor * hv * U[:, col_o2]
    return hv, ng, f


def levelset_advance(phi, U, col, dt, rate, gain):
    """phi - dt rate (1 + gain U[:, col])."""
    return phi - dt * rate * (1.0 + gain * U[:, col])


def effective_diffusion(phi, F, Fmax, film_floor, D0):
    """physics/interface_velocity.py:90-155: (De_Zn, De_Cl, De_OH, De_O2)."""
    fm = max(Fmax, 1e-20)
    sat = np.clip(F / fm, 0.0, 1.0)
    ff = (1.0 - sat) + sat * film_floor
    med = np.where(phi <= 0.0, 1.0, 0.0)
    return D0[0] * ff, D0[1] * ff * med, D0[2] * ff * med, D0[3] * ff * med


def zn_coefficients(phi, F, Cl, kf, kd, Fmax):
    """dissolve.py:746-755: alpha and source of the Zn transport."""
    med = np.where(phi <= 0.0, 1.0, 0.0)
    return med * kf * (1.0 - F / Fmax), med * kd * F * (Cl * Cl)


def mean_cell_diameter(coords, cells):
    """domain/mesh_utils.py:559-575 (dolfinx mesh.h of a tetrahedron: longest edge)."""
    p = coords[cells]
    h2 = np.zeros(cells.shape[0])
    for a in range(4):
        for b in range(a + 1, 4):
            h2 = np.maximum(h2, ((p[:, a] - p[:, b]) ** 2).sum(axis=1))
    return float(np.sqrt(h2).mean())


def redistance(cells, detJ, JinvT, phi, iters, h_avg, band_factor=3.0, eps_factor=1.5):
    """domain/mesh_utils.py:450-542: Sussman pseudo-time steps with the frozen band."""
    phi = np.array(phi, dtype=np.float64)
    mask = np.abs(phi) < band_factor * h_avg
    eps = eps_factor * h_avg
    sign = phi / np.sqrt(phi ** 2 + eps ** 2)
    for _ in range(iters):
        g = nodal_gradient(cells, detJ, JinvT, phi)
        gm = np.sqrt(g[:, 0] ** 2 + g[:, 1] ** 2 + g[:, 2] ** 2 + 1e-12)
        dtau = 0.5 * h_avg / np.maximum(gm, 0.5)
        phi = phi + np.where(mask, 0.0, dtau * sign * (1.0 - gm))
    return phi

def phi_from_regions(coords, cells, regions, scaffold_label=1):
    """domain/mesh_utils.py:367-449 (_init_phi_from_regions) on a P1 mesh whose dofs are its
    vertices: vertices of scaffold cells +1, others -1; interface vertices = in a scaffold
    cell and in another cell; phi = sign * (distance to the nearest interface vertex by a
    KD-tree query, as the reference), or sign * 0.5 without interface vertices."""
    from scipy.spatial import cKDTree

    nv = coords.shape[0]
    scaf = regions == scaffold_label
    sign = np.full(nv, -1.0)
    sign[np.unique(cells[scaf])] = 1.0
    in_s = np.zeros(nv, bool)
    in_f = np.zeros(nv, bool)
    in_s[cells[scaf].ravel()] = True
    in_f[cells[~scaf].ravel()] = True
    iface = np.nonzero(in_s & in_f)[0]
    if iface.size == 0:
        return sign * 0.5
    dist, _ = cKDTree(coords[iface]).query(coords)
    return sign * dist


def under_relax(u_new, u_old, omega):
    """numerics/solvers.py:278-279."""
    return omega * u_new + (1.0 - omega) * u_old


def direct_solve(indptr, indices, data, b):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    n = b.shape[0]
    A = sp.csr_matrix((data, indices, indptr), shape=(n, n))
    return spla.spsolve(A.tocsc(), b)


def transport_steps(coords, cells, coef, D, k, dt, U, steps, rtol=1e-12, lumped=1):
    """Backward-Euler steps of the multi-species transport (numerics/solvers.py:322-372 per
    species, dissolve.py:780-954 species by species): per species the FP64 assembly of
    (1/dt + k_s) M + D_s coef K (gpu_assembler.py:60-139), the RHS M u/dt
    (:176-221) and a Jacobi-PCG solve to ||b - A x|| <= rtol ||b|| from the previous
    state (a tight rtol stands in for the exact solution).  Returns the state after each
    step."""
    detJ, G, _ = geometry(coords, cells)
    ip, ix, sm = csr_pattern(cells, coords.shape[0])
    n = cells.shape[0]
    As = [assemble(detJ, G, D[s] * coef, np.full(n, float(k[s])), 1.0 / dt, lumped, sm,
                   ix.size) for s in range(len(D))]
    U = np.array(U, dtype=np.float64)
    out = []
    for _ in range(steps):
        new = np.empty_like(U)
        for s in range(len(D)):
            b = assemble_rhs(cells, detJ, U[:, s], None, 1.0 / dt, lumped)
            x, _, st, _ = pcg_jacobi(ip, ix, As[s], b, U[:, s], rtol)
            if st != 0:
                raise RuntimeError(f"oracle PCG did not converge (species {s})")
            new[:, s] = x
        U = new
        out.append(U.copy())
    return out


def gyroid_steps(coords, cells, phi, coef, U, steps, dt, eps, D=(1.0, 1.0, 2.6),
                 k=(0.5, 0.0, 0.2), k_orr=2.0, orr=2.0, rate=0.01, gain=0.5, rtol=None):
    """Coupled gyroid-scaffold steps: interface reaction from phi (hv = k_orr H_eps(phi),
    O2 consumption alpha = cell mean of hv, OH- source orr hv c_O2), the three species
    solved one at a time (FP64 assembly, RHS, direct solve, or Jacobi-PCG to rtol when
    given), then phi -= dt rate (1 + gain c_Cl).  Returns (U, phi) after the steps."""
    detJ, G, JT = geometry(coords, cells)
    ip, ix, sm = csr_pattern(cells, coords.shape[0])
    phi, U = np.array(phi, dtype=np.float64), np.array(U, dtype=np.float64)
    n = cells.shape[0]
    for _ in range(steps):
        grad = nodal_gradient(cells, detJ, JT, phi)
        hv, _, f = interface_terms(phi, grad, eps, k_orr, orr, U)
        hv_cell = hv[cells].sum(axis=1) / 4.0
        new = np.empty_like(U)
        for s in range(3):
            alpha = k[s] + (hv_cell if s == 0 else 0.0)
            A = assemble(detJ, G, D[s] * coef, np.broadcast_to(alpha, (n,)), 1.0 / dt, 1, sm,
                         ix.size)
            b = assemble_rhs(cells, detJ, U[:, s], f[:, s] if s == 2 else None, 1.0 / dt, 1)
            if rtol is None:
                new[:, s] = direct_solve(ip, ix, A, b)
            else:
                x, _, st, _ = pcg_jacobi(ip, ix, A, b, U[:, s], rtol)
                if st != 0:
                    raise RuntimeError(f"oracle PCG did not converge (species {s})")
                new[:, s] = x
        U = new
        phi = levelset_advance(phi, U, 1, dt, rate, gain)
    return U, phi

