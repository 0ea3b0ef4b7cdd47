"""ctypes binding of libdissolve_tp.so (the C ABI in include/dissolve_tp.h).

The library is built in-tree by dissolve_tp.build.  There is no fallback: if the
shared library is missing, importing this module raises, and every entry point
returns a status that `check` turns into an exception carrying tp_last_error().
"""
from __future__ import annotations

import ctypes
import os

from .build import LIB

_c_i64 = ctypes.c_int64
_c_i32 = ctypes.c_int32
_c_dbl = ctypes.c_double
_vp = ctypes.c_void_p

TP_OK = 0
TP_ERR_ARG = 1
TP_ERR_CUDA = 2
TP_ERR_INDEX = 3
TP_ERR_DEGENERATE = 4
TP_ERR_CAPACITY = 5
TP_ERR_NOT_CONVERGED = 6
TP_ERR_BREAKDOWN = 7
TP_ERR_NONFINITE = 8
TP_ERR_TIMEOUT = 9

TP_ASM_FULL = 0
TP_ASM_STIFF = 1
TP_ASM_MASS = 2
TP_MAX_COLS = 4


class TransportError(RuntimeError):
    """A C-ABI call returned a TP_ERR_* status."""

    def __init__(self, status: int, where: str, detail: str):
        super().__init__(f"{where}: {status_string(status)} ({detail})")
        self.status = status


class TpMesh(ctypes.Structure):
    _fields_ = [("n_cells", _c_i64), ("n_verts", _c_i64), ("nnz", _c_i64),
                ("max_row_len", _c_i32), ("max_degree", _c_i32),
                ("cells", _vp), ("coords4", _vp), ("geo", _vp), ("v2c_ptr", _vp),
                ("v2c", _vp), ("v2c_slots", _vp), ("indptr", _vp), ("indices", _vp),
                ("tiles", _vp)]


class TpCsrOp(ctypes.Structure):
    _fields_ = [("n_rows", _c_i64), ("S", _c_i32), ("ld", _c_i32),
                ("indptr", _vp), ("indices", _vp), ("K64", _vp), ("K32", _vp),
                ("M64", _vp), ("M32", _vp), ("diag64", _vp), ("diag32", _vp),
                ("bc_mask", _vp), ("dscale", _c_dbl * 4), ("cscale", _c_dbl * 4),
                ("n_systems", _c_i32), ("sys_row_ptr", _vp)]


class TpCgConfig(ctypes.Structure):
    _fields_ = [("max_it", _c_i32), ("inner_fp32", _c_i32), ("delta", _c_dbl),
                ("group", _c_i32), ("block", _c_i32), ("rows_per_tile", _c_i32),
                ("use_graph_loop", _c_i32)]


class TpSell(ctypes.Structure):
    _fields_ = [("n_rows", _c_i64), ("n_entries", _c_i64), ("slice_ptr", _vp), ("sell_col", _vp),
                ("sK32", _vp), ("sK64", _vp), ("sM32", _vp), ("sM64", _vp)]


class TpMlpInputs(ctypes.Structure):
    _fields_ = [("n_verts", _c_i64), ("S", _c_i32), ("ld", _c_i32), ("U", _vp), ("U_prev", _vp),
                ("phi", _vp), ("normgradphi", _vp), ("opU", _vp), ("opDU", _vp),
                ("logD", _c_dbl * 4), ("k", _c_dbl * 4), ("mean", _c_dbl * 10),
                ("istd", _c_dbl * 10), ("base", _c_i32), ("tc_status", _vp)]


class TpMfcgResult(ctypes.Structure):
    _fields_ = [("status", _c_i32), ("iterations", _c_i32), ("lane_status", _c_i32 * 4),
                ("lane_iters", _c_i32 * 4), ("lane_rnorm", _c_dbl * 4), ("lane_bnorm", _c_dbl * 4)]


class TpCgResult(ctypes.Structure):
    _fields_ = [("status", _c_i32), ("iterations", _c_i32), ("n_reliable", _c_i32),
                ("n_lanes", _c_i32)]


_P = ctypes.POINTER

# name: (restype, argtypes) -- mirrors include/dissolve_tp.h
SIGNATURES = {
    "tp_version": (ctypes.c_int, []),
    "tp_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "tp_last_error": (ctypes.c_char_p, []),
    "tp_device_sm_count": (ctypes.c_int, []),
    "tp_cell_geometry": (ctypes.c_int, [_c_i64, _c_i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                        _vp]),
    "tp_pack_geometry": (ctypes.c_int, [_c_i64, _vp, _vp, _vp, _vp]),
    "tp_setup_scratch_bytes": (ctypes.c_size_t, [_c_i64, _c_i64]),
    "tp_incidence": (ctypes.c_int, [_c_i64, _c_i64, _vp, _vp, _vp, _vp, _P(_c_i32), _vp]),
    "tp_pattern": (ctypes.c_int, [_c_i64, _c_i64, _vp, _vp, _vp, _c_i32, _vp, _vp, _vp,
                                  _P(_c_i64), _P(_c_i32), _vp]),
    "tp_scatter_map": (ctypes.c_int, [_c_i64, _vp, _vp, _vp, _vp, _vp]),
    "tp_incidence_slots": (ctypes.c_int, [_P(TpMesh), _vp, _vp, _vp]),
    "tp_cell_average": (ctypes.c_int, [_c_i64, _vp, _vp, _vp, _vp]),
    "tp_bc_mask": (ctypes.c_int, [_c_i64, _vp, _c_i64, _vp, _vp, _vp]),
    "tp_assemble_csr": (ctypes.c_int, [_P(TpMesh), _vp, _vp, _c_dbl, ctypes.c_int, ctypes.c_int,
                                       _vp, _vp, _vp, _vp]),
    "tp_dirichlet_rows": (ctypes.c_int, [_c_i64, _vp, _c_i64, _vp, _vp, _vp, _vp]),
    "tp_lumped_diag": (ctypes.c_int, [_P(TpMesh), ctypes.c_int, ctypes.c_int, _vp, _P(_c_dbl),
                                      _vp, _vp, _vp, _vp]),
    "tp_assemble_stiffness_diag": (ctypes.c_int, [_P(TpMesh), _vp, ctypes.c_int, ctypes.c_int,
                                                  _vp, _P(_c_dbl), _vp, _vp, _vp, _vp, _vp, _vp,
                                                  _vp, _vp]),
    "tp_lumped_rhs": (ctypes.c_int, [_c_i64, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _c_dbl,
                                     _c_i64, _vp, _P(_c_dbl), _vp, _vp]),
    "tp_assemble_rhs": (ctypes.c_int, [_P(TpMesh), ctypes.c_int, ctypes.c_int, _vp, _vp, _c_dbl,
                                       ctypes.c_int, _c_i64, _vp, _P(_c_dbl), _vp, _vp]),
    "tp_nodal_gradient": (ctypes.c_int, [_P(TpMesh), _vp, _vp, _vp, _vp]),
    "tp_scaffold_volume": (ctypes.c_int, [_P(TpMesh), _vp, _c_dbl, _vp, _vp, _vp]),
    "tp_scaffold_volume_static": (ctypes.c_int, [_P(TpMesh), _vp, _c_dbl, _vp, _vp]),
    "tp_o2_alpha": (ctypes.c_int, [_c_i64, _vp, _vp, _c_dbl, _c_dbl, _vp, _vp]),
    "tp_oh_source": (ctypes.c_int, [_c_i64, _vp, _vp, _vp, _vp, _vp, _c_dbl, _c_dbl, _c_dbl,
                                    _c_dbl, _vp, _vp]),
    "tp_interface_terms": (ctypes.c_int, [_c_i64, _vp, _vp, _c_dbl, _c_dbl, _c_dbl, ctypes.c_int, _vp,
                                          ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "tp_cell_average_col": (ctypes.c_int, [_c_i64, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "tp_levelset_advance": (ctypes.c_int, [_c_i64, _vp, ctypes.c_int, _vp, ctypes.c_int, _c_dbl,
                                           _c_dbl, _c_dbl, _vp]),
    "tp_effective_diffusion": (ctypes.c_int, [_c_i64, _vp, _vp, _c_dbl, _c_dbl, _vp, _vp, _vp, _vp,
                                              _vp, _vp, _vp]),
    "tp_zn_coefficients": (ctypes.c_int, [_c_i64, _vp, _vp, _vp, _c_dbl, _c_dbl, _c_dbl, _vp, _vp,
                                          _vp]),
    "tp_redistance_scratch_bytes": (ctypes.c_size_t, [_c_i64]),
    "tp_redistance": (ctypes.c_int, [_P(TpMesh), _vp, ctypes.c_int, _c_dbl, _c_dbl, _c_dbl, _vp,
                                     _vp]),
    "tp_mean_cell_diameter": (ctypes.c_int, [_P(TpMesh), _vp, _vp, _vp]),
    "tp_phi_from_regions_scratch_bytes": (ctypes.c_size_t, [_c_i64]),
    "tp_phi_from_regions": (ctypes.c_int, [_P(TpMesh), _vp, ctypes.c_int, _vp, _vp, _vp]),
    "tp_advance_state": (ctypes.c_int, [_c_i64, _vp, _vp, _vp, _vp, _vp]),
    "tp_advance_history": (ctypes.c_int, [_c_i64, _vp, _vp, _vp, ctypes.c_int,
                                          _P(ctypes.c_void_p), _P(ctypes.c_void_p), _vp]),
    "tp_axpby": (ctypes.c_int, [_c_i64, _c_dbl, _vp, _c_dbl, _vp, _vp]),
    "tp_pack_columns": (ctypes.c_int, [_c_i64, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "tp_unpack_columns": (ctypes.c_int, [_c_i64, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "tp_matfree_apply": (ctypes.c_int, [_P(TpMesh), ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                        _vp, _P(_c_dbl), _P(_c_dbl), _c_dbl, ctypes.c_int,
                                        ctypes.c_int, _vp, _vp, _vp]),
    "tp_csr_apply": (ctypes.c_int, [_P(TpCsrOp), ctypes.c_int, _vp, _vp, _vp]),
    "tp_csr_images": (ctypes.c_int, [_P(TpCsrOp), _vp, _vp, _vp, _vp, _vp]),
    "tp_guess_project_workspace_doubles": (ctypes.c_size_t, []),
    "tp_guess_project": (ctypes.c_int, [_P(TpCsrOp), _vp, _vp, _vp, _vp, _vp, ctypes.c_int,
                                        _P(ctypes.c_void_p), _P(ctypes.c_void_p), _vp, _vp,
                                        _vp]),
    "tp_cg_workspace_bytes": (ctypes.c_size_t, [_P(TpCsrOp), _P(TpCgConfig)]),
    "tp_cg_create": (ctypes.c_int, [_P(TpCsrOp), _P(TpCgConfig), _vp, _vp, _vp, _vp,
                                    ctypes.c_size_t, _vp, _P(_vp)]),
    "tp_cg_run": (ctypes.c_int, [_vp, _vp]),
    "tp_cg_result_get": (ctypes.c_int, [_vp, _P(TpCgResult), _vp, _vp, _vp, _vp, _vp]),
    "tp_cg_destroy": (ctypes.c_int, [_vp]),
    "tp_cg_time_spmv": (ctypes.c_int, [_vp, ctypes.c_int, _P(ctypes.c_float), _vp]),
    "tp_sell_build": (ctypes.c_int, [_c_i64, _vp, _vp, _vp, _vp, _vp, _P(_c_i64), _vp]),
    "tp_sell_scatter": (ctypes.c_int, [_c_i64, _vp, _vp, _vp, _vp, _vp]),
    "tp_pcg_workspace_bytes": (ctypes.c_size_t, [_P(TpCsrOp), ctypes.c_int]),
    "tp_pcg_create": (ctypes.c_int, [_P(TpCsrOp), _P(TpSell), ctypes.c_int, ctypes.c_int, _c_dbl,
                                     ctypes.c_int, _vp, _vp, _vp, _vp, ctypes.c_size_t, _vp,
                                     _P(_vp)]),
    "tp_pcg_run": (ctypes.c_int, [_vp, _vp]),
    "tp_pcg_result_get": (ctypes.c_int, [_vp, _P(TpCgResult), _vp, _vp, _vp, _vp, _vp]),
    "tp_pcg_grid": (ctypes.c_int, [_vp, _P(ctypes.c_int), _P(ctypes.c_int)]),
    "tp_pcg_engine": (ctypes.c_int, [_vp, _P(ctypes.c_int), _P(ctypes.c_size_t)]),
    "tp_pcg_set_profile": (ctypes.c_int, [_vp, _vp]),
    "tp_tiles_create": (ctypes.c_int, [_P(TpMesh), ctypes.c_int, _vp, _P(_vp)]),
    "tp_tiles_info": (ctypes.c_int, [_vp, _P(_c_i32), _P(_c_i32), _P(_c_i32), _P(_c_i64),
                                     _P(ctypes.c_size_t)]),
    "tp_tiles_destroy": (ctypes.c_int, [_vp]),
    "tp_mfcg_workspace_bytes": (ctypes.c_size_t, [_c_i64, ctypes.c_int]),
    "tp_mfcg_solve": (ctypes.c_int, [_P(TpMesh), ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp,
                                     _c_dbl, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp,
                                     ctypes.c_int, _vp, ctypes.c_size_t, _P(TpMfcgResult), _vp]),
    "tp_pcg_set_wait_limit": (ctypes.c_int, [_vp, ctypes.c_ulonglong, ctypes.c_uint]),
    "tp_pcg_destroy": (ctypes.c_int, [_vp]),
    "tp_mlp_param_count": (ctypes.c_int, []),
    "tp_mlp_tensor_status": (ctypes.c_int, [_P(ctypes.c_int), _vp]),
    "tp_mlp_set_wait_limit": (ctypes.c_int, [ctypes.c_uint, ctypes.c_int]),
    "tp_mlp_predict": (ctypes.c_int, [_P(TpMlpInputs), _vp, ctypes.c_float, _vp, _vp, _vp]),
    "tp_mlp_features": (ctypes.c_int, [_P(TpMlpInputs), _vp, _vp]),
    "tp_mlp_target": (ctypes.c_int, [_c_i64, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _c_dbl,
                                     _vp, _vp]),
    "tp_mlp_grad_workspace_floats": (ctypes.c_size_t, [ctypes.c_int]),
    "tp_mlp_train_step": (ctypes.c_int, [_vp, _vp, _c_i64, _c_i64, _vp, _vp, _vp, ctypes.c_int,
                                         ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                         ctypes.c_float, ctypes.c_float, ctypes.c_int, _vp, _vp,
                                         _vp, _vp]),
}


def _load():
    if not os.path.exists(LIB):
        raise ImportError(
            f"{LIB} is missing: build it with `python -m dissolve_tp.build` "
            "(there is no CPU fallback for the transport path)")
    lib = ctypes.CDLL(LIB)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def status_string(status: int) -> str:
    return lib.tp_status_string(int(status)).decode()


def last_error() -> str:
    return lib.tp_last_error().decode()


def check(rc: int, where: str = "") -> None:
    if rc != TP_OK:
        detail = last_error()
        if rc in (TP_ERR_ARG, TP_ERR_INDEX, TP_ERR_DEGENERATE, TP_ERR_CAPACITY):
            raise ValueError(f"{where}: {status_string(rc)} ({detail})")
        raise TransportError(rc, where, detail)


def call(name: str, *args) -> int:
    rc = getattr(lib, name)(*args)
    check(rc, name)
    return rc
