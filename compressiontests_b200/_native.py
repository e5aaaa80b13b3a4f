"""ctypes binding of libduvigpu.so (the C ABI in include/duvi_gpu.h).

The shared library is built in-tree (compressiontests_b200/libduvigpu.so).
There is no fallback: if the library is missing the import fails, and every
compute call needs a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libduvigpu.so")

DV_OK = 0
DV_ERR_ARG = -1
DV_ERR_CUDA = -2
DV_ERR_NOT_INITIALIZED = -3
DV_ERR_UNSUPPORTED = -4
DV_ERR_NOMEM = -5
DV_ERR_FORMAT = -6
DV_ERR_NO_DEVICE = -7
DV_ERR_SINGULAR = -8

FORMAT_CSR, FORMAT_DUVI, FORMAT_HEX, FORMAT_TRILINEAR = 0, 1, 2, 3
F64, F32, MIXED = 0, 1, 2
SMOOTHER_JACOBI, SMOOTHER_GS_LEX, SMOOTHER_GS_COLOR = 0, 1, 2
OMEGA_ABSOLUTE, OMEGA_SPECTRAL = 0, 1
TOL_ABS_MAX, TOL_REL_L2 = 0, 1


class DuviError(RuntimeError):
    """A libduvigpu call returned a non-zero status."""

    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


class NotInitializedError(DuviError):
    """Mirrors InvalidOperationException('You must call Initialize(model) first')."""


class NotImplementedFeatureError(DuviError):
    """Mirrors NotImplementedException of the reference (e.g. firstLevel != 0)."""


class NoDeviceError(DuviError):
    pass


class CsrHost(C.Structure):
    _fields_ = [("n_rows", C.c_int32), ("n_cols", C.c_int32), ("rowptr", C.c_void_p), ("col", C.c_void_p),
                ("val", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("failed", C.c_int32),
                ("reserved", C.c_int32), ("residual_max", C.c_double), ("residual_norm2", C.c_double),
                ("relative_residual", C.c_double), ("solve_ms", C.c_double)]


class MatrixInfo(C.Structure):
    _fields_ = [("n_rows", C.c_int32), ("n_cols", C.c_int32), ("nnz", C.c_int64), ("nblocks", C.c_int64),
                ("nuniq", C.c_int64), ("format", C.c_int32), ("precision", C.c_int32),
                ("value_index_bits", C.c_int32), ("kernel_variant", C.c_int32), ("device_bytes", C.c_int64),
                ("row_group", C.c_int32), ("reserved", C.c_int32)]


class GmgConfig(C.Structure):
    _fields_ = [("smoother", C.c_int32), ("format", C.c_int32), ("max_cycles", C.c_int32),
                ("coarse_relaxation", C.c_int32), ("tol", C.c_double), ("n_steps", C.c_int32),
                ("level_down", C.c_void_p), ("n_level_iterations", C.c_int32), ("level_iterations", C.c_void_p),
                ("cycles_per_sync", C.c_int32)]


class MgpcgConfig(C.Structure):
    _fields_ = [("precision", C.c_int32), ("format", C.c_int32), ("outer_format", C.c_int32), ("nu", C.c_int32),
                ("omega", C.c_double), ("omega_mode", C.c_int32), ("max_iterations", C.c_int32),
                ("tol", C.c_double), ("iterations_per_sync", C.c_int32), ("use_graphs", C.c_int32),
                ("smoother", C.c_int32)]


_vp = C.c_void_p
_P = C.POINTER
_SIGNATURES = {
    "dv_status_string": (C.c_char_p, [C.c_int]),
    "dv_last_error": (C.c_char_p, []),
    "dv_version": (C.c_int, []),
    "dv_context_create": (C.c_int, [C.c_int, _P(_vp)]),
    "dv_context_destroy": (C.c_int, [_vp]),
    "dv_context_synchronize": (C.c_int, [_vp]),
    "dv_context_stream": (_vp, [_vp]),
    "dv_context_launch_count": (C.c_int64, [_vp]),
    "dv_matrix_create_csr": (C.c_int, [_vp, _P(CsrHost), C.c_int32, _P(_vp)]),
    "dv_matrix_create_duvi": (C.c_int, [_vp, _P(CsrHost), C.c_int32, C.c_int32, C.c_double, _P(_vp)]),
    "dv_matrix_create_duvi_soa": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp, _vp, _vp, C.c_int64, _vp, C.c_int64, _vp,
                                            C.c_int32, _vp, C.c_int64, C.c_int32, _P(_vp)]),
    "dv_matrix_get_info": (C.c_int, [_vp, _P(MatrixInfo)]),
    "dv_matrix_export_duvi": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dv_matrix_destroy": (C.c_int, [_vp]),
    "dv_spmv": (C.c_int, [_vp, _vp, _vp, C.c_int32]),
    "dv_spmv_device": (C.c_int, [_vp, _vp, _vp, C.c_int32, C.c_int32]),
    "dv_residual_device": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int32]),
    "dv_spmm_device": (C.c_int, [_vp, C.c_int32, _vp, _vp, C.c_int32, C.c_int32]),
    "dv_gmg_create": (C.c_int, [_vp, C.c_int32, _P(CsrHost), _P(CsrHost), _P(CsrHost), _P(GmgConfig), _P(_vp)]),
    "dv_gmg_solve": (C.c_int, [_vp, _vp, _vp, _vp, _P(Stats)]),
    "dv_gmg_omega": (C.c_int, [_vp, C.c_int32, _P(C.c_double)]),
    "dv_gmg_destroy": (C.c_int, [_vp]),
    "dv_pcg_create": (C.c_int, [_vp, _P(CsrHost), C.c_int32, C.c_int32, C.c_double, _P(_vp)]),
    "dv_pcg_solve": (C.c_int, [_vp, _vp, _vp, _vp, _P(Stats)]),
    "dv_pcg_set_tolerance_kind": (C.c_int, [_vp, C.c_int32]),
    "dv_pcg_destroy": (C.c_int, [_vp]),
    "dv_pcg_solve_noalloc": (C.c_int, [_vp, _vp, _vp, C.c_int32, C.c_int32, C.c_double, _P(Stats)]),
    "dv_mgpcg_create": (C.c_int, [_vp, C.c_int32, _P(CsrHost), _P(CsrHost), _P(MgpcgConfig), _P(_vp)]),
    "dv_mgpcg_create_hex": (C.c_int, [_vp, _vp, C.c_double, C.c_double, C.c_int32, _P(MgpcgConfig), _P(_vp)]),
    "dv_mgpcg_solve": (C.c_int, [_vp, _vp, _vp, _P(Stats)]),
    "dv_mgpcg_solve_device": (C.c_int, [_vp, _vp, _vp, _P(Stats)]),
    "dv_mgpcg_omega": (C.c_int, [_vp, C.c_int32, _P(C.c_double)]),
    "dv_mgpcg_solve_multi": (C.c_int, [_vp, C.c_int32, _vp, _vp, _vp, _P(Stats)]),
    "dv_mgpcg_solve_multi_device": (C.c_int, [_vp, C.c_int32, _vp, _vp, _vp, _P(Stats)]),
    "dv_mgpcg_destroy": (C.c_int, [_vp]),
    "dv_batch_create_hex": (C.c_int, [_vp, C.c_int32, _vp, C.c_double, C.c_double, C.c_int32, _P(MgpcgConfig),
                                      _P(_vp)]),
    "dv_batch_create": (C.c_int, [_vp, C.c_int32, _vp, _vp, _vp, _P(MgpcgConfig), _P(_vp)]),
    "dv_batch_info": (C.c_int, [_vp, _P(C.c_int32), _P(C.c_int32), _P(C.c_int32)]),
    "dv_batch_omega": (C.c_int, [_vp, C.c_int32, _P(C.c_double)]),
    "dv_batch_solve": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _P(Stats)]),
    "dv_batch_solve_device": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _P(Stats)]),
    "dv_batch_destroy": (C.c_int, [_vp]),
    "dv_adjoint_create": (C.c_int, [_vp, _vp, _vp, C.c_double, C.c_double, C.c_double, C.c_int32, _P(MgpcgConfig),
                                    _P(_vp)]),
    "dv_adjoint_info": (C.c_int, [_vp, _P(C.c_int32), _P(C.c_int64)]),
    "dv_adjoint_forward": (C.c_int, [_vp, _vp, _vp, _P(Stats)]),
    "dv_adjoint_backward": (C.c_int, [_vp, _vp, _vp, _vp, _P(Stats)]),
    "dv_adjoint_destroy": (C.c_int, [_vp]),
    "dv_hex_element_gradient": (C.c_int, [_vp, _vp, _vp, C.c_double, C.c_double, C.c_double, _vp, _vp, _vp]),
    "dv_hex_csr_size": (C.c_int, [_vp, _P(C.c_int32), _P(C.c_int64)]),
    "dv_hex_assemble": (C.c_int, [_vp, _vp, C.c_double, C.c_double, C.c_double, _vp, _vp, _vp]),
    "dv_matrix_create_duvi_device": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp, _vp, _vp, C.c_int32, C.c_int32,
                                               C.c_double, _P(_vp)]),
    "dv_matrix_create_hex": (C.c_int, [_vp, _vp, _vp, C.c_double, C.c_double, C.c_double, C.c_int32, _P(_vp)]),
    "dv_matrix_create_trilinear": (C.c_int, [_vp, _vp, C.c_int32, C.c_int32, _P(_vp)]),
    "dv_hex_assemble_device": (C.c_int, [_vp, _vp, _vp, C.c_double, C.c_double, C.c_double, _vp, _vp, _vp]),
    "dv_hex_trilinear_size": (C.c_int, [_vp, _P(C.c_int32), _P(C.c_int32), _P(C.c_int64)]),
    "dv_hex_trilinear": (C.c_int, [_vp, _vp, _vp, _vp]),
    "dv_duvi_encode": (C.c_int, [_P(CsrHost), C.c_int32, C.c_double, _P(C.c_int64), _P(C.c_int64), _P(C.c_int32),
                                 _vp, _vp, _vp, _vp, _vp, _vp]),
    "dv_units_encode": (C.c_int, [_P(CsrHost), C.c_double, _P(C.c_int64), _P(C.c_int64), _P(C.c_int64),
                                  _P(C.c_int64), _vp, _vp, _vp, _vp]),
    "dv_units_decode": (C.c_int, [C.c_int32, C.c_int32, _vp, C.c_int64, _vp, C.c_int64, _vp, C.c_int64,
                                  _P(C.c_int64), _vp, _vp, _vp]),
    "dv_galerkin_size": (C.c_int, [_P(CsrHost), _P(CsrHost), _P(C.c_int32), _P(C.c_int64)]),
    "dv_galerkin": (C.c_int, [_P(CsrHost), _P(CsrHost), _vp, _vp, _vp]),
    "dv_cartesian_transfer_size": (C.c_int, [C.c_int32, _vp, _vp, C.c_int32, C.c_int32, _vp, C.c_int32, _vp,
                                             _P(C.c_int64), _P(C.c_int64)]),
    "dv_cartesian_transfer": (C.c_int, [C.c_int32, _vp, _vp, C.c_int32, C.c_int32, _vp, C.c_int32, _vp, _vp, _vp, _vp,
                                        _vp, _vp, _vp]),
}

_lib = None


def lib():
    """Load libduvigpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libduvigpu.so not built at {LIB_PATH}; run __graft_entry__.build() or make -C "
                              "compressiontests_b200/csrc")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGNATURES)


def check(status: int):
    if status == DV_OK:
        return
    msg = lib().dv_last_error().decode(errors="replace")
    cls = {DV_ERR_NOT_INITIALIZED: NotInitializedError, DV_ERR_UNSUPPORTED: NotImplementedFeatureError,
           DV_ERR_NO_DEVICE: NoDeviceError}.get(status, DuviError)
    raise cls(status, msg)


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def csr_host(rowptr, col, val, shape):
    """Build the C view of a CSR matrix; returns (struct, keepalive arrays)."""
    rp = np.ascontiguousarray(rowptr, np.int32)
    ci = np.ascontiguousarray(col, np.int32)
    va = np.ascontiguousarray(val, np.float64)
    h = CsrHost(int(shape[0]), int(shape[1]), ptr(rp), ptr(ci), ptr(va))
    return h, (rp, ci, va)
