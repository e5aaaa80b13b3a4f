"""Device context and sparse matrices (CSR and DuVi) behind the C ABI.

Mirrors the matrix side of the reference: the CSR upload of
OpenCLCsrPcgSolver.Initialize (OpenCLCsrPcgSolver.cs:125-130), the GPU DuVi
SoA of OpenCLDuViGeometricMultigridSolver (OpenCLDuViGeometricMultigridSolver.cs:16-31,
753-851) and IMatrix.Multiply of DuViCompressedSparseMatrix
(DuViCompressedSparseMatrix.cs:419-441).
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _native as N


class CudaContext:
    """One CUDA device and one stream (replaces the OpenCL platform/device/queue)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        N.check(N.lib().dv_context_create(device, C.byref(h)))
        self.h = h
        self.device = device
        self._dependents = weakref.WeakSet()

    def register(self, obj):
        """Track an object holding native resources of this context (released first on close)."""
        self._dependents.add(obj)

    @property
    def stream(self):
        return N.lib().dv_context_stream(self.h)

    def synchronize(self):
        N.check(N.lib().dv_context_synchronize(self.h))

    def launch_count(self) -> int:
        return int(N.lib().dv_context_launch_count(self.h))

    def close(self):
        if getattr(self, "h", None):
            for d in list(getattr(self, "_dependents", ())):
                try:
                    d.release()
                except Exception:
                    pass
            N.lib().dv_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _csr_arrays(a):
    """(rowptr, col, val, shape) from a scipy matrix or a (rowptr, col, val, shape) tuple."""
    if hasattr(a, "tocsr"):
        a = a.tocsr()
        a.sort_indices()
        return a.indptr, a.indices, a.data, a.shape
    return a


class SparseMatrix:
    """A device-resident matrix in CSR or DuVi format (FP64 or FP32 values)."""

    def __init__(self, ctx: CudaContext, a, fmt="csr", precision="f64", value_index_bits=0, dedup_tol=1e-10):
        rp, ci, va, shape = _csr_arrays(a)
        host, keep = N.csr_host(rp, ci, va, shape)
        prec = {"f64": N.F64, "f32": N.F32}[precision]
        h = C.c_void_p()
        if fmt == "csr":
            N.check(N.lib().dv_matrix_create_csr(ctx.h, C.byref(host), prec, C.byref(h)))
        elif fmt == "duvi":
            N.check(N.lib().dv_matrix_create_duvi(ctx.h, C.byref(host), prec, value_index_bits, dedup_tol, C.byref(h)))
        else:
            raise ValueError("fmt must be 'csr' or 'duvi'")
        del keep
        self.ctx = ctx
        self.h = h
        ctx.register(self)
        self.shape = (int(shape[0]), int(shape[1]))
        self.format = fmt
        self.precision = precision

    @classmethod
    def duvi_from_device_csr(cls, ctx, n_rows, n_cols, d_rowptr, d_col, d_val, precision="f64", value_index_bits=0,
                             dedup_tol=1e-10):
        """DuVi matrix encoded on the device from device CSR arrays (pointers: int32 rowptr and col,
        float64 values), the same arrays as the host encoder's."""
        self = cls.__new__(cls)
        h = C.c_void_p()
        N.check(N.lib().dv_matrix_create_duvi_device(ctx.h, n_rows, n_cols, d_rowptr, d_col, d_val,
                                                     {"f64": N.F64, "f32": N.F32}[precision], value_index_bits,
                                                     dedup_tol, C.byref(h)))
        self.ctx, self.h, self.shape, self.format, self.precision = ctx, h, (n_rows, n_cols), "duvi", precision
        ctx.register(self)
        return self

    @classmethod
    def hex_operator(cls, ctx, ne, elem_E=None, scale=1.0, E=1.0, nu=0.3, precision="f64"):
        """Matrix-free structured hexahedral stiffness (format "hex"): the operator of
        hex_stiffness(ne, elem_E, scale, E, nu) applied element by element, nothing stored
        but one factor per element."""
        self = cls.__new__(cls)
        nea = np.ascontiguousarray(ne, np.int32)
        e = None if elem_E is None else np.ascontiguousarray(elem_E, np.float64)
        h = C.c_void_p()
        N.check(N.lib().dv_matrix_create_hex(ctx.h, N.ptr(nea), N.ptr(e), scale, E, nu,
                                             {"f64": N.F64, "f32": N.F32}[precision], C.byref(h)))
        n = 3 * int(nea[0]) * (int(nea[1]) + 1) * (int(nea[2]) + 1)
        self.ctx, self.h, self.shape, self.format, self.precision = ctx, h, (n, n), "hex", precision
        ctx.register(self)
        return self

    @classmethod
    def trilinear_transfer(cls, ctx, ne_fine, restriction=False, precision="f64"):
        """Matrix-free trilinear transfer of an even structured grid (format "trilinear"): the
        prolongation hex_trilinear(ne_fine) or, with restriction=True, its transpose, applied
        without storing the matrix (same products bit for bit)."""
        self = cls.__new__(cls)
        nea = np.ascontiguousarray(ne_fine, np.int32)
        h = C.c_void_p()
        N.check(N.lib().dv_matrix_create_trilinear(ctx.h, N.ptr(nea), int(bool(restriction)),
                                                   {"f64": N.F64, "f32": N.F32}[precision], C.byref(h)))
        nf = 3 * int(nea[0]) * (int(nea[1]) + 1) * (int(nea[2]) + 1)
        nc = 3 * (int(nea[0]) // 2) * (int(nea[1]) // 2 + 1) * (int(nea[2]) // 2 + 1)
        self.ctx, self.h, self.format, self.precision = ctx, h, "trilinear", precision
        self.shape = (nc, nf) if restriction else (nf, nc)
        ctx.register(self)
        return self

    @classmethod
    def from_duvi_soa(cls, ctx, n_rows, n_cols, arrays, precision="f64"):
        """Upload pre-encoded DuVi arrays (row_to_col, row_to_dist, col_idx, dist, vidx, values, vi_bits)."""
        self = cls.__new__(cls)
        rc = np.ascontiguousarray(arrays["row_to_col"], np.uint32)
        rd = np.ascontiguousarray(arrays["row_to_dist"], np.uint32)
        ci = np.ascontiguousarray(arrays["col_idx"], np.uint32)
        di = np.ascontiguousarray(arrays["dist"], np.uint8)
        bits = int(arrays["vi_bits"])
        vi = np.ascontiguousarray(arrays["vidx"], {8: np.uint8, 16: np.uint16, 32: np.uint32}[bits])
        vals = np.ascontiguousarray(arrays["values"], np.float64)
        h = C.c_void_p()
        N.check(N.lib().dv_matrix_create_duvi_soa(ctx.h, n_rows, n_cols, N.ptr(rc), N.ptr(rd), N.ptr(ci), len(ci),
                                                  N.ptr(di), len(di), N.ptr(vi), bits, N.ptr(vals), len(vals),
                                                  {"f64": N.F64, "f32": N.F32}[precision], C.byref(h)))
        self.ctx, self.h, self.shape, self.format, self.precision = ctx, h, (n_rows, n_cols), "duvi", precision
        ctx.register(self)
        return self

    def info(self):
        i = N.MatrixInfo()
        N.check(N.lib().dv_matrix_get_info(self.h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in i._fields_}

    def export_duvi(self):
        i = self.info()
        n = self.shape[0]
        out = dict(row_to_col=np.empty(n + 1, np.uint32), row_to_dist=np.empty(n + 1, np.uint32),
                   col_idx=np.empty(i["nblocks"], np.uint32), dist=np.empty(i["nnz"], np.uint8),
                   vidx=np.empty(i["nnz"], np.uint32), values=np.empty(i["nuniq"], np.float64))
        N.check(N.lib().dv_matrix_export_duvi(self.h, *(N.ptr(out[k]) for k in
                                                        ("row_to_col", "row_to_dist", "col_idx", "dist", "vidx",
                                                         "values"))))
        out["vi_bits"] = i["value_index_bits"]
        return out

    def Multiply(self, x, y=None, clear=True):
        """y = A x (clear) or y += A x, host FP64 vectors (IMatrix.Multiply)."""
        x = np.ascontiguousarray(x, np.float64)
        if y is None:
            y = np.zeros(self.shape[0])
        N.check(N.lib().dv_spmv(self.h, N.ptr(x), N.ptr(y), 1 if clear else 0))
        return y

    def multiply_device(self, x_ptr, y_ptr, vec_precision="f64", clear=True):
        N.check(N.lib().dv_spmv_device(self.h, x_ptr, y_ptr, {"f64": N.F64, "f32": N.F32}[vec_precision],
                                       1 if clear else 0))

    def residual_device(self, b_ptr, x_ptr, r_ptr, vec_precision="f64"):
        N.check(N.lib().dv_residual_device(self.h, b_ptr, x_ptr, r_ptr, {"f64": N.F64, "f32": N.F32}[vec_precision]))

    def multiply_many_device(self, k, X_ptr, Y_ptr, vec_precision="f64", clear=True):
        N.check(N.lib().dv_spmm_device(self.h, k, X_ptr, Y_ptr, {"f64": N.F64, "f32": N.F32}[vec_precision],
                                       1 if clear else 0))

    def release(self):
        if getattr(self, "h", None):
            N.lib().dv_matrix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
