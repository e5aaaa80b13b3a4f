"""ctypes view of the CPU oracle (oracle/build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, never by the product package.  The oracle is a
single-threaded restatement of the reference's C# solver path; see oracle.h
for the file:line each function follows.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "liboracle.so")
_lib = None

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_vp = C.c_void_p


def build() -> str:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        sig = {
            "or_csr_create": (_vp, [C.c_int32, C.c_int32, _i32p, _i32p, _f64p]),
            "or_csr_free": (None, [_vp]),
            "or_csr_info": (None, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
            "or_csr_copy": (None, [_vp, _i32p, _i32p, _f64p]),
            "or_csr_spmv": (None, [_vp, _f64p, _f64p]),
            "or_csr_spmv_omp": (None, [_vp, _f64p, _f64p]),
            "or_csr_gs_forward": (None, [_vp, _f64p, _f64p]),
            "or_model_create": (_vp, [C.c_int, _i32p, _f64p, C.c_double, C.c_double, C.c_double, _vp]),
            "or_model_free": (None, [_vp]),
            "or_model_num_free": (C.c_int32, [_vp]),
            "or_model_num_all": (C.c_int32, [_vp]),
            "or_model_kff": (_vp, [_vp]),
            "or_model_rhs": (None, [_vp, _f64p]),
            "or_model_uf": (None, [_vp, _f64p]),
            "or_model_free_dofs": (None, [_vp, _i32p]),
            "or_model_element_stiffness": (None, [C.c_int, C.c_double, C.c_double, _f64p]),
            "or_model_row_ratio_bound": (C.c_double, [_vp]),
            "or_traction_rhs": (None, [C.c_int, _i32p, _f64p, _f64p, _f64p]),
            "or_transfer_create": (None, [C.c_int, _i32p, _i32p, C.POINTER(_vp), C.POINTER(_vp)]),
            "or_duvi_encode": (_vp, [_vp, C.c_double, C.c_int]),
            "or_duvi_free": (None, [_vp]),
            "or_duvi_info": (None, [_vp, _i64p]),
            "or_duvi_copy": (None, [_vp, _u32p, _u32p, _u32p, _u8p, _u32p, _f64p]),
            "or_duvi_spmv": (None, [_vp, _f64p, _f64p, C.c_int]),
            "or_duvi_to_dense": (None, [_vp, C.c_int32, _f64p]),
            "or_units_from_csr": (_vp, [_vp, C.c_double]),
            "or_units_from_dense": (_vp, [C.c_int32, C.c_int32, _f64p, C.c_double]),
            "or_units_free": (None, [_vp]),
            "or_units_info": (None, [_vp, _i64p]),
            "or_units_copy": (None, [_vp, _u8p, _i64p, _i32p, _f64p]),
            "or_units_multiply": (None, [_vp, _f64p, _f64p]),
            "or_units_get": (C.c_double, [_vp, C.c_int32, C.c_int32]),
            "or_units_gs": (None, [_vp, _f64p, _f64p]),
            "or_power_bound": (C.c_double, [_vp, _f64p]),
            "or_ldl_factor": (C.c_int, [C.c_int32, _f64p, C.c_double]),
            "or_ldl_solve": (None, [C.c_int32, _f64p, _f64p, _f64p]),
            "or_make_path": (C.c_int32, [_u8p, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
            "or_gmg_create": (_vp, [C.c_int, _i32p, _f64p, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int32,
                                    C.c_int, C.c_double, _u8p, C.c_int32, _i32p, C.c_int32]),
            "or_gmg_free": (None, [_vp]),
            "or_gmg_solve": (None, [_vp, _vp, _f64p, _i32p, _f64p]),
            "or_gmg_num_levels": (C.c_int32, [_vp]),
            "or_gmg_omega_scale": (C.c_double, [_vp, C.c_int32]),
            "or_pcg_jacobi": (C.c_int32, [_vp, _f64p, _f64p, C.c_int32, C.c_double]),
            "or_pcg_jacobi_rel": (C.c_int32, [_vp, _f64p, _f64p, C.c_int32, C.c_double]),
            "or_hex_stiffness": (_vp, [_i32p, _vp, C.c_double, C.c_double, C.c_double]),
            "or_hex_trilinear": (_vp, [_i32p]),
            "or_galerkin": (_vp, [_vp, _vp]),
            "or_mg_fcg": (C.c_int32, [C.c_int32, C.POINTER(_vp), C.POINTER(_vp), C.c_double, C.c_int32, _f64p, _f64p,
                                      C.c_int32, C.c_double, C.POINTER(C.c_double)]),
            "or_adjoint_element_gradient": (None, [_i32p, C.c_double, C.c_double, _f64p, _f64p, _f64p, _f64p]),
            "or_omp_threads": (C.c_int, []),
            "or_set_threads": (None, [C.c_int]),
            "or_last_solve_seconds": (C.c_double, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Csr:
    """Owning handle of an oracle CSR matrix (sorted, int32, float64)."""

    def __init__(self, handle, owned=True):
        self.h = handle
        self.owned = owned
        r, c, n = C.c_int32(), C.c_int32(), C.c_int64()
        lib().or_csr_info(self.h, C.byref(r), C.byref(c), C.byref(n))
        self.shape = (r.value, c.value)
        self.nnz = n.value

    @classmethod
    def from_arrays(cls, n_rows, n_cols, rowptr, col, val):
        h = lib().or_csr_create(n_rows, n_cols, np.ascontiguousarray(rowptr, np.int32),
                                np.ascontiguousarray(col, np.int32), np.ascontiguousarray(val, np.float64))
        return cls(h)

    @classmethod
    def from_scipy(cls, m):
        m = m.tocsr()
        m.sort_indices()
        return cls.from_arrays(m.shape[0], m.shape[1], m.indptr, m.indices, m.data)

    def arrays(self):
        rp = np.empty(self.shape[0] + 1, np.int32)
        col = np.empty(self.nnz, np.int32)
        val = np.empty(self.nnz, np.float64)
        lib().or_csr_copy(self.h, rp, col, val)
        return rp, col, val

    def to_scipy(self):
        import scipy.sparse as sp
        rp, col, val = self.arrays()
        return sp.csr_matrix((val, col, rp), shape=self.shape)

    def spmv(self, x, parallel=False):
        y = np.empty(self.shape[0])
        (lib().or_csr_spmv_omp if parallel else lib().or_csr_spmv)(self.h, np.ascontiguousarray(x, np.float64), y)
        return y

    def gs_forward(self, b, x):
        lib().or_csr_gs_forward(self.h, np.ascontiguousarray(b, np.float64), x)

    def __del__(self):
        if getattr(self, "owned", False) and self.h and _lib is not None:
            _lib.or_csr_free(self.h)
            self.h = None


class Model:
    """FemCantilever2D/3D restatement: Kff (sorted CSR), manufactured b, u_EB."""

    def __init__(self, ne, length=(20.0, 1.0, 1.0), E=1.0, nu=0.3, q=1.0, densities=None):
        self.dim = len(ne)
        ne3 = np.array(list(ne) + [1] * (3 - len(ne)), np.int32)
        self.h = lib().or_model_create(self.dim, ne3, np.array(length, np.float64), E, nu, q,
                                       None if densities is None else _ptr(np.ascontiguousarray(densities, np.float64)))
        self.n_free = lib().or_model_num_free(self.h)
        self.kff = Csr(lib().or_model_kff(self.h), owned=False)
        self.kff._owner = self   # the borrowed handle lives inside this model

    def rhs(self):
        b = np.empty(self.n_free)
        lib().or_model_rhs(self.h, b)
        return b

    def uf(self):
        u = np.empty(self.n_free)
        lib().or_model_uf(self.h, u)
        return u

    def free_dofs(self):
        f = np.empty(self.n_free, np.int32)
        lib().or_model_free_dofs(self.h, f)
        return f

    def row_ratio_bound(self):
        return lib().or_model_row_ratio_bound(self.h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_model_free(self.h)
            self.h = None


def element_stiffness(dim=3, E=1.0, nu=0.3):
    n = 24 if dim == 3 else 8
    ke = np.empty(n * n)
    lib().or_model_element_stiffness(dim, E, nu, ke)
    return ke.reshape(n, n)


def traction_rhs(ne, length, t):
    dim = len(ne)
    ne3 = np.array(list(ne) + [1] * (3 - dim), np.int32)
    nn = [n + 1 for n in ne]
    nfree = dim * int(np.prod(nn)) - dim * int(np.prod(nn[1:]))
    b = np.empty(nfree)
    lib().or_traction_rhs(dim, ne3, np.array(length, np.float64), np.array(t, np.float64), b)
    return b


def transfer(ne_fine, ne_coarse):
    dim = len(ne_fine)
    f = np.array(list(ne_fine) + [1] * (3 - dim), np.int32)
    c = np.array(list(ne_coarse) + [1] * (3 - dim), np.int32)
    R, P = _vp(), _vp()
    lib().or_transfer_create(dim, f, c, C.byref(R), C.byref(P))
    return Csr(R.value), Csr(P.value)


class DuVi:
    """GPU SoA DuVi encoding produced by the oracle encoder."""

    def __init__(self, csr: Csr, tol=1e-10, force_bits=0):
        self.h = lib().or_duvi_encode(csr.h, tol, force_bits)
        s = np.empty(5, np.int64)
        lib().or_duvi_info(self.h, s)
        self.n_rows, self.nblocks, self.nnz, self.nuniq, self.vi_bits = (int(v) for v in s)
        self.n_cols = csr.shape[1]

    def arrays(self):
        rc = np.empty(self.n_rows + 1, np.uint32)
        rd = np.empty(self.n_rows + 1, np.uint32)
        ci = np.empty(self.nblocks, np.uint32)
        dist = np.empty(self.nnz, np.uint8)
        vidx = np.empty(self.nnz, np.uint32)
        vals = np.empty(self.nuniq, np.float64)
        lib().or_duvi_copy(self.h, rc, rd, ci, dist, vidx, vals)
        return dict(row_to_col=rc, row_to_dist=rd, col_idx=ci, dist=dist, vidx=vidx, values=vals)

    def spmv(self, x, y=None, clear=True):
        if y is None:
            y = np.zeros(self.n_rows)
        lib().or_duvi_spmv(self.h, np.ascontiguousarray(x, np.float64), y, 1 if clear else 0)
        return y

    def to_dense(self):
        d = np.empty((self.n_rows, self.n_cols))
        lib().or_duvi_to_dense(self.h, self.n_cols, d)
        return d

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_duvi_free(self.h)
            self.h = None


class Units:
    """CPU DuVi Unit stream (DuViCompressedSparseMatrix)."""

    def __init__(self, handle):
        self.h = handle
        s = np.empty(4, np.int64)
        lib().or_units_info(self.h, s)
        self.n_units, self.n_bytes, self.n_vidx, self.nuniq = (int(v) for v in s)

    @classmethod
    def from_csr(cls, csr: Csr, tol=1e-10):
        return cls(lib().or_units_from_csr(csr.h, tol))

    @classmethod
    def from_dense(cls, dense, tol=1e-10):
        d = np.ascontiguousarray(dense, np.float64)
        return cls(lib().or_units_from_dense(d.shape[0], d.shape[1], d, tol))

    def arrays(self):
        b = np.empty(self.n_bytes, np.uint8)
        off = np.empty(self.n_units + 1, np.int64)
        vi = np.empty(self.n_vidx, np.int32)
        vals = np.empty(self.nuniq, np.float64)
        lib().or_units_copy(self.h, b, off, vi, vals)
        return dict(bytes=b, offsets=off, vidx=vi, values=vals)

    def multiply(self, x, y):
        lib().or_units_multiply(self.h, np.ascontiguousarray(x, np.float64), y)
        return y

    def get(self, r, c):
        return lib().or_units_get(self.h, r, c)

    def gs(self, b, x):
        lib().or_units_gs(self.h, np.ascontiguousarray(b, np.float64), x)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_units_free(self.h)
            self.h = None


def make_path(level_down):
    ld = np.zeros(len(level_down) + 64, np.uint8)
    ld[:len(level_down)] = level_down
    tl, fl = C.c_int32(), C.c_int32()
    m = lib().or_make_path(ld, len(level_down), len(ld), C.byref(tl), C.byref(fl))
    return [bool(v) for v in ld[:m]], tl.value, fl.value


class Gmg:
    """GeometricMultigridSolver (CPU) restatement on the cantilever hierarchy."""

    def __init__(self, ne, length=(20.0, 1.0, 1.0), gauss_seidel=True, duvi=False, max_cycles=2000,
                 coarse_relaxation=False, tol=1e-5, depth=2, level_iterations=4, E=1.0, nu=0.3, level_down=None):
        dim = len(ne)
        ne3 = np.array(list(ne) + [1] * (3 - dim), np.int32)
        if level_down is None:
            level_down = [1] * depth + [0] * depth
        ld = np.array(level_down, np.uint8)
        li = np.atleast_1d(np.array(level_iterations, np.int32))
        self.h = lib().or_gmg_create(dim, ne3, np.array(length, np.float64), E, nu, int(gauss_seidel), int(duvi),
                                     max_cycles, int(coarse_relaxation), tol, ld, len(ld), li, len(li))
        self.n0 = Model(ne, length, E, nu).n_free

    def solve(self, x0=None):
        x = np.empty(self.n0)
        st = np.zeros(3, np.int32)
        res = np.zeros(2)
        lib().or_gmg_solve(self.h, None if x0 is None else _ptr(np.ascontiguousarray(x0, np.float64)), x, st, res)
        return x, dict(cycles=int(st[0]), converged=bool(st[1]), failed=bool(st[2]), max_abs=res[0], norm2=res[1])

    def omega_scale(self, level):
        return lib().or_gmg_omega_scale(self.h, level)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_gmg_free(self.h)
            self.h = None


def pcg_jacobi(csr: Csr, b, max_iter=2000, tol=1e-5, x0=None, rel_l2=False):
    """Jacobi PCG of GMCantileverTests.cs:400-433; rel_l2 stops on ||r||_2 <= tol ||b||_2 instead of
    the reference's max |r_i| <= tol.  Returns (x, iteration index at the stop, -1 if not converged)."""
    x = np.zeros(csr.shape[0]) if x0 is None else np.array(x0, np.float64)
    f = lib().or_pcg_jacobi_rel if rel_l2 else lib().or_pcg_jacobi
    it = f(csr.h, np.ascontiguousarray(b, np.float64), x, max_iter, tol)
    return x, it


def power_bound(csr: Csr, inv_diag):
    return lib().or_power_bound(csr.h, np.ascontiguousarray(inv_diag, np.float64))


def ldl_solve_dense(a, b, tol=1e-15):
    f = np.ascontiguousarray(a, np.float64).copy()
    n = f.shape[0]
    if lib().or_ldl_factor(n, f.reshape(-1), tol) != 0:
        raise ArithmeticError("LDL pivot below tolerance")
    x = np.empty(n)
    lib().or_ldl_solve(n, f.reshape(-1), np.ascontiguousarray(b, np.float64), x)
    return x


def hex_stiffness(ne, elem_E=None, scale=1.0, E=1.0, nu=0.3):
    e = None if elem_E is None else np.ascontiguousarray(elem_E, np.float64)
    return Csr(lib().or_hex_stiffness(np.array(ne, np.int32), _ptr(e), scale, E, nu))


def hex_trilinear(ne_fine):
    return Csr(lib().or_hex_trilinear(np.array(ne_fine, np.int32)))


def galerkin(a: Csr, p: Csr):
    return Csr(lib().or_galerkin(a.h, p.h))


def mg_fcg(A_levels, P_levels, b, omega_eff, nu=2, max_iter=200, tol=1e-8):
    L = len(A_levels)
    Aa = (C.c_void_p * L)(*[a.h for a in A_levels])
    Pa = (C.c_void_p * max(L - 1, 1))(*([p.h for p in P_levels] or [None]))
    x = np.zeros(A_levels[0].shape[0])
    rel = C.c_double()
    it = lib().or_mg_fcg(L, Aa, Pa, omega_eff, nu, np.ascontiguousarray(b, np.float64), x, max_iter, tol,
                         C.byref(rel))
    return x, it, rel.value


def adjoint_element_gradient(ne, rho, u, lam, E=1.0, nu=0.3):
    g = np.empty(int(np.prod(ne)))
    lib().or_adjoint_element_gradient(np.array(ne, np.int32), E, nu, np.ascontiguousarray(rho, np.float64),
                                      np.ascontiguousarray(u, np.float64), np.ascontiguousarray(lam, np.float64), g)
    return g
