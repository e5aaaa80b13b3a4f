"""Solver classes with the interface of the reference's GPU solvers.

  CudaCsrGeometricMultigridSolver / CudaDuViGeometricMultigridSolver
      <- OpenCLCsrGeometricMultigridSolver / OpenCLDuViGeometricMultigridSolver
         (CreateSimpleV, CreateDeepV, Solve, ReleaseOpenCLResources;
          OpenCLCsrGeometricMultigridSolver.cs:55-83, 334-536)
  CudaCsrPcgSolver <- OpenCLCsrPcgSolver (OpenCLCsrPcgSolver.cs:40-45, 84-218, 250-331)
  MultigridPcgSolver: build-defined FP64 / mixed-precision flexible CG with a
      V-cycle preconditioner, composed from the same kernels.

Solve returns (x, IterativeStatistics, level_times) like
IGeometricMultigridSolver.Solve (IGeometricMultigridSolver.cs:8).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .sparse import CudaContext, _csr_arrays

MAX_CIRCLE_ITERATIONS = 10000   # GeometricMultigridSolver.cs:35


@dataclass
class IterativeStatistics:
    NumIterationsRequired: int
    HasConverged: bool
    ConvergenceCriterion: tuple
    Failed: bool = False
    ResidualMaxNorm: float = float("nan")
    ResidualNorm2: float = float("nan")
    RelativeResidual: float = float("nan")
    SolveMilliseconds: float = float("nan")


def _stats(s: N.Stats, label="max-norm of residual"):
    return IterativeStatistics(int(s.iterations), bool(s.converged), (label, float(s.residual_max)), bool(s.failed),
                               float(s.residual_max), float(s.residual_norm2), float(s.relative_residual),
                               float(s.solve_ms))


def _hosts(mats):
    arr = (N.CsrHost * max(1, len(mats)))()
    keep = []
    for i, m in enumerate(mats):
        rp, ci, va, shape = _csr_arrays(m)
        h, k = N.csr_host(rp, ci, va, shape)
        arr[i] = h
        keep.append(k)
    return arr, keep


def make_path(level_down):
    """MakePath (GeometricMultigridSolver.cs:178-201)."""
    ld = [bool(v) for v in level_down]
    cur, total, first = 0, 1, 0
    for d in ld:
        if d:
            cur += 1
            if cur == total:
                total += 1
        elif cur == 0:
            first += 1
            total += 1
        else:
            cur -= 1
    if cur > first:
        ld += [False] * (cur - first)
    elif cur < first:
        ld += [True] * (first - cur)
    return ld, total, first


class _GeometricMultigridBase:
    FORMAT = N.FORMAT_CSR

    def __init__(self, context: CudaContext, maxCircleIterations, convergenceTolerance, levelDown, levelIterations,
                 GaussSeidel=True, gauss_seidel_ordering="lexicographic", cycles_per_sync=16):
        self.context = context
        self.GaussSeidel = GaussSeidel
        self.LevelDown = list(levelDown)
        self.LevelIterations = [4] if levelIterations is None else list(levelIterations)
        self.MaxIterations = maxCircleIterations
        self.ConvergenceTolerance = convergenceTolerance
        self.ordering = gauss_seidel_ordering
        self.cycles_per_sync = cycles_per_sync
        self.h = None
        self.b = None
        self.LevelDoFs = None

    @classmethod
    def CreateSimpleV(cls, context, model, GaussSeidel=True, maxCircleIterations=MAX_CIRCLE_ITERATIONS,
                      coarseRelaxation=True, convergenceTolerance=1e-6, levelIterations=4, **kw):
        s = cls(context, maxCircleIterations, convergenceTolerance, [True, False], [levelIterations], GaussSeidel, **kw)
        s.Initialize(model, coarseRelaxation)
        return s

    @classmethod
    def CreateDeepV(cls, context, model, GaussSeidel=True, maxCircleIterations=MAX_CIRCLE_ITERATIONS,
                    coarseRelaxation=True, convergenceTolerance=1e-6, depth=2, levelIterations=4, **kw):
        s = cls(context, maxCircleIterations, convergenceTolerance, [True] * depth + [False] * depth,
                [levelIterations], GaussSeidel, **kw)
        s.Initialize(model, coarseRelaxation)
        return s

    def Initialize(self, model, coarseRelaxation=True, rhs=None):
        """Build the level hierarchy from the model (OpenCLCsrGeometricMultigridSolver.cs:145-285)."""
        path, total, first = make_path(self.LevelDown)
        if first != 0:
            raise N.NotImplementedFeatureError(N.DV_ERR_UNSUPPORTED, "firstLevel != 0 is not implementent yet")
        A, R, P = [], [], []
        Am, b = model.CreateLinearSystem()
        self.b = np.asarray(b if rhs is None else rhs, np.float64)
        A.append(Am)
        m = model
        for _ in range(total - 1):
            c = m.CreateCoarserModel()
            r, p = m.transfer_to(c)
            R.append(r)
            P.append(p)
            Ac, _ = c.CreateLinearSystem()
            A.append(Ac)
            m = c
        self.initialize_from_levels(A, R, P, coarseRelaxation, path)

    def initialize_from_levels(self, A, R, P, coarseRelaxation=True, path=None):
        path = self.LevelDown if path is None else path
        ah, ka = _hosts(A)
        rh, kr = _hosts(R)
        ph, kp = _hosts(P)
        ld = np.array(path, np.uint8)
        li = np.array(self.LevelIterations, np.int32)
        smoother = N.SMOOTHER_JACOBI
        if self.GaussSeidel:
            smoother = N.SMOOTHER_GS_LEX if self.ordering == "lexicographic" else N.SMOOTHER_GS_COLOR
        cfg = N.GmgConfig(smoother, self.FORMAT, self.MaxIterations, 1 if coarseRelaxation else 0,
                          self.ConvergenceTolerance, len(ld), N.ptr(ld), len(li), N.ptr(li), self.cycles_per_sync)
        h = C.c_void_p()
        N.check(N.lib().dv_gmg_create(self.context.h, len(A), ah, rh, ph, C.byref(cfg), C.byref(h)))
        del ka, kr, kp
        self.h = h
        self.context.register(self)
        self.LevelDoFs = [a.shape[0] for a in A]

    def omega(self, level):
        w = C.c_double()
        N.check(N.lib().dv_gmg_omega(self.h, level, C.byref(w)))
        return w.value

    def Solve(self, xInitialGuess=None, b=None):
        if self.h is None:
            raise N.NotInitializedError(N.DV_ERR_NOT_INITIALIZED, "You must call Initialize(model) first")
        b = self.b if b is None else np.ascontiguousarray(b, np.float64)
        x = np.empty(self.LevelDoFs[0])
        x0 = None if xInitialGuess is None else np.ascontiguousarray(xInitialGuess, np.float64)
        st = N.Stats()
        N.check(N.lib().dv_gmg_solve(self.h, N.ptr(b), N.ptr(x0), N.ptr(x), C.byref(st)))
        return x, _stats(st), np.zeros(len(self.LevelDoFs))

    def ReleaseCudaResources(self):
        if self.h is not None:
            N.lib().dv_gmg_destroy(self.h)
            self.h = None

    ReleaseOpenCLResources = ReleaseCudaResources
    release = ReleaseCudaResources

    def __del__(self):
        try:
            self.ReleaseCudaResources()
        except Exception:
            pass


class CudaCsrGeometricMultigridSolver(_GeometricMultigridBase):
    FORMAT = N.FORMAT_CSR


class CudaDuViGeometricMultigridSolver(_GeometricMultigridBase):
    FORMAT = N.FORMAT_DUVI


class CudaCsrPcgSolver:
    """Jacobi-preconditioned CG, FP64.  Stop when every |r_i| <= tol (the reference's test,
    tol_kind="abs_max"), or when ||r||_2 <= tol ||b||_2 (tol_kind="rel_l2")."""

    FORMAT = N.FORMAT_CSR

    def __init__(self, context: CudaContext, maxIterations, convergenceTolerance, fmt="csr", tol_kind="abs_max"):
        self.context = context
        self.MaxIterations = maxIterations
        self.ConvergenceTolerance = convergenceTolerance
        self.fmt = N.FORMAT_DUVI if fmt == "duvi" else N.FORMAT_CSR
        if tol_kind not in ("abs_max", "rel_l2"):
            raise ValueError("tol_kind must be 'abs_max' or 'rel_l2'")
        self.tol_kind = N.TOL_REL_L2 if tol_kind == "rel_l2" else N.TOL_ABS_MAX
        self.h = None
        self.DoFs = 0

    def Initialize(self, model=None, A=None, b=None):
        if model is not None:
            A, b = model.CreateLinearSystem()
        (ah, keep) = _hosts([A])
        h = C.c_void_p()
        N.check(N.lib().dv_pcg_create(self.context.h, ah, self.fmt, self.MaxIterations, self.ConvergenceTolerance,
                                      C.byref(h)))
        del keep
        self.h = h
        N.check(N.lib().dv_pcg_set_tolerance_kind(h, self.tol_kind))
        self.context.register(self)
        self.b = None if b is None else np.asarray(b, np.float64)
        self.DoFs = A.shape[0]
        return self

    def Solve(self, xInitialGuess=None, b=None):
        if self.h is None:
            raise N.NotInitializedError(N.DV_ERR_NOT_INITIALIZED, "You must call Initialize(model) first")
        b = self.b if b is None else np.ascontiguousarray(b, np.float64)
        x = np.empty(self.DoFs)
        x0 = None if xInitialGuess is None else np.ascontiguousarray(xInitialGuess, np.float64)
        st = N.Stats()
        N.check(N.lib().dv_pcg_solve(self.h, N.ptr(b), N.ptr(x0), N.ptr(x), C.byref(st)))
        return x, _stats(st)

    def ReleaseCudaResources(self):
        if self.h is not None:
            N.lib().dv_pcg_destroy(self.h)
            self.h = None

    ReleaseOpenCLResources = ReleaseCudaResources
    release = ReleaseCudaResources

    def __del__(self):
        try:
            self.ReleaseCudaResources()
        except Exception:
            pass


class MultigridPcgSolver:
    """Flexible CG preconditioned by a V(nu, nu) cycle (weighted Jacobi, or forward Gauss-Seidel
    in the reference's row order / multicolor with smoother="gs_lex" / "gs_color").

    precision='mixed': FP32 V-cycle (values, vectors, accumulation) inside an
    FP64 outer loop; precision='f64': everything FP64.  Stop: ||r||/||b|| <= tol,
    verified on the true FP64 residual at exit.
    """

    def __init__(self, context: CudaContext, A_levels, P_levels, precision="mixed", fmt="duvi", outer_fmt=None,
                 nu=2, omega=2.0 / 3.0, omega_mode="spectral", tol=1e-8, max_iterations=500, iterations_per_sync=4,
                 use_graphs=True, smoother="jacobi"):
        self.context = context
        ah, ka = _hosts(A_levels)
        ph, kp = _hosts(P_levels)
        cfg = self._config(precision, fmt, outer_fmt, nu, omega, omega_mode, tol, max_iterations, iterations_per_sync,
                           use_graphs, smoother)
        h = C.c_void_p()
        N.check(N.lib().dv_mgpcg_create(context.h, len(A_levels), ah, ph, C.byref(cfg), C.byref(h)))
        del ka, kp
        self.h = h
        context.register(self)
        self.n = A_levels[0].shape[0]

    @staticmethod
    def _config(precision, fmt, outer_fmt, nu, omega, omega_mode, tol, max_iterations, iterations_per_sync, use_graphs,
                smoother):
        f = {"csr": N.FORMAT_CSR, "duvi": N.FORMAT_DUVI}
        sm = {"jacobi": N.SMOOTHER_JACOBI, "gs_lex": N.SMOOTHER_GS_LEX, "gs_color": N.SMOOTHER_GS_COLOR}[smoother]
        return N.MgpcgConfig({"mixed": N.MIXED, "f64": N.F64}[precision], f[fmt], f[outer_fmt or fmt], nu, omega,
                             {"absolute": N.OMEGA_ABSOLUTE, "spectral": N.OMEGA_SPECTRAL}[omega_mode], max_iterations,
                             tol, iterations_per_sync, 1 if use_graphs else 0, sm)

    @classmethod
    def from_hex(cls, context: CudaContext, ne, E=1.0, nu_poisson=0.3, coarse_ne=8, precision="mixed", nu=2,
                 omega=2.0 / 3.0, omega_mode="spectral", tol=1e-8, max_iterations=500, iterations_per_sync=4,
                 use_graphs=True):
        """The solver of hex_hierarchy(ne, coarse_ne) for the uniform cantilever, with the
        hierarchy assembled and DuVi-encoded on the device (same operators, same solves)."""
        self = cls.__new__(cls)
        self.context = context
        cfg = cls._config(precision, "duvi", "duvi", nu, omega, omega_mode, tol, max_iterations, iterations_per_sync,
                          use_graphs, "jacobi")
        h = C.c_void_p()
        nea = np.ascontiguousarray(ne, np.int32)
        N.check(N.lib().dv_mgpcg_create_hex(context.h, N.ptr(nea), E, nu_poisson, coarse_ne, C.byref(cfg), C.byref(h)))
        self.h = h
        context.register(self)
        self.n = 3 * int(nea[0]) * (int(nea[1]) + 1) * (int(nea[2]) + 1)
        return self

    def omega(self, level):
        w = C.c_double()
        N.check(N.lib().dv_mgpcg_omega(self.h, level, C.byref(w)))
        return w.value

    def Solve(self, b):
        b = np.ascontiguousarray(b, np.float64)
        x = np.empty(self.n)
        st = N.Stats()
        N.check(N.lib().dv_mgpcg_solve(self.h, N.ptr(b), N.ptr(x), C.byref(st)))
        return x, _stats(st, "relative residual")

    def solve_device(self, b_ptr, x_ptr):
        st = N.Stats()
        N.check(N.lib().dv_mgpcg_solve_device(self.h, b_ptr, x_ptr, C.byref(st)))
        return _stats(st, "relative residual")

    def solve_many(self, B):
        """Solve k load cases at once: B is n x k (column j = load case j), k <= 128.

        Returns (X, stats, converged) with X n x k and converged a length-k bool array.
        Replaces PcgSolver2.InverseSystemMatrixTimesOtherMatrix (PcgSolver2.cs:92-136),
        which solves the columns one after another.
        """
        B = np.ascontiguousarray(B, np.float64)
        if B.ndim != 2 or B.shape[0] != self.n:
            raise ValueError(f"B must be {self.n} x k")
        k = B.shape[1]
        X = np.empty_like(B)
        conv = np.zeros(k, np.int32)
        st = N.Stats()
        N.check(N.lib().dv_mgpcg_solve_multi(self.h, k, N.ptr(B), N.ptr(X), N.ptr(conv), C.byref(st)))
        return X, _stats(st, "worst relative residual"), conv.astype(bool)

    def solve_many_device(self, k, B_ptr, X_ptr):
        """Device-resident n x k FP64 blocks (row-interleaved); returns (stats, converged)."""
        conv = np.zeros(k, np.int32)
        st = N.Stats()
        N.check(N.lib().dv_mgpcg_solve_multi_device(self.h, k, B_ptr, X_ptr, N.ptr(conv), C.byref(st)))
        return _stats(st, "worst relative residual"), conv.astype(bool)

    def release(self):
        if getattr(self, "h", None) is not None:
            N.lib().dv_mgpcg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class BatchedMultigridSolver:
    """Many independent meshes solved together (block-diagonal levels, one launch per
    operation for all meshes, CUDA-graph-captured iterations).

    meshes: list of (A_levels, P_levels), each as accepted by MultigridPcgSolver; the
    meshes may have different sizes and depths.  Every mesh's coarsest level is solved
    with a dense inverse.  Solve takes and returns one vector per mesh.
    """

    def __init__(self, context: CudaContext, meshes, precision="mixed", fmt="duvi", outer_fmt=None, nu=2,
                 omega=2.0 / 3.0, omega_mode="spectral", tol=1e-8, max_iterations=500, iterations_per_sync=4,
                 use_graphs=True, smoother="jacobi"):
        self.context = context
        f = {"csr": N.FORMAT_CSR, "duvi": N.FORMAT_DUVI}
        sm = {"jacobi": N.SMOOTHER_JACOBI, "gs_lex": N.SMOOTHER_GS_LEX, "gs_color": N.SMOOTHER_GS_COLOR}[smoother]
        cfg = N.MgpcgConfig({"mixed": N.MIXED, "f64": N.F64}[precision], f[fmt], f[outer_fmt or fmt], nu, omega,
                            {"absolute": N.OMEGA_ABSOLUTE, "spectral": N.OMEGA_SPECTRAL}[omega_mode], max_iterations,
                            tol, iterations_per_sync, 1 if use_graphs else 0, sm)
        nm = len(meshes)
        nlev = np.array([len(a) for a, _ in meshes], np.int32)
        keep, a_arrs, p_arrs = [], (C.c_void_p * nm)(), (C.c_void_p * nm)()
        for m, (A, P) in enumerate(meshes):
            if len(P) != len(A) - 1:
                raise ValueError(f"mesh {m}: need len(P) == len(A) - 1")
            ah, ka = _hosts(A)
            ph, kp = _hosts(P)
            keep += [ah, ka, ph, kp]
            a_arrs[m] = C.cast(ah, C.c_void_p)
            p_arrs[m] = C.cast(ph, C.c_void_p)
        h = C.c_void_p()
        N.check(N.lib().dv_batch_create(context.h, nm, N.ptr(nlev), a_arrs, p_arrs, C.byref(cfg), C.byref(h)))
        del keep
        self.h = h
        context.register(self)
        self.sizes = [A[0].shape[0] for A, _ in meshes]
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.n = int(self.offsets[-1])

    @classmethod
    def from_hex(cls, context: CudaContext, dims, E=1.0, nu_poisson=0.3, max_coarse_dofs=1000, precision="mixed",
                 nu=2, omega=2.0 / 3.0, omega_mode="spectral", tol=1e-8, max_iterations=500, iterations_per_sync=4,
                 use_graphs=True):
        """The batch of cantilever_batch's meshes (dims: element counts per mesh) with its Galerkin
        hierarchies built in the library and the finest operators of all meshes applied matrix-free."""
        self = cls.__new__(cls)
        self.context = context
        cfg = MultigridPcgSolver._config(precision, "duvi", "duvi", nu, omega, omega_mode, tol, max_iterations,
                                         iterations_per_sync, use_graphs, "jacobi")
        ne = np.ascontiguousarray(np.asarray(dims, np.int32).reshape(-1))
        h = C.c_void_p()
        N.check(N.lib().dv_batch_create_hex(context.h, len(dims), N.ptr(ne), E, nu_poisson, max_coarse_dofs,
                                            C.byref(cfg), C.byref(h)))
        self.h = h
        context.register(self)
        self.sizes = [3 * int(d[0]) * (int(d[1]) + 1) * (int(d[2]) + 1) for d in dims]
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.n = int(self.offsets[-1])
        return self

    def info(self):
        n, L, k = C.c_int32(), C.c_int32(), C.c_int32()
        N.check(N.lib().dv_batch_info(self.h, C.byref(n), C.byref(L), C.byref(k)))
        return {"n_rows": n.value, "n_levels_max": L.value, "launches_per_chunk": k.value}

    def omega(self, level):
        w = C.c_double()
        N.check(N.lib().dv_batch_omega(self.h, level, C.byref(w)))
        return w.value

    def Solve(self, rhs):
        """rhs: list of per-mesh vectors (or one concatenated vector).  Returns
        (list of solutions, stats, converged per mesh, iterations per mesh)."""
        b = np.ascontiguousarray(np.concatenate(rhs) if isinstance(rhs, (list, tuple)) else rhs, np.float64)
        if b.shape != (self.n,):
            raise ValueError(f"rhs must hold {self.n} values")
        x = np.empty_like(b)
        nm = len(self.sizes)
        conv, its = np.zeros(nm, np.int32), np.zeros(nm, np.int32)
        st = N.Stats()
        N.check(N.lib().dv_batch_solve(self.h, N.ptr(b), N.ptr(x), N.ptr(conv), N.ptr(its), C.byref(st)))
        xs = [x[self.offsets[m]:self.offsets[m + 1]] for m in range(nm)]
        return xs, _stats(st, "worst relative residual"), conv.astype(bool), its

    def solve_device(self, b_ptr, x_ptr):
        nm = len(self.sizes)
        conv, its = np.zeros(nm, np.int32), np.zeros(nm, np.int32)
        st = N.Stats()
        N.check(N.lib().dv_batch_solve_device(self.h, b_ptr, x_ptr, N.ptr(conv), N.ptr(its), C.byref(st)))
        return _stats(st, "worst relative residual"), conv.astype(bool), its

    def release(self):
        if getattr(self, "h", None) is not None:
            N.lib().dv_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
