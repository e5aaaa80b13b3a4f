"""Adjoint sensitivities of a density-parametrised hexahedral cantilever.

Forward/Backward pair over the C ABI (dv_adjoint_*): forward solves
u = K(rho)^-1 f with the multigrid-preconditioned CG; backward takes dJ/du,
solves K lambda = dJ/du with the same solver (K is symmetric) and returns
dJ/drho_e = -penal rho_e^(penal-1) lambda_e^T Ke u_e from an element kernel.
CantileverSolve wraps the pair as a torch.autograd.Function.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .solvers import _stats
from .sparse import CudaContext


class AdjointCantilever:
    """K(rho) = sum_e rho_e^penal Ke(E0, nu) on an ne grid of unit cubes (x = 0 clamped)."""

    def __init__(self, context: CudaContext, ne, rho, penal=3.0, E0=1.0, nu=0.3, max_coarse_dofs=2000,
                 precision="f64", fmt="duvi", tol=1e-10, max_iterations=1000, nu_smooth=2, omega=2.0 / 3.0):
        self.context = context
        self.ne = tuple(int(v) for v in ne)
        rho = np.ascontiguousarray(rho, np.float64)
        if rho.shape != (int(np.prod(self.ne)),):
            raise ValueError("rho needs one density per element (x fastest)")
        f = {"csr": N.FORMAT_CSR, "duvi": N.FORMAT_DUVI}[fmt]
        cfg = N.MgpcgConfig({"mixed": N.MIXED, "f64": N.F64}[precision], f, f, nu_smooth, omega, N.OMEGA_SPECTRAL,
                            max_iterations, tol, 4, 1)
        h = C.c_void_p()
        nea = np.array(self.ne, np.int32)
        N.check(N.lib().dv_adjoint_create(context.h, N.ptr(nea), N.ptr(rho), penal, E0, nu, max_coarse_dofs,
                                          C.byref(cfg), C.byref(h)))
        self.h = h
        context.register(self)
        n, ne_ = C.c_int32(), C.c_int64()
        N.check(N.lib().dv_adjoint_info(h, C.byref(n), C.byref(ne_)))
        self.n_dofs, self.n_elements = n.value, ne_.value

    def forward(self, f):
        f = np.ascontiguousarray(f, np.float64)
        u = np.empty(self.n_dofs)
        st = N.Stats()
        N.check(N.lib().dv_adjoint_forward(self.h, N.ptr(f), N.ptr(u), C.byref(st)))
        return u, _stats(st, "relative residual")

    def backward(self, dJdu, return_lambda=False):
        g = np.ascontiguousarray(dJdu, np.float64)
        grad = np.empty(self.n_elements)
        lam = np.empty(self.n_dofs) if return_lambda else None
        st = N.Stats()
        N.check(N.lib().dv_adjoint_backward(self.h, N.ptr(g), N.ptr(grad), N.ptr(lam), C.byref(st)))
        return (grad, _stats(st, "relative residual")) + ((lam,) if return_lambda else ())

    def release(self):
        if getattr(self, "h", None) is not None:
            N.lib().dv_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def element_gradient_device(context: CudaContext, ne, rho_ptr, u_ptr, lam_ptr, grad_ptr, penal=3.0, E0=1.0, nu=0.3):
    """The element kernel alone on device pointers (FP64)."""
    nea = np.array(ne, np.int32)
    N.check(N.lib().dv_hex_element_gradient(context.h, N.ptr(nea), C.c_void_p(rho_ptr), penal, E0, nu,
                                            C.c_void_p(u_ptr), C.c_void_p(lam_ptr), C.c_void_p(grad_ptr)))


def cantilever_solve_function():
    """torch.autograd.Function: u = CantileverSolve.apply(rho, f, context, ne, options) with
    d(u)/d(rho) through the adjoint (returns the class; torch is imported on use)."""
    import torch

    class CantileverSolve(torch.autograd.Function):
        @staticmethod
        def forward(ctx, rho, f, context, ne, options=None):
            prob = AdjointCantilever(context, ne, rho.detach().cpu().numpy(), **(options or {}))
            u, _ = prob.forward(f.detach().cpu().numpy())
            ctx.prob = prob
            return torch.from_numpy(u).to(rho.device)

        @staticmethod
        def backward(ctx, grad_u):
            grad, _ = ctx.prob.backward(grad_u.detach().cpu().numpy())
            ctx.prob.release()
            return torch.from_numpy(grad).to(grad_u.device), None, None, None, None

    return CantileverSolve
