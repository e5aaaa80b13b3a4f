"""The allocation-free Jacobi PCG entry point (dv_pcg_solve_noalloc).

For callers that cannot allocate device memory while they solve (a host that
reserved all device memory up front, or a time-critical loop that cannot afford
cudaFree's device-wide synchronisation).  Called through the C ABI, its result must match the allocating entry
point (dv_pcg_solve) on the same matrix and right-hand side, within the
tolerance of the other PCG tests, on two calls in a row: the second call finds
the previous call's data in the shared device array and must not depend on it.
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

REL = 1e-7   # tolerance of test_pcg_matches_oracle


@pytest.mark.parametrize("fmt", ["csr", "duvi"])
def test_noalloc_pcg_matches_allocating_pcg(ctx, native, oracle, fmt):
    import torch
    N = native._native
    m = oracle.Model((16, 4, 4), (20, 1, 1))
    A, b = m.kff.to_scipy(), m.rhs()
    ref = native.CudaCsrPcgSolver(ctx, 2000, 1e-8, fmt=fmt).Initialize(A=A, b=b)
    x_ref, st_ref = ref.Solve()
    assert st_ref.HasConverged
    M = native.SparseMatrix(ctx, A, fmt, "f64")
    db = torch.from_numpy(b).cuda()
    dx = torch.full_like(db, float("nan"))
    torch.cuda.synchronize()
    for call in range(2):
        st = N.Stats()
        # free device memory around the call: the warm (second) call must not allocate
        free_before = torch.cuda.mem_get_info()[0]
        N.check(N.lib().dv_pcg_solve_noalloc(M.h, C.c_void_p(db.data_ptr()), C.c_void_p(dx.data_ptr()), 0, 2000,
                                             1e-8, C.byref(st)))
        free_after = torch.cuda.mem_get_info()[0]
        if call == 1:
            assert free_after == free_before, (free_before, free_after)
        x = dx.cpu().numpy()
        assert st.converged and not st.failed, call
        assert st.iterations == st_ref.NumIterationsRequired, call
        assert np.max(np.abs(x - x_ref)) <= REL * np.max(np.abs(x_ref)), call
        # the relative residual is recomputed in FP64 at exit, as for the allocating solver
        true_rel = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
        assert abs(st.relative_residual - true_rel) <= 1e-3 * true_rel, call
        assert abs(st.relative_residual - st_ref.RelativeResidual) <= 1e-3 * st_ref.RelativeResidual, call
        dx.fill_(float("nan"))   # the next call must not read the old solution
        torch.cuda.synchronize()
    # warm start from the solution: converged at once
    dx.copy_(torch.from_numpy(x_ref))
    torch.cuda.synchronize()
    st = N.Stats()
    N.check(N.lib().dv_pcg_solve_noalloc(M.h, C.c_void_p(db.data_ptr()), C.c_void_p(dx.data_ptr()), 1, 2000, 1e-8,
                                         C.byref(st)))
    assert st.converged and st.iterations <= 1
    ref.ReleaseCudaResources()
    M.release()


def test_noalloc_rejects_systems_above_the_limit(ctx, native):
    import torch
    N = native._native
    n = 131073
    A = sp.identity(n, format="csr") * 2.0
    M = native.SparseMatrix(ctx, A, "csr", "f64")
    db = torch.ones(n, dtype=torch.float64, device="cuda")
    dx = torch.zeros_like(db)
    torch.cuda.synchronize()
    st = N.Stats()
    status = N.lib().dv_pcg_solve_noalloc(M.h, C.c_void_p(db.data_ptr()), C.c_void_p(dx.data_ptr()), 0, 10, 1e-8,
                                          C.byref(st))
    assert status == N.DV_ERR_ARG
    assert b"131072" in N.lib().dv_last_error()
    M.release()
