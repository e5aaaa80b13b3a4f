"""Multi-right-hand-side MG-PCG (k load cases in one solve) on the GPU.

Bar: every load case reaches its own FP64-verified relative residual; each
column agrees with the single-vector solve of the same load case (both at
1e-10) and with the oracle's FP64 MG-FCG solve; iteration counts within one of
the single solves.  The reference solves load cases one after another
(PcgSolver2.InverseSystemMatrixTimesOtherMatrix, PcgSolver2.cs:92-136).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def problem(native):
    ne = (16, 16, 16)
    A, P = native.hex_hierarchy(ne, coarse_ne=4)
    return ne, A, P


@pytest.mark.parametrize("precision,fmt", [("mixed", "duvi"), ("f64", "csr"), ("mixed", "csr"), ("f64", "duvi")])
def test_multi_rhs_matches_single_solves(ctx, native, problem, precision, fmt):
    ne, A, P = problem
    k = 8
    B = native.random_face_loads(ne, k, seed=3)
    s = native.MultigridPcgSolver(ctx, A, P, precision=precision, fmt=fmt, nu=2, tol=1e-10, max_iterations=200)
    X, st, conv = s.solve_many(B)
    assert conv.all() and st.HasConverged and st.RelativeResidual <= 1e-10
    its = []
    for j in range(k):
        r = B[:, j] - A[0] @ X[:, j]
        assert np.linalg.norm(r) / np.linalg.norm(B[:, j]) <= 1e-10
        x1, st1 = s.Solve(B[:, j])
        its.append(st1.NumIterationsRequired)
        assert rel(X[:, j], x1) < 1e-7, j
    assert st.NumIterationsRequired <= max(its) + 1


def test_multi_rhs_matches_oracle(ctx, native, oracle, problem):
    ne, A, P = problem
    B = native.random_face_loads(ne, 3, seed=11)
    Ao = [oracle.Csr.from_scipy(a) for a in A]
    Po = [oracle.Csr.from_scipy(p) for p in P]
    s = native.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", tol=1e-10, max_iterations=200)
    X, st, conv = s.solve_many(B)
    assert conv.all()
    for j in range(3):
        x_ref, it_ref, _ = oracle.mg_fcg(Ao, Po, B[:, j], 4 / (3 * 3.09), 2, 200, 1e-10)
        assert rel(X[:, j], x_ref) < 1e-8
        assert st.NumIterationsRequired <= it_ref + 6


@pytest.mark.parametrize("k", [1, 33, 64])
def test_multi_rhs_widths(ctx, native, problem, k):
    # k = 1 (one lane per row), 33 (two column slots per lane, ragged), 64 (full)
    ne, A, P = problem
    B = native.random_face_loads(ne, k, seed=k)
    s = native.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", tol=1e-8, max_iterations=200)
    X, st, conv = s.solve_many(B)
    assert conv.all() and st.RelativeResidual <= 1e-8
    R = B - A[0] @ X
    assert np.max(np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)) <= 1e-8
    if k == 1:
        x1, st1 = s.Solve(B[:, 0])
        assert abs(st1.NumIterationsRequired - st.NumIterationsRequired) <= 1
        assert rel(X[:, 0], x1) < 1e-6


def test_multi_rhs_zero_and_repeated_columns(ctx, native, problem):
    # a zero load case converges at once with x = 0; identical columns give identical solutions
    ne, A, P = problem
    B = native.random_face_loads(ne, 4, seed=5)
    B[:, 1] = 0.0
    B[:, 3] = B[:, 0]
    s = native.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", tol=1e-8, max_iterations=200)
    X, st, conv = s.solve_many(B)
    assert conv.all()
    assert not X[:, 1].any()
    np.testing.assert_array_equal(X[:, 3], X[:, 0])


def test_multi_rhs_device_api_repeat_and_limits(ctx, native, problem):
    import torch
    ne, A, P = problem
    k = 16
    B = native.random_face_loads(ne, k, seed=9)
    s = native.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", tol=1e-8, max_iterations=200)
    dB = torch.from_numpy(np.ascontiguousarray(B)).cuda()
    dX = torch.zeros_like(dB)
    torch.cuda.synchronize()
    its = []
    for _ in range(3):   # first call eager, later calls replay the captured graph
        st, conv = s.solve_many_device(k, dB.data_ptr(), dX.data_ptr())
        assert conv.all()
        its.append(st.NumIterationsRequired)
    assert its[0] == its[1] == its[2]
    X = dX.cpu().numpy()
    assert np.max(np.linalg.norm(B - A[0] @ X, axis=0) / np.linalg.norm(B, axis=0)) <= 1e-8
    with pytest.raises(native.DuviError):
        s.solve_many(np.zeros((A[0].shape[0], 129)))
    # the single-vector path still works after block solves on the same hierarchy
    x1, st1 = s.Solve(B[:, 0])
    assert st1.HasConverged


def test_multi_rhs_iteration_limit(ctx, native, problem):
    ne, A, P = problem
    B = native.random_face_loads(ne, 4, seed=1)
    s = native.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", tol=1e-14, max_iterations=3)
    X, st, conv = s.solve_many(B)
    assert not st.HasConverged and not conv.any()
    assert st.NumIterationsRequired == 3


@pytest.mark.parametrize("k", [5, 8, 32, 40, 64, 128])
def test_block_grid_stencil_equals_pattern_kernel(ctx, native, rng, k, monkeypatch):
    # FP32 block products of a hex operator on the grid layout: the grid-stencil block kernel
    # (tiles of 8 x 4 nodes streaming z planes, lanes over 32 right-hand sides; the face groups on
    # the pattern kernel) sums each row in the pattern kernel's column order with the same fused
    # multiply-adds, skipping only exact zeros, so both give the same floats.  k = 5 (a block whose
    # rows are not 16-byte multiples) takes the pattern kernel either way.
    import torch
    monkeypatch.setenv("DV_AUTOTUNE", "0")
    A = native.hex_stiffness((20, 9, 13), scale=2.0)
    M = native.SparseMatrix(ctx, A, "duvi", "f32")
    assert M.info()["kernel_variant"] == 303
    X = rng.standard_normal((A.shape[1], k)).astype(np.float32)
    dX = torch.from_numpy(X).cuda()
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("DV_BGRID", flag)
        dY = torch.full((A.shape[0], k), np.nan, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        M.multiply_many_device(k, dX.data_ptr(), dY.data_ptr(), "f32")
        ctx.synchronize()
        out[flag] = dY.cpu().numpy()
    np.testing.assert_array_equal(out["1"], out["0"])
    ref = A @ X.astype(np.float64)
    scale = np.abs(A) @ np.abs(X.astype(np.float64)) + 1e-300
    assert np.max(np.abs(out["1"] - ref) / scale) <= 1e-5


def test_block_grid_stencil_solver_equals_pattern_solver(ctx, native, problem, monkeypatch):
    # The multi-right-hand-side V-cycle on the grid-stencil block kernel gives the same iterates
    # as on the pattern kernel (every block product equal): same iteration count, same solution.
    ne, A, P = problem
    B = native.random_face_loads(ne, 16, seed=5)
    res = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("DV_BGRID", flag)
        s = native.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", nu=2, tol=1e-10, max_iterations=200)
        X, st, conv = s.solve_many(B)
        assert conv.all()
        res[flag] = (X, st.NumIterationsRequired)
        s.release()
    assert res["1"][1] == res["0"][1]
    np.testing.assert_array_equal(res["1"][0], res["0"][0])
