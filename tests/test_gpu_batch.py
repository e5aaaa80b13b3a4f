"""Batched MG-PCG over independent meshes of uneven sizes and depths (GPU).

Bar: every mesh reaches its own FP64-verified relative residual; each mesh's
solution agrees with the oracle's FP64 MG-FCG solve of that mesh alone and
with the single-mesh GPU solver (all at 1e-10); results come back in the
caller's mesh order although the batch reorders meshes by depth inside.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIMS = [(5, 3, 4), (12, 6, 10), (8, 8, 8), (4, 4, 4), (7, 9, 5), (16, 5, 3)]


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def batch(native):
    meshes = [native.galerkin_hierarchy(ne, max_coarse_dofs=200) for ne in DIMS]
    rhs = [native.traction_rhs(ne) for ne in DIMS]
    return meshes, rhs


def test_depths_differ(batch):
    meshes, _ = batch
    assert len({len(A) for A, _ in meshes}) >= 2


@pytest.mark.parametrize("precision,fmt", [("mixed", "duvi"), ("f64", "csr"), ("mixed", "csr"), ("f64", "duvi")])
def test_batch_matches_oracle_and_single_solves(ctx, native, oracle, batch, precision, fmt):
    meshes, rhs = batch
    s = native.BatchedMultigridSolver(ctx, meshes, precision=precision, fmt=fmt, tol=1e-10, max_iterations=300)
    xs, st, conv, its = s.Solve(rhs)
    assert conv.all() and st.HasConverged and st.RelativeResidual <= 1e-10
    for m, ((A, P), b, x) in enumerate(zip(meshes, rhs, xs)):
        assert np.linalg.norm(b - A[0] @ x) / np.linalg.norm(b) <= 1e-10, m
        Ao = [oracle.Csr.from_scipy(a) for a in A]
        Po = [oracle.Csr.from_scipy(p) for p in P]
        x_ref, it_ref, _ = oracle.mg_fcg(Ao, Po, b, 4 / (3 * 3.09), 2, 300, 1e-10)
        assert rel(x, x_ref) < 1e-8, m
        assert 1 <= its[m] <= st.NumIterationsRequired
    if precision == "mixed" and fmt == "duvi":
        for m in (0, 2):
            A, P = meshes[m]
            one = native.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", tol=1e-10, max_iterations=300)
            x1, st1 = one.Solve(rhs[m])
            assert rel(xs[m], x1) < 1e-8
            assert abs(st1.NumIterationsRequired - its[m]) <= 3


def test_batch_random_loads_zero_mesh_and_repeat(ctx, native, batch):
    import torch
    meshes, rhs = batch
    rng = np.random.default_rng(4)
    loads = [rng.standard_normal(A[0].shape[0]) for A, _ in meshes]
    loads[3][:] = 0.0
    s = native.BatchedMultigridSolver(ctx, meshes, precision="mixed", fmt="duvi", tol=1e-8)
    b = torch.from_numpy(np.concatenate(loads)).cuda()
    x = torch.zeros_like(b)
    torch.cuda.synchronize()
    seen = []
    for _ in range(3):   # eager first chunk, then graph replays
        st, conv, its = s.solve_device(b.data_ptr(), x.data_ptr())
        assert conv.all()
        seen.append(its.copy())
    assert all((a == seen[0]).all() for a in seen)
    xs = np.split(x.cpu().numpy(), s.offsets[1:-1])
    assert not xs[3].any() and seen[0][3] == 0
    for m, (A, _) in enumerate(meshes):
        if m != 3:
            assert np.linalg.norm(loads[m] - A[0] @ xs[m]) / np.linalg.norm(loads[m]) <= 1e-8
    info = s.info()
    assert info["n_rows"] == s.n and info["n_levels_max"] == max(len(A) for A, _ in meshes)
    assert info["launches_per_chunk"] > 0


def test_batch_iteration_limit_and_single_mesh(ctx, native, batch):
    meshes, rhs = batch
    s = native.BatchedMultigridSolver(ctx, meshes, precision="mixed", fmt="duvi", tol=1e-14, max_iterations=2)
    xs, st, conv, its = s.Solve(rhs)
    assert not st.HasConverged and st.NumIterationsRequired == 2 and not conv.all()
    one = native.BatchedMultigridSolver(ctx, meshes[2:3], precision="f64", fmt="csr", tol=1e-9)
    xs, st, conv, its = one.Solve(rhs[2:3])
    assert conv.all()
    A = meshes[2][0][0]
    assert np.linalg.norm(rhs[2] - A @ xs[0]) / np.linalg.norm(rhs[2]) <= 1e-9


@pytest.mark.parametrize("precision", ["mixed", "f64"])
def test_batch_from_hex_matrix_free_finest_level(ctx, native, oracle, batch, precision):
    # dv_batch_create_hex: the same meshes and Galerkin hierarchies built in the library, the finest
    # operators of all meshes applied matrix-free in one launch (a table of meshes, some with a
    # single level): every mesh's solution matches the oracle's FP64 MG-FCG solve at 1e-10.
    meshes, rhs = batch
    s = native.BatchedMultigridSolver.from_hex(ctx, DIMS, max_coarse_dofs=200, precision=precision, tol=1e-10,
                                               max_iterations=300)
    xs, st, conv, its = s.Solve(rhs)
    assert conv.all() and st.HasConverged and st.RelativeResidual <= 1e-10
    for m, ((A, P), b, x) in enumerate(zip(meshes, rhs, xs)):
        assert np.linalg.norm(b - A[0] @ x) / np.linalg.norm(b) <= 1e-10, m
        Ao = [oracle.Csr.from_scipy(a) for a in A]
        Po = [oracle.Csr.from_scipy(p) for p in P]
        x_ref, _, _ = oracle.mg_fcg(Ao, Po, b, 4 / (3 * 3.09), 2, 300, 1e-10)
        assert rel(x, x_ref) < 1e-8, m
    s.release()
