"""GPU solvers against the CPU oracle.

Reference-semantics solvers (Jacobi PCG, stationary V-cycle GMG with Jacobi
and Gauss-Seidel) must stop after the same number of iterations as the oracle
(+-1 where the warp-split SpMV reorders sums) and return the same iterate to
1e-8 relative.  The multigrid-preconditioned flexible CG (FP64 and mixed)
must reach the requested FP64 relative residual and agree with the oracle's
FP64 solution to the stated tolerance.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("fmt", ["csr", "duvi"])
def test_pcg_matches_oracle(ctx, native, oracle, fmt):
    m = oracle.Model((16, 4, 4), (20, 1, 1))
    A, b = m.kff.to_scipy(), m.rhs()
    x_ref, it_ref = oracle.pcg_jacobi(m.kff, b, 2000, 1e-8)
    s = native.CudaCsrPcgSolver(ctx, 2000, 1e-8, fmt=fmt).Initialize(A=A, b=b)
    x, st = s.Solve()
    assert st.HasConverged and not st.Failed
    assert abs(st.NumIterationsRequired - it_ref) <= 1
    assert rel(x, x_ref) < 1e-7
    assert st.ResidualMaxNorm <= 1e-8
    # warm start (initialize with x0, CsrCG.cl:191-211)
    x2, st2 = s.Solve(xInitialGuess=x)
    assert st2.NumIterationsRequired <= 1
    s.ReleaseCudaResources()


@pytest.mark.parametrize("fmt", ["csr", "duvi"])
@pytest.mark.parametrize("tol_kind", ["abs_max", "rel_l2"])
def test_pcg_cantilever_16cube_traction_matches_oracle(ctx, native, oracle, fmt, tol_kind):
    """The 16^3 cantilever under unit traction (13,872 dofs), Jacobi-PCG from zero to 1e-8, in CSR
    and in DuVi: the reference's stop test (every |r_i| <= 1e-8) and the relative one
    (||r||_2 <= 1e-8 ||b||_2).  Same system as the oracle's own assembly; iterations within 1,
    solution within 1e-7."""
    ne = (16, 16, 16)
    K = oracle.hex_stiffness(ne)
    b = oracle.traction_rhs(ne, ne, (0.0, 0.0, -1.0))
    rel_l2 = tol_kind == "rel_l2"
    x_ref, it_ref = oracle.pcg_jacobi(K, b, 20000, 1e-8, rel_l2=rel_l2)
    assert it_ref > 0
    A = K.to_scipy()
    s = native.CudaCsrPcgSolver(ctx, 20000, 1e-8, fmt=fmt, tol_kind=tol_kind).Initialize(A=A, b=b)
    x, st = s.Solve()
    s.ReleaseCudaResources()
    assert st.HasConverged and not st.Failed
    assert abs(st.NumIterationsRequired - it_ref) <= 1, (st.NumIterationsRequired, it_ref)
    assert rel(x, x_ref) < 1e-7
    true_rel = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
    assert abs(st.RelativeResidual - true_rel) <= 1e-3 * true_rel
    if rel_l2:
        assert true_rel <= 1.01e-8
    else:
        assert st.ResidualMaxNorm <= 1e-8 and np.max(np.abs(b - A @ x)) <= 1.01e-8


def test_pcg_max_iterations_and_not_initialized(ctx, native, oracle):
    m = oracle.Model((8, 2, 2), (20, 1, 1))
    s = native.CudaCsrPcgSolver(ctx, 3, 1e-14).Initialize(A=m.kff.to_scipy(), b=m.rhs())
    x, st = s.Solve()
    assert not st.HasConverged and st.NumIterationsRequired == 4   # stops when currentIteration > MaxIterations
    s.ReleaseCudaResources()
    with pytest.raises(native.NotInitializedError):
        s.Solve()


def test_pcg_nan_input_fails_not_hangs(ctx, native, oracle):
    m = oracle.Model((8, 2, 2), (20, 1, 1))
    b = m.rhs()
    b[3] = np.nan
    s = native.CudaCsrPcgSolver(ctx, 100, 1e-8).Initialize(A=m.kff.to_scipy(), b=b)
    x, st = s.Solve()
    assert st.Failed and not st.HasConverged


def _levels_from_oracle(oracle, ne, depth):
    A, R, P = [], [], []
    cur = list(ne)
    for d in range(depth + 1):
        A.append(oracle.Model(cur, (20, 1, 1)).kff.to_scipy())
        if d < depth:
            nxt = [v >> 1 if v > 1 else v for v in cur]
            r, p = oracle.transfer(cur, nxt)
            R.append(r.to_scipy())
            P.append(p.to_scipy())
            cur = nxt
    return A, R, P


GMG_CASES = [
    ("jacobi", "csr", False), ("jacobi", "duvi", False), ("gs", "csr", False), ("gs", "duvi", False),
    ("jacobi", "csr", True), ("gs", "duvi", True),
]


@pytest.mark.parametrize("smoother,fmt,coarse_relax", GMG_CASES)
def test_gmg_matches_oracle(ctx, native, oracle, smoother, fmt, coarse_relax):
    ne, depth, li = (16, 4, 4), 2, 4
    gs = smoother == "gs"
    g = oracle.Gmg(ne, (20, 1, 1), gauss_seidel=gs, duvi=(fmt == "duvi"), max_cycles=3000,
                   coarse_relaxation=coarse_relax, tol=1e-5, depth=depth, level_iterations=li)
    x_ref, st_ref = g.solve()
    A, R, P = _levels_from_oracle(oracle, ne, depth)
    cls = native.CudaDuViGeometricMultigridSolver if fmt == "duvi" else native.CudaCsrGeometricMultigridSolver
    s = cls(ctx, 3000, 1e-5, [True] * depth + [False] * depth, [li], GaussSeidel=gs)
    s.b = oracle.Model(ne, (20, 1, 1)).rhs()
    s.initialize_from_levels(A, R, P, coarse_relax)
    x, st, _ = s.Solve()
    assert st.HasConverged == st_ref["converged"] and st.HasConverged
    tolc = 0 if gs else 1
    assert abs(st.NumIterationsRequired - st_ref["cycles"]) <= max(tolc, 1)
    assert rel(x, x_ref) < 1e-6
    if not gs:
        assert abs(s.omega(0) / g.omega_scale(0) - 1) < 1e-12


def test_gmg_multicolor_converges(ctx, native, oracle):
    ne = (16, 4, 4)
    A, R, P = _levels_from_oracle(oracle, ne, 2)
    s = native.CudaCsrGeometricMultigridSolver(ctx, 3000, 1e-5, [True, True, False, False], [4], GaussSeidel=True,
                                               gauss_seidel_ordering="multicolor")
    m = oracle.Model(ne, (20, 1, 1))
    s.b = m.rhs()
    s.initialize_from_levels(A, R, P, False)
    x, st, _ = s.Solve()
    assert st.HasConverged
    u = m.uf()
    assert rel(x, u) < 1e-3


def test_gmg_from_model_interface(ctx, native):
    # CreateDeepV from the product's own model (IGeometricMultigridModel contract)
    model = native.FemCantilever3D((16, 4, 4), (20, 1, 1))
    s = native.CudaDuViGeometricMultigridSolver.CreateDeepV(ctx, model, GaussSeidel=False, maxCircleIterations=3000,
                                                             coarseRelaxation=False, convergenceTolerance=1e-5,
                                                             depth=2, levelIterations=4)
    x, st, times = s.Solve()
    assert st.HasConverged and len(times) == 3
    u = model.free_displacements()
    assert rel(x, u) < 1e-3
    s.ReleaseOpenCLResources()
    with pytest.raises(native.NotInitializedError):
        s.Solve()


def test_gmg_first_level_not_zero_unsupported(ctx, native):
    model = native.FemCantilever3D((8, 2, 2))
    s = native.CudaCsrGeometricMultigridSolver(ctx, 10, 1e-5, [False, True], [2])
    with pytest.raises(native.NotImplementedFeatureError):
        s.Initialize(model)


@pytest.mark.parametrize("precision,fmt", [("f64", "csr"), ("f64", "duvi"), ("mixed", "duvi"), ("mixed", "csr")])
def test_mgpcg_matches_oracle(ctx, native, oracle, precision, fmt):
    ne = (16, 16, 16)
    A, P = native.hex_hierarchy(ne, coarse_ne=4)
    b = native.traction_rhs(ne)
    Ao = [oracle.Csr.from_scipy(a) for a in A]
    Po = [oracle.Csr.from_scipy(p) for p in P]
    s = native.MultigridPcgSolver(ctx, A, P, precision=precision, fmt=fmt, nu=2, omega=2 / 3, omega_mode="spectral",
                                  tol=1e-10, max_iterations=200)
    x, st = s.Solve(b)
    assert st.HasConverged and st.RelativeResidual <= 1e-10
    r = b - A[0] @ x
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10
    x_ref, it_ref, rel_ref = oracle.mg_fcg(Ao, Po, b, 4 / (3 * 3.09), 2, 200, 1e-10)
    assert it_ref > 0
    assert rel(x, x_ref) < 1e-8
    assert st.NumIterationsRequired <= it_ref + 6


def test_mgpcg_absolute_omega_and_nu1(ctx, native):
    ne = (16, 16, 16)
    A, P = native.hex_hierarchy(ne, coarse_ne=4)
    b = native.traction_rhs(ne)
    for nu, mode, om in ((1, "spectral", 2 / 3), (2, "absolute", 0.4), (3, "spectral", 2 / 3)):
        s = native.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", nu=nu, omega=om, omega_mode=mode,
                                      tol=1e-8, max_iterations=300)
        x, st = s.Solve(b)
        assert st.HasConverged and st.RelativeResidual <= 1e-8, (nu, mode)


def test_mgpcg_device_api_and_repeat(ctx, native):
    import torch
    ne = (16, 16, 16)
    A, P = native.hex_hierarchy(ne, coarse_ne=4)
    b = native.traction_rhs(ne)
    s = native.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", tol=1e-8)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros_like(db)
    torch.cuda.synchronize()
    its = []
    for _ in range(3):   # first call eager, later calls through the captured graph
        st = s.solve_device(db.data_ptr(), dx.data_ptr())
        its.append(st.NumIterationsRequired)
        assert st.HasConverged
    assert its[0] == its[1] == its[2]
    x = dx.cpu().numpy()
    assert np.linalg.norm(b - A[0] @ x) / np.linalg.norm(b) <= 1e-8


def test_mgpcg_deterministic_across_solver_lifetimes(ctx, native):
    # Buffers of new solvers reuse memory of destroyed ones; every solve must see
    # fully initialised data (no zero-fill racing the uploads).
    ne = (16, 16, 16)
    A, P = native.hex_hierarchy(ne, coarse_ne=4)
    b = native.traction_rhs(ne)
    seen = {}
    for rep in range(3):
        for nu in (1, 2, 3, 4):
            for fmt, prec in (("duvi", "mixed"), ("csr", "f64")):
                s = native.MultigridPcgSolver(ctx, A, P, precision=prec, fmt=fmt, nu=nu, tol=1e-8, max_iterations=100)
                x, st = s.Solve(b)
                assert st.HasConverged
                key = (nu, fmt, prec)
                seen.setdefault(key, st.NumIterationsRequired)
                assert seen[key] == st.NumIterationsRequired, key
                s.release()
    assert seen[(4, "csr", "f64")] <= 12 and seen[(3, "duvi", "mixed")] <= 13


@pytest.mark.parametrize("smoother,precision,fmt", [("gs_lex", "f64", "csr"), ("gs_lex", "mixed", "duvi"),
                                                    ("gs_color", "mixed", "duvi"), ("gs_color", "f64", "duvi")])
def test_mgpcg_gauss_seidel_smoothing(ctx, native, oracle, smoother, precision, fmt):
    # V(2,2) with forward Gauss-Seidel (the reference's row order, or multicolor) inside the
    # flexible CG: same system, so the solution must match the oracle's FP64 MG-FCG solve,
    # and Gauss-Seidel needs fewer outer iterations than weighted Jacobi.
    ne = (16, 16, 16)
    A, P = native.hex_hierarchy(ne, coarse_ne=4)
    b = native.traction_rhs(ne)
    s = native.MultigridPcgSolver(ctx, A, P, precision=precision, fmt=fmt, nu=2, tol=1e-10, max_iterations=200,
                                  smoother=smoother)
    x, st = s.Solve(b)
    assert st.HasConverged and st.RelativeResidual <= 1e-10
    Ao = [oracle.Csr.from_scipy(a) for a in A]
    Po = [oracle.Csr.from_scipy(p) for p in P]
    x_ref, it_ref, _ = oracle.mg_fcg(Ao, Po, b, 4 / (3 * 3.09), 2, 200, 1e-10)
    assert rel(x, x_ref) < 1e-8
    assert st.NumIterationsRequired < it_ref
    x2, st2 = s.Solve(b)   # graph replay gives the same iterate
    np.testing.assert_array_equal(x, x2)


def test_batch_rejects_gauss_seidel(ctx, native):
    A, P = native.hex_hierarchy((8, 8, 8), coarse_ne=4)
    with pytest.raises(native.NotImplementedFeatureError):
        native.BatchedMultigridSolver(ctx, [(A, P)], smoother="gs_color")


def test_mgpcg_on_uneven_galerkin_meshes(ctx, native):
    # Uneven cantilevers (odd edges, Galerkin levels): node-pattern tables of every size,
    # including ones just under the default shared-memory limit, with reducing epilogues
    # (the power method at set-up) and plain ones.
    for ne in ((29, 25, 19), (19, 35, 15), (46, 29, 9)):
        A, P = native.galerkin_hierarchy(ne, max_coarse_dofs=1000)
        b = native.traction_rhs(ne)
        for prec in ("mixed", "f64"):
            s = native.MultigridPcgSolver(ctx, A, P, precision=prec, fmt="duvi", tol=1e-8, max_iterations=300)
            x, st = s.Solve(b)
            assert st.HasConverged, (ne, prec)
            assert np.linalg.norm(b - A[0] @ x) / np.linalg.norm(b) <= 1e-8
            s.release()


def test_mgpcg_chunk_lengths_do_not_change_the_iterate(ctx, native):
    # Outer iterations run in captured chunks whose length follows the convergence rate
    # seen so far (at most iterations_per_sync); the host reads in between change nothing
    # on the device, so every chunking gives the same iterate bit for bit.
    ne = (16, 16, 16)
    A, P = native.hex_hierarchy(ne, coarse_ne=4)
    b = native.traction_rhs(ne)
    out = []
    for per in (1, 3, 4, 16):
        s = native.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", tol=1e-8, iterations_per_sync=per)
        for _ in range(3):   # the eager first chunk, then a captured graph per chunk length
            x, st = s.Solve(b)
            assert st.HasConverged
            out.append((x, st.NumIterationsRequired))
        s.release()
    for x, it in out[1:]:
        assert it == out[0][1]
        np.testing.assert_array_equal(x, out[0][0])


@pytest.mark.parametrize("precision", ["mixed", "f64"])
def test_mgpcg_device_built_hierarchy_equals_host_built(ctx, native, precision):
    # dv_mgpcg_create_hex assembles and DuVi-encodes the hierarchy on the device: the operators are
    # the host-built ones bit for bit, so the solve returns the same iterate and iteration count.
    ne = (16, 16, 16)
    A, P = native.hex_hierarchy(ne, coarse_ne=4)
    b = native.traction_rhs(ne)
    host = native.MultigridPcgSolver(ctx, A, P, precision=precision, fmt="duvi", tol=1e-10, max_iterations=200)
    dev = native.MultigridPcgSolver.from_hex(ctx, ne, coarse_ne=4, precision=precision, tol=1e-10, max_iterations=200)
    x_h, st_h = host.Solve(b)
    x_d, st_d = dev.Solve(b)
    assert st_h.HasConverged and st_d.HasConverged
    assert st_d.NumIterationsRequired == st_h.NumIterationsRequired
    np.testing.assert_array_equal(x_d, x_h)
    for l in range(len(A) - 1):
        assert dev.omega(l) == host.omega(l)
    host.release()
    dev.release()


def test_mgpcg_tight_tolerance_mixed_and_fp64(ctx, native):
    # The multigrid configuration's 1e-10 runs: the device-built mixed solver (FP32 V-cycle in the
    # FP64 flexible CG, restarts from the FP64 true residual where the recurrence drifts) and the FP64
    # one both reach a true relative residual of 1e-10, in the same number of iterations within one.
    ne = (16, 16, 16)
    A = native.hex_stiffness(ne)
    b = native.traction_rhs(ne)
    res = {}
    for precision in ("mixed", "f64"):
        s = native.MultigridPcgSolver.from_hex(ctx, ne, coarse_ne=4, precision=precision, tol=1e-10,
                                               max_iterations=200)
        x, st = s.Solve(b)
        assert st.HasConverged and st.RelativeResidual <= 1e-10, st
        assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) <= 1e-10
        res[precision] = (x, st.NumIterationsRequired)
        s.release()
    assert abs(res["mixed"][1] - res["f64"][1]) <= 1
    assert rel(res["mixed"][0], res["f64"][0]) < 1e-8


def test_slab_operator_on_device_single_rank(ctx, native, oracle):
    # The slab layer's device path on one rank: the owned rows (all of them here) as a DuVi device
    # matrix, the product through the C ABI, and the slab Jacobi-PCG against the oracle's PCG.
    import torch
    from compressiontests_b200 import slabs
    ne = (8, 6, 7)
    A = native.hex_stiffness(ne)
    op = slabs.SlabOperator(ctx, A, ne, 0, 1, fmt="duvi")
    x = np.random.default_rng(3).standard_normal(A.shape[0])
    y = torch.empty(A.shape[0], dtype=torch.float64, device="cuda")
    op.apply(torch.from_numpy(x).cuda(), y)
    ref = A @ x
    assert np.max(np.abs(y.cpu().numpy() - ref)) <= 1e-12 * np.max(np.abs(A) @ np.abs(x))
    b = native.traction_rhs(ne)
    xs, its, conv = slabs.slab_pcg(op, torch.from_numpy(b).cuda(), 2000, 1e-10, rel_l2=True)
    x_ref, it_ref = oracle.pcg_jacobi(oracle.Csr.from_scipy(A), b, 2000, 1e-10, rel_l2=True)
    assert conv and abs(its - it_ref) <= 1
    assert rel(xs.cpu().numpy(), x_ref) < 1e-7
    op.release()
