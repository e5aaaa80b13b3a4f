"""Adjoint sensitivities dJ/drho of a density-parametrised cantilever (GPU).

Model: E_e = rho_e^3 (E0 = 1, nu = 0.3), unit traction on the free face, J = c^T u
with c ~ N(0, 1).  Bars:
  - element kernel bit-exact with the oracle's element gradient on the same u, lambda;
  - full gradient (GPU forward + adjoint solves + kernel) against the CPU FP64
    reference (direct solves, oracle element gradient) to 1e-6 of max |g| (solutions
    to 1e-8; the kernel itself is bit-exact on the GPU's u and lambda);
  - central finite differences, h = 1e-6, on 32 seeded elements, to 1e-5 relative.
    J(rho + h e_i) - J(rho - h e_i) = c^T d with K+ d = (K- - K+) u-, which is the exact
    difference of the two solutions (K+ u+ = K- u- = f) without cancellation.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

pytestmark = pytest.mark.gpu

NE = (12, 6, 6)


def scatter_elem(ne, e):
    """Free-dof indices of element e's 24 local dofs (VTK corner order), -1 where clamped."""
    off = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    a, b, c = e % ne[0], (e // ne[0]) % ne[1], e // (ne[0] * ne[1])
    nx, ny = ne[0] + 1, ne[1] + 1
    idx = []
    for (di, dj, dk) in off:
        i, j, k = a + di, b + dj, c + dk
        for d in range(3):
            idx.append(-1 if i == 0 else 3 * ((i - 1) + (nx - 1) * (j + ny * k)) + d)
    return np.array(idx)


@pytest.fixture(scope="module")
def model(native):
    rng = np.random.default_rng(20261203)
    rho = rng.uniform(0.01, 1.0, int(np.prod(NE)))
    f = native.traction_rhs(NE)
    c = rng.standard_normal(f.shape[0])
    return rho, f, c


def test_element_kernel_bit_exact(ctx, native, oracle, rng):
    import torch
    ne = (6, 4, 5)
    n = 3 * ne[0] * (ne[1] + 1) * (ne[2] + 1)
    rho = rng.uniform(0.01, 1.0, int(np.prod(ne)))
    u, lam = rng.standard_normal(n), rng.standard_normal(n)
    d = [torch.from_numpy(v).cuda() for v in (rho, u, lam)]
    g = torch.zeros(int(np.prod(ne)), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    native.element_gradient_device(ctx, ne, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), g.data_ptr())
    np.testing.assert_array_equal(g.cpu().numpy(), oracle.adjoint_element_gradient(ne, rho, u, lam))


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_gradient_matches_cpu_reference(ctx, native, oracle, model, precision):
    rho, f, c = model
    prob = native.AdjointCantilever(ctx, NE, rho, max_coarse_dofs=300, precision=precision, tol=1e-12)
    u, st = prob.forward(f)
    assert st.HasConverged
    g, st2, lam = prob.backward(c, return_lambda=True)
    assert st2.HasConverged
    K = native.hex_stiffness(NE, rho ** 3).tocsc()
    u_ref = spla.spsolve(K, f)
    lam_ref = spla.spsolve(K, c)
    assert np.linalg.norm(u - u_ref) <= 1e-8 * np.linalg.norm(u_ref)
    assert np.linalg.norm(lam - lam_ref) <= 1e-8 * np.linalg.norm(lam_ref)
    # the kernel on the GPU's own u, lambda is the oracle's element gradient bit for bit ...
    np.testing.assert_array_equal(g, oracle.adjoint_element_gradient(NE, rho, u, lam))
    # ... so the distance to the reference gradient is the solution error alone (moduli span 1e-6..1:
    # element sums of lambda_e^T Ke u_e cancel, 1e-8 in the solutions gives ~1e-7 in single elements)
    g_ref = oracle.adjoint_element_gradient(NE, rho, u_ref, lam_ref)
    assert np.max(np.abs(g - g_ref)) <= 1e-6 * np.max(np.abs(g_ref))


def test_gradient_matches_central_differences(ctx, native, oracle, model):
    rho, f, c = model
    h = 1e-6
    prob = native.AdjointCantilever(ctx, NE, rho, max_coarse_dofs=300, precision="f64", tol=1e-12)
    prob.forward(f)
    g, _ = prob.backward(c)
    ke = oracle.element_stiffness(3, 1.0, 0.3).reshape(24, 24)
    rng = np.random.default_rng(7)
    elems = rng.choice(rho.size, 32, replace=False)
    for e in elems:
        rp, rm = rho.copy(), rho.copy()
        rp[e] += h
        rm[e] -= h
        Kp = native.hex_stiffness(NE, rp ** 3).tocsc()
        Km = native.hex_stiffness(NE, rm ** 3).tocsc()
        um = spla.spsolve(Km, f)
        idx = scatter_elem(NE, e)
        live = idx >= 0
        ue = np.where(live, um[np.maximum(idx, 0)], 0.0)
        rhs = np.zeros_like(f)
        np.add.at(rhs, idx[live], ((rm[e] ** 3 - rp[e] ** 3) * (ke @ ue))[live])
        d = spla.spsolve(Kp, rhs)
        fd = c @ d / (2 * h)
        assert abs(fd - g[e]) <= 1e-5 * abs(fd) + 1e-9 * np.max(np.abs(g)), (e, fd, g[e])


def test_backward_before_forward_and_repeat(ctx, native, model):
    rho, f, c = model
    prob = native.AdjointCantilever(ctx, NE, rho, max_coarse_dofs=300, precision="mixed", tol=1e-10)
    with pytest.raises(native.NotInitializedError):
        prob.backward(c)
    u1, _ = prob.forward(f)
    g1, _ = prob.backward(c)
    u2, _ = prob.forward(f)
    g2, _ = prob.backward(c)
    np.testing.assert_array_equal(u1, u2)
    np.testing.assert_array_equal(g1, g2)
    # J is linear in c: the gradient of (2c)^T u is twice the gradient
    g3, _ = prob.backward(2 * c)
    assert np.max(np.abs(g3 - 2 * g1)) <= 1e-8 * np.max(np.abs(g1))


def test_autograd_function(ctx, native, model):
    import torch
    rho, f, c = model
    Solve = native.cantilever_solve_function()
    r = torch.from_numpy(rho).requires_grad_(True)
    u = Solve.apply(r, torch.from_numpy(f), ctx, NE, {"max_coarse_dofs": 300, "tol": 1e-12})
    J = (torch.from_numpy(c) * u).sum()
    J.backward()
    prob = native.AdjointCantilever(ctx, NE, rho, max_coarse_dofs=300, tol=1e-12)
    prob.forward(f)
    g, _ = prob.backward(c)
    assert np.max(np.abs(r.grad.numpy() - g)) <= 1e-9 * np.max(np.abs(g))


@pytest.mark.slow
@pytest.mark.skipif(not __import__("os").environ.get("DV_FULL_ADJOINT"),
                    reason="96x48x48 check builds 2 solvers per probed element (minutes); set DV_FULL_ADJOINT=1")
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_full_size_gradient_central_differences(ctx, native, oracle, precision):
    # 96 x 48 x 48 elements, rho ~ U[0.01, 1] (seeded), E = rho^3, unit traction, J = c^T u.
    # The probes solve on the GPU: u- with K(rho - h e_i), then d = u+ - u- from
    # K(rho + h e_i) d = (K- - K+) u-, each with its own solver.
    ne = (96, 48, 48)
    rng = np.random.default_rng(20261203)
    rho = rng.uniform(0.01, 1.0, int(np.prod(ne)))
    f = native.traction_rhs(ne)
    c = rng.standard_normal(f.shape[0])
    h = 1e-6
    opts = dict(max_coarse_dofs=2000, precision=precision, tol=1e-12, max_iterations=2000)
    prob = native.AdjointCantilever(ctx, ne, rho, **opts)
    u, st = prob.forward(f)
    assert st.HasConverged
    g, st2 = prob.backward(c)
    assert st2.HasConverged
    prob.release()
    ke = oracle.element_stiffness(3, 1.0, 0.3).reshape(24, 24)
    elems = np.random.default_rng(7).choice(rho.size, 32, replace=False)
    worst = 0.0
    for e in elems:
        rp, rm = rho.copy(), rho.copy()
        rp[e] += h
        rm[e] -= h
        pm = native.AdjointCantilever(ctx, ne, rm, **dict(opts, precision="f64"))
        um, _ = pm.forward(f)
        pm.release()
        idx = scatter_elem(ne, e)
        live = idx >= 0
        ue = np.where(live, um[np.maximum(idx, 0)], 0.0)
        rhs = np.zeros_like(f)
        np.add.at(rhs, idx[live], ((rm[e] ** 3 - rp[e] ** 3) * (ke @ ue))[live])
        pp = native.AdjointCantilever(ctx, ne, rp, **dict(opts, precision="f64"))
        d, _ = pp.forward(rhs)
        pp.release()
        fd = c @ d / (2 * h)
        err = abs(fd - g[e]) / (abs(fd) + 1e-4 * np.max(np.abs(g)))
        worst = max(worst, err)
        assert err <= 1e-5, (e, fd, g[e])
    print(f"full-size FD check ({precision}): worst relative error {worst:.2e} over 32 elements")
