"""The CPU oracle against the reference's own known answers and invariants.

The reference (C#, MSolve NuGet packages) cannot run here, so the oracle is
pinned by (1) the known-answer tests of the reference's test project, read as
text, (2) the manufactured-solution property of its cantilever model
(b = K u_EB, so a converged solve returns u_EB), and (3) structural invariants
of the element stiffness (symmetry, rigid-body null space).  tests/golden/
holds oracle outputs of small cases, regenerated by tests/golden/make_golden.py,
so that any later change of the oracle shows up.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "oracle_small.npz")


def test_duvi_dense_and_csr_kat(oracle):
    # CompressedSparseMatrixTests.cs:15-39 (also checks mat2, which the reference builds but never multiplies)
    w, h = 1024, 2
    el = np.zeros(w * h)
    el[5] = 1; el[6] = 1; el[8] = 1; el[w - 24] = 2; el[w - 1] = 2
    el[w + 50] = 3; el[w + w - 4] = 3
    m1 = oracle.Units.from_dense(el.reshape(h, w), 1e-10)
    csr = oracle.Csr.from_arrays(2, w, [0, 5, 7], [5, 6, 8, w - 24, w - 1, 50, w - 4], [1, 1, 1, 2, 2, 3, 3.0])
    m2 = oracle.Units.from_csr(csr, 1e-10)
    x = el[:w].copy()
    y1 = m1.multiply(x, np.zeros(2))
    y2 = m2.multiply(x, np.zeros(2))
    assert y1[0] == 11 and y1[1] == 0 and y2[0] == 11 and y2[1] == 0
    np.testing.assert_array_equal(m1.arrays()["bytes"], m2.arrays()["bytes"])
    # element lookup (DuViCompressedSparseMatrix indexer, :450-484)
    assert m1.get(0, 1000) == 2 and m1.get(0, 7) == 0 and m1.get(1, 1020) == 3


def test_diagonal_csr_kat(oracle):
    # GMCantileverOpenCLTests.cs:16-52: 16x16 diagonal, y_i = v_i^2 exactly
    v = np.arange(16, 0, -1.0)
    d = oracle.Csr.from_arrays(16, 16, np.arange(17), np.arange(16), v)
    np.testing.assert_array_equal(d.spmv(v), v * v)
    np.testing.assert_array_equal(oracle.DuVi(d).spmv(v), v * v)


@pytest.mark.parametrize("dim", [2, 3])
def test_element_stiffness_rigid_body_modes(oracle, dim):
    ke = oracle.element_stiffness(dim)
    assert np.array_equal(ke, ke.T)
    if dim == 3:
        pts = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)], float)
        modes = [np.tile(np.eye(3)[a], 8) for a in range(3)] + [np.cross(np.eye(3)[a], pts).ravel() for a in range(3)]
    else:
        pts = np.array([(0, 0), (1, 0), (1, 1), (0, 1)], float)
        modes = [np.tile([1, 0], 4), np.tile([0, 1], 4), np.column_stack([-pts[:, 1], pts[:, 0]]).ravel()]
    for m in modes:
        assert np.abs(ke @ m).max() < 1e-14
    ev = np.linalg.eigvalsh(ke)
    assert ev.min() > -1e-14 and np.sum(ev > 1e-10) == ke.shape[0] - len(modes)


@pytest.mark.parametrize("ne", [(4, 2, 2), (5, 3, 2), (6, 4, 4)])
def test_rowwise_assembly_equals_dok(oracle, ne):
    a1 = oracle.Model(ne, (20, 1, 1)).kff.arrays()
    a2 = oracle.hex_stiffness(ne).arrays()
    for p, q in zip(a1, a2):
        np.testing.assert_array_equal(p, q)
    n = ne[0] * (ne[1] + 1) * (ne[2] + 1) * 3
    nnz = 9 * (3 * ne[0] - 2) * (3 * ne[1] + 1) * (3 * ne[2] + 1) if ne[0] > 1 else None
    assert len(a1[0]) == n + 1


def test_nnz_formula_cube(oracle):
    N = 4
    a = oracle.hex_stiffness((N, N, N))
    assert a.shape[0] == 3 * N * (N + 1) ** 2
    assert a.nnz == 9 * (3 * N - 2) * (3 * N + 1) ** 2


@pytest.mark.parametrize("ne", [(16, 4, 4), (8, 2, 2)])
def test_manufactured_solution_recovered(oracle, ne):
    # FemCantileverBase.cs:53-62: b = Kff * u_EB, so the exact solution is u_EB
    m = oracle.Model(ne, (20, 1, 1))
    x, it = oracle.pcg_jacobi(m.kff, m.rhs(), 20000, 1e-12)
    assert it >= 0
    u = m.uf()
    assert np.abs(x - u).max() <= 1e-9 * np.abs(u).max()


def test_manufactured_solution_2d(oracle):
    m = oracle.Model((32, 4), (20, 1, 1))
    x, it = oracle.pcg_jacobi(m.kff, m.rhs(), 20000, 1e-12)
    u = m.uf()
    assert it >= 0 and np.abs(x - u).max() <= 1e-9 * np.abs(u).max()


def test_trilinear_transfer_equals_reference_weights(oracle):
    # At factor 2 the normalised radial interpolation reduces to trilinear weights
    ne = (4, 4, 4)
    R, P = oracle.transfer(ne, (2, 2, 2))
    T = oracle.hex_trilinear(ne)
    np.testing.assert_allclose(P.to_scipy().toarray(), T.to_scipy().toarray(), atol=1e-15)
    # restriction rows sum to 1 in the interior (before fixed dofs were removed)
    r = R.to_scipy()
    s = np.asarray(r.sum(axis=1)).ravel()
    assert np.all(s <= 1 + 1e-12) and np.isclose(s.max(), 1.0)


@pytest.mark.parametrize("ne", [(4, 4, 4), (5, 3, 4), (7, 9, 1)])
def test_trilinear_reproduces_linear_fields(oracle, ne):
    # Vertex coarsening per axis: coarse nodes at the even fine nodes and at the last
    # one.  Interpolating a linear field given at the coarse nodes must reproduce it
    # exactly at every fine node (odd counts included).
    def axis(n):
        return np.array(sorted(set(range(0, n + 1, 2)) | {n}), float)
    cx, cy, cz = axis(ne[0]), axis(ne[1]), axis(ne[2])
    fx, fy, fz = np.arange(ne[0] + 1.0), np.arange(ne[1] + 1.0), np.arange(ne[2] + 1.0)

    def field(xs, ys, zs, d):
        Z, Y, X = np.meshgrid(zs, ys, xs[1:], indexing="ij")   # x = 0 nodes are clamped
        f = np.stack([1 + 2 * X - Y + 0.5 * Z, -X + 3 * Z, 0.25 * Y + X], axis=-1)
        return f.reshape(-1)
    P = oracle.hex_trilinear(ne).to_scipy()
    assert P.shape == (3 * ne[0] * (ne[1] + 1) * (ne[2] + 1), 3 * (len(cx) - 1) * len(cy) * len(cz))
    # the clamped coarse node 0 carries the field value 1 + 0.5 z - y etc.; subtract its share
    full = oracle.hex_trilinear(ne).to_scipy()
    fine = field(fx, fy, fz, 0)
    coarse = field(cx, cy, cz, 0)
    # fine nodes at x = 1 interpolate from the clamped plane (x = 0) too: test away from it
    Zf, Yf, Xf = np.meshgrid(fz, fy, fx[1:], indexing="ij")
    mask = np.repeat((Xf.reshape(-1) >= 2), 3)
    np.testing.assert_allclose((full @ coarse)[mask], fine[mask], atol=1e-12)


def test_galerkin_of_trilinear_equals_rediscretised(oracle):
    ne = (4, 4, 4)
    A = oracle.hex_stiffness(ne)
    P = oracle.hex_trilinear(ne)
    G = oracle.galerkin(A, P).to_scipy().toarray()
    C2 = oracle.hex_stiffness((2, 2, 2), scale=2.0).to_scipy().toarray()
    np.testing.assert_allclose(G, C2, atol=1e-12 * np.abs(C2).max())


def test_duvi_soa_structure(oracle):
    m = oracle.Model((16, 4, 4), (20, 1, 1))
    d = oracle.DuVi(m.kff)
    a = d.arrays()
    assert d.nuniq == 28 and d.vi_bits == 8      # 28 distinct values at E = 1
    np.testing.assert_array_equal(d.to_dense(), m.kff.to_scipy().toarray())
    x = np.random.default_rng(1).standard_normal(m.n_free)
    np.testing.assert_array_equal(d.spmv(x), m.kff.spmv(x))
    assert a["row_to_dist"][-1] == m.kff.nnz
    # block starts hold counts, the rest hold gaps - 1
    blocks = oracle.DuVi(oracle.hex_stiffness((128 // 16, 128 // 16, 128 // 16)))
    assert blocks.nblocks >= blocks.n_rows


def test_duvi_block_split_at_256_gap_and_count(oracle):
    # FromDokRowMajor block rule (OpenCLDuViGeometricMultigridSolver.cs:779-789): a block ends at a
    # gap of 256 or more columns, or after 255 following entries.
    cols = list(range(0, 5)) + [305] + list(range(400, 700))
    n = len(cols)
    csr = oracle.Csr.from_arrays(1, 1000, [0, n], cols, np.arange(1, n + 1, dtype=float))
    d = oracle.DuVi(csr, tol=0)
    a = d.arrays()
    # blocks: [0..4] (count 4), [305, 400..654] (gap 94 kept, count 255), [655..699] (count 44)
    np.testing.assert_array_equal(a["col_idx"], [0, 305, 655])
    assert a["dist"][0] == 4 and a["dist"][5] == 255 and a["dist"][6] == 94 and a["dist"][7] == 0
    assert a["dist"][261] == 44
    assert d.vi_bits == 16 and d.nuniq == n
    x = np.arange(1000.0)
    np.testing.assert_array_equal(d.spmv(x), csr.spmv(x))


def test_tolerance_dedup_semantics(oracle):
    # values within 1e-10 merge only inside one hash class round(v / 2e-10)
    tol = 1e-10
    base = 1.0
    vals = np.array([base, base + 0.3e-10, base + 1.5e-10, base - 0.9e-10])
    csr = oracle.Csr.from_arrays(1, 4, [0, 4], [0, 1, 2, 3], vals)
    d = oracle.DuVi(csr, tol=tol)
    a = d.arrays()
    cls = np.rint(vals / (2 * tol))
    tab = a["values"]
    # each value maps to a table entry of its hash class within the tolerance
    for i in range(4):
        rep = tab[a["vidx"][i]]
        assert np.rint(rep / (2 * tol)) == cls[i] and abs(rep - vals[i]) < tol
    # 1 + 1.5e-10 rounds to another class and stays distinct although it is within 2 tol of 1
    np.testing.assert_array_equal(a["vidx"], [0, 0, 1, 0])
    np.testing.assert_array_equal(tab, vals[[0, 2]])


def test_units_from_csr_roundtrip(oracle):
    m = oracle.Model((16, 4, 4), (20, 1, 1))
    u = oracle.Units.from_csr(m.kff)
    x = np.random.default_rng(2).standard_normal(m.n_free)
    np.testing.assert_array_equal(u.multiply(x, np.zeros(m.n_free)), m.kff.spmv(x))
    # Gauss-Seidel over the unit stream equals the CSR forward sweep
    b = m.rhs()
    x1 = np.zeros(m.n_free)
    x2 = np.zeros(m.n_free)
    u.gs(b, x1)
    m.kff.gs_forward(b, x2)
    np.testing.assert_array_equal(x1, x2)


def test_make_path(oracle):
    assert oracle.make_path([1, 1, 0, 0]) == ([True, True, False, False], 3, 0)
    ld, tl, fl = oracle.make_path([1, 1, 0])
    assert ld == [True, True, False, False] and tl == 3 and fl == 0
    ld, tl, fl = oracle.make_path([0, 1])
    assert fl == 1 and tl == 2


@pytest.mark.parametrize("gs,duvi", [(True, False), (False, False), (True, True), (False, True)])
def test_cpu_gmg_converges_to_manufactured_solution(oracle, gs, duvi):
    g = oracle.Gmg((16, 4, 4), (20, 1, 1), gauss_seidel=gs, duvi=duvi, max_cycles=2000, coarse_relaxation=False,
                   tol=1e-5, depth=2, level_iterations=4)
    x, st = g.solve()
    assert st["converged"] and not st["failed"]
    u = oracle.Model((16, 4, 4), (20, 1, 1)).uf()
    assert np.abs(x - u).max() < 1e-6 * np.abs(u).max() * 1e3


def test_mg_fcg_fp64(oracle):
    ne = (8, 8, 8)
    A = [oracle.hex_stiffness(ne), oracle.hex_stiffness((4, 4, 4), scale=2.0)]
    P = [oracle.hex_trilinear(ne)]
    b = oracle.traction_rhs(ne, (8, 8, 8), (0, 0, -1.0))
    x, it, rel = oracle.mg_fcg(A, P, b, 4 / (3 * 3.09), 2, 200, 1e-10)
    assert it > 0 and rel <= 1e-10
    r = b - A[0].spmv(x)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10


def test_golden_fixture_unchanged(oracle):
    if not os.path.exists(GOLDEN):
        pytest.skip("golden fixture not generated")
    g = np.load(GOLDEN)
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import compute
    cur = compute(oracle)
    for k in g.files:
        np.testing.assert_array_equal(g[k], cur[k], err_msg=k)
