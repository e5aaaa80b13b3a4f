"""GPU SpMV/SpMM and DuVi encoding against the CPU oracle.

Bar: DuVi structure and value indices bit-exact with the oracle encoder
(FromDokRowMajor, OpenCLDuViGeometricMultigridSolver.cs:753-851); FP64 DuVi
products bit-exact with the oracle's kernel-order walk
(DuViGeometricMultigrid.cl:84-98); FP64 CSR products within 1e-12 relative per
row (the warp-split summation reorders the sum); FP32 within 1e-5 relative to
the FP64 oracle.
"""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

REL64 = 1e-12
REL32 = 1e-5


def rowwise_rel(y, ref, A_abs, x):
    scale = np.abs(A_abs) @ np.abs(x) + 1e-300
    return np.max(np.abs(y - ref) / scale)


def random_csr(rng, n, m, density, empty_rows=()):
    A = sp.random(n, m, density=density, random_state=np.random.RandomState(7), format="csr")
    A.data = rng.standard_normal(A.nnz)
    A = A.tolil()
    for r in empty_rows:
        A[r, :] = 0
    A = A.tocsr()
    A.eliminate_zeros()
    A.sort_indices()
    return A


@pytest.fixture(scope="module")
def cantilever(oracle):
    m = oracle.Model((16, 4, 4), (20, 1, 1))
    return m, m.kff.to_scipy()


def test_diagonal_kat(ctx, native):
    # GMCantileverOpenCLTests.cs:16-52
    v = np.arange(16, 0, -1.0)
    A = sp.csr_matrix((v, np.arange(16), np.arange(17)), shape=(16, 16))
    for fmt in ("csr", "duvi"):
        M = native.SparseMatrix(ctx, A, fmt)
        np.testing.assert_array_equal(M.Multiply(v), v * v)


def test_duvi_2x1024_kat(ctx, native):
    # CompressedSparseMatrixTests.cs:15-39 through the GPU SoA format
    w = 1024
    A = sp.csr_matrix(([1, 1, 1, 2, 2, 3, 3.0], [5, 6, 8, w - 24, w - 1, 50, w - 4], [0, 5, 7]), shape=(2, w))
    x = A.toarray()[0].copy()
    for fmt in ("csr", "duvi"):
        y = native.SparseMatrix(ctx, A, fmt).Multiply(x)
        assert y[0] == 11 and y[1] == 0


@pytest.mark.parametrize("bits", [0, 16, 32])
def test_duvi_encoding_bit_exact(ctx, native, oracle, cantilever, bits):
    m, A = cantilever
    M = native.SparseMatrix(ctx, A, "duvi", value_index_bits=bits)
    got = M.export_duvi()
    ref = oracle.DuVi(m.kff, 1e-10, bits).arrays()
    for k in ("row_to_col", "row_to_dist", "col_idx", "dist", "vidx", "values"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert got["vi_bits"] == (8 if bits == 0 else bits)


def test_duvi_encoding_many_values(ctx, native, oracle, rng):
    # moduli drawn log-uniform: ~nnz/2 distinct values, 16/32-bit indices
    ne = (6, 4, 4)
    E = 10.0 ** rng.uniform(-2, 0, size=int(np.prod(ne)))
    A = native.hex_stiffness(ne, E)
    M = native.SparseMatrix(ctx, A, "duvi")
    got = M.export_duvi()
    ref = oracle.DuVi(oracle.Csr.from_scipy(A), 1e-10, 0)
    r = ref.arrays()
    assert got["vi_bits"] == ref.vi_bits and ref.vi_bits in (16, 32)
    for k in ("col_idx", "dist", "vidx", "values"):
        np.testing.assert_array_equal(got[k], r[k], err_msg=k)
    x = rng.standard_normal(A.shape[1])
    np.testing.assert_array_equal(M.Multiply(x), ref.spmv(x))


@pytest.mark.parametrize("fmt", ["csr", "duvi"])
def test_spmv_f64_cantilever(ctx, native, oracle, cantilever, rng, fmt):
    m, A = cantilever
    x = rng.standard_normal(A.shape[1])
    M = native.SparseMatrix(ctx, A, fmt)
    y = M.Multiply(x)
    if fmt == "duvi":
        np.testing.assert_array_equal(y, oracle.DuVi(m.kff).spmv(x))
        # accumulate mode (clear = 0): y += A x in the reference's order
        y0 = rng.standard_normal(A.shape[0])
        got = M.Multiply(x, y0.copy(), clear=False)
        np.testing.assert_array_equal(got, oracle.DuVi(m.kff).spmv(x, y0.copy(), clear=False))
    else:
        assert rowwise_rel(y, m.kff.spmv(x), A, x) <= REL64


@pytest.mark.parametrize("fmt", ["csr", "duvi"])
def test_spmv_f32(ctx, native, cantilever, rng, fmt):
    m, A = cantilever
    x = rng.standard_normal(A.shape[1])
    y = native.SparseMatrix(ctx, A, fmt, "f32").Multiply(x)
    assert rowwise_rel(y, A @ x, A, x) <= REL32


@pytest.mark.parametrize("fmt", ["csr", "duvi"])
def test_spmv_random_with_empty_rows(ctx, native, oracle, rng, fmt):
    A = random_csr(rng, 700, 900, 0.02, empty_rows=(0, 5, 699))
    x = rng.standard_normal(900)
    y = native.SparseMatrix(ctx, A, fmt, dedup_tol=0.0).Multiply(x)
    ref = oracle.Csr.from_scipy(A)
    if fmt == "duvi":
        np.testing.assert_array_equal(y, oracle.DuVi(ref, 0.0).spmv(x))
    else:
        assert rowwise_rel(y, ref.spmv(x), A, x) <= REL64
    assert y[0] == 0 and y[5] == 0 and y[699] == 0


def test_duvi_long_rows_fallback(ctx, native, oracle, rng):
    # rows longer than one stage (3008 entries) take the unstaged path
    n, m = 40, 20000
    rows, cols = [], []
    for r in range(n):
        k = 5000 if r in (3, 17) else 50
        c = np.sort(rng.choice(m, size=k, replace=False))
        rows += [r] * k
        cols += list(c)
    A = sp.csr_matrix((rng.standard_normal(len(rows)), (rows, cols)), shape=(n, m))
    A.sort_indices()
    x = rng.standard_normal(m)
    y = native.SparseMatrix(ctx, A, "duvi", dedup_tol=0.0).Multiply(x)
    np.testing.assert_array_equal(y, oracle.DuVi(oracle.Csr.from_scipy(A), 0.0).spmv(x))


def _spmm(native, M, X, dtype):
    import torch
    dX = torch.from_numpy(np.ascontiguousarray(X, dtype)).cuda()
    dY = torch.zeros((M.shape[0], X.shape[1]), dtype=dX.dtype, device="cuda")
    torch.cuda.synchronize()
    M.multiply_many_device(X.shape[1], dX.data_ptr(), dY.data_ptr(), "f64" if dtype == np.float64 else "f32")
    M.ctx.synchronize()
    return dY.cpu().numpy()


@pytest.mark.parametrize("fmt", ["csr", "duvi"])
@pytest.mark.parametrize("k", [1, 7, 33, 64, 130])
def test_spmm_bit_exact(ctx, native, oracle, cantilever, rng, fmt, k):
    # One warp per node group, lanes over right-hand sides, each row summed in
    # storage order: every column equals the oracle's sequential product bit for bit.
    m, A = cantilever
    X = rng.standard_normal((A.shape[1], k))
    M = native.SparseMatrix(ctx, A, fmt)
    assert M.info()["row_group"] == 3
    Y = _spmm(native, M, X, np.float64)
    ref_op = oracle.DuVi(m.kff) if fmt == "duvi" else m.kff
    for j in range(k):
        np.testing.assert_array_equal(Y[:, j], ref_op.spmv(X[:, j]))


@pytest.mark.parametrize("fmt", ["csr", "duvi"])
def test_spmm_ungrouped_rows_bit_exact(ctx, native, oracle, rng, fmt):
    A = random_csr(rng, 700, 900, 0.02, empty_rows=(0, 5, 699))
    X = rng.standard_normal((900, 40))
    M = native.SparseMatrix(ctx, A, fmt, dedup_tol=0.0)
    assert M.info()["row_group"] == 1
    Y = _spmm(native, M, X, np.float64)
    ref = oracle.Csr.from_scipy(A)
    ref_op = oracle.DuVi(ref, 0.0) if fmt == "duvi" else ref
    for j in range(40):
        np.testing.assert_array_equal(Y[:, j], ref_op.spmv(X[:, j]))
    assert not Y[[0, 5, 699]].any()


def test_spmm_f32_duvi_equals_single_products(ctx, native, cantilever, rng):
    # FP32 DuVi: the block product and the single-vector kernel both sum each row
    # in storage order with fused multiply-adds, so the results are identical.
    m, A = cantilever
    X = rng.standard_normal((A.shape[1], 33)).astype(np.float32)
    M = native.SparseMatrix(ctx, A, "duvi", "f32")
    Y = _spmm(native, M, X, np.float32)
    for j in (0, 17, 32):
        np.testing.assert_array_equal(Y[:, j], M.Multiply(X[:, j].astype(np.float64)).astype(np.float32))
    X64 = X.astype(np.float64)
    assert np.max(np.abs(Y - A @ X64) / (abs(A) @ np.abs(X64) + 1e-300)) <= REL32


def test_residual_device(ctx, native, cantilever, rng):
    import torch
    m, A = cantilever
    x = rng.standard_normal(A.shape[1])
    b = rng.standard_normal(A.shape[0])
    M = native.SparseMatrix(ctx, A, "duvi")
    dx, db = torch.from_numpy(x).cuda(), torch.from_numpy(b).cuda()
    dr = torch.zeros_like(db)
    torch.cuda.synchronize()
    M.residual_device(db.data_ptr(), dx.data_ptr(), dr.data_ptr())
    ctx.synchronize()
    assert rowwise_rel(dr.cpu().numpy(), b - A @ x, A, x) <= REL64


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_lane_kernel_gaps_of_256_inside_blocks(ctx, native, oracle, prec):
    # Node-grouped rows (3 rows share columns) whose runs contain gaps of exactly 255, 256
    # and 257: a gap of 256 stays inside a DuVi block (its byte is 255), which the lane
    # layout must not take for a block start.
    n = 3 * 700
    rows, cols, vals = [], [], []
    for g in range(n // 3):
        c, cs = (g * 7) % 50, []
        for gap in (1, 256, 256, 1, 255, 257, 256, 2, 256):
            if c >= n:
                break
            cs.append(c)
            c += gap
        for d in range(3):
            for x in cs:
                rows.append(3 * g + d)
                cols.append(x)
                vals.append(1.0 + 0.25 * ((x + d) % 5))
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    A.sort_indices()
    M = native.SparseMatrix(ctx, A, "duvi", prec)
    assert M.info()["kernel_variant"] == 103   # the lane kernel, 3-row groups
    x = np.random.default_rng(3).standard_normal(n)
    y = M.Multiply(x)
    if prec == "f64":
        np.testing.assert_array_equal(y, oracle.DuVi(oracle.Csr.from_scipy(A)).spmv(x))
    else:
        assert rowwise_rel(y, A @ x, A, x) <= REL32


@pytest.mark.parametrize("ne", [(8, 6, 6), (7, 9, 5)])
@pytest.mark.parametrize("patterns", ["1", "0"])
def test_transfer_products_shifted_groups_bit_exact(ctx, native, oracle, ne, patterns, monkeypatch):
    # Trilinear P and R = P^T: the 3 rows of a node read columns shifted by the dof
    # component.  With patterns on, each node stores its first column and a pattern id
    # (offsets from that column; variant 203); with them off, the lane layout keeps the
    # shifted groups once per node (variant 103).
    monkeypatch.setenv("DV_PATTERNS", patterns)
    P = native.hex_trilinear(ne)
    for M in (P, P.T.tocsr()):
        M.sort_indices()
        D = native.SparseMatrix(ctx, M, "duvi", "f64")
        assert D.info()["kernel_variant"] == (203 if patterns == "1" else 103)
        x = np.random.default_rng(5).standard_normal(M.shape[1])
        np.testing.assert_array_equal(D.Multiply(x), oracle.DuVi(oracle.Csr.from_scipy(M)).spmv(x))
        F = native.SparseMatrix(ctx, M, "duvi", "f32")
        assert rowwise_rel(F.Multiply(x), M @ x, M, x) <= REL32


@pytest.mark.parametrize("pool", [40, 200])
def test_lane_kernel_node_tuples_and_fallback(ctx, native, oracle, rng, pool, monkeypatch):
    # 3-row node groups with 8-bit value indices: few distinct (v0, v1, v2) per node-entry
    # (pool 40 of 2 patterns) use one tuple index per node-entry; random values from a pool
    # of 200 give far more than 256 combinations and fall back to per-row indices.
    n = 3 * 900
    vals_pool = np.round(rng.standard_normal(pool), 6)
    rows, cols, vals = [], [], []
    for g in range(n // 3):
        cs = sorted(set(((g * 3 + np.array([0, 3, 6, 150, 153, 600, 903])) % n).tolist()))
        for d in range(3):
            for j, c in enumerate(cs):
                if pool == 40:
                    v = vals_pool[(j + 7 * d + (g % 2)) % pool]
                else:
                    v = vals_pool[rng.integers(pool)]
                rows.append(3 * g + d)
                cols.append(c)
                vals.append(v)
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    A.sort_indices()
    monkeypatch.setenv("DV_PATTERNS", "0")   # the repeating case would otherwise take the node-pattern kernel
    M = native.SparseMatrix(ctx, A, "duvi", "f64", dedup_tol=0.0)
    info = M.info()
    assert info["kernel_variant"] == 103 and info["value_index_bits"] == 8
    x = rng.standard_normal(n)
    np.testing.assert_array_equal(M.Multiply(x), oracle.DuVi(oracle.Csr.from_scipy(A), 0.0).spmv(x))
    F = native.SparseMatrix(ctx, A, "duvi", "f32", dedup_tol=0.0)
    assert rowwise_rel(F.Multiply(x), A @ x, A, x) <= REL32



LAYOUTS = {"grid": ("1", "1", 303), "patterns": ("1", "0", 203), "lanes": ("0", "0", 103)}


@pytest.mark.parametrize("ne", [(8, 8, 8), (16, 4, 4), (7, 5, 9), (40, 21, 13)])
@pytest.mark.parametrize("layout", ["grid", "patterns", "lanes"])
def test_hex_operator_grid_pattern_and_lane_kernels_bit_exact(ctx, native, oracle, rng, ne, layout, monkeypatch):
    # The hex stiffness repeats one entry list per node class (interior, faces, edges,
    # corners).  grid (variant 303): interior nodes by the plane-streaming stencil with the
    # interior pattern's values as kernel parameters, the others from their records;
    # patterns (203): one pattern id per node and a shared-memory pattern table; lanes
    # (103): the lane layout with stencil offsets and node tuples.  All sum every row in
    # storage order: bit-exact in FP64.  (40, 21, 13) spans two x tiles (one partial), three
    # y tiles and several z runs.
    patterns, grid, variant = LAYOUTS[layout]
    monkeypatch.setenv("DV_PATTERNS", patterns)
    monkeypatch.setenv("DV_GRID", grid)
    A = native.hex_stiffness(ne)
    x = rng.standard_normal(A.shape[1])
    ref = oracle.DuVi(oracle.Csr.from_scipy(A)).spmv(x)
    M = native.SparseMatrix(ctx, A, "duvi", "f64")
    assert M.info()["kernel_variant"] == variant
    np.testing.assert_array_equal(M.Multiply(x), ref)
    y0 = rng.standard_normal(A.shape[0])
    np.testing.assert_array_equal(M.Multiply(x, y0.copy(), clear=False),
                                  oracle.DuVi(oracle.Csr.from_scipy(A)).spmv(x, y0.copy(), clear=False))
    F = native.SparseMatrix(ctx, A, "duvi", "f32")
    assert F.info()["kernel_variant"] == variant
    assert rowwise_rel(F.Multiply(x), A @ x, A, x) <= REL32


def _device_product(ctx, M, x, dtype):
    import torch
    dx = torch.from_numpy(np.ascontiguousarray(x, dtype)).cuda()
    dy = torch.zeros(M.shape[0], dtype=dx.dtype, device="cuda")
    torch.cuda.synchronize()
    M.multiply_device(dx.data_ptr(), dy.data_ptr(), "f32" if dtype == np.float32 else "f64")
    ctx.synchronize()
    return dy.cpu().numpy()


def _grid_vs_patterns(native, ctx, A, x, prec, monkeypatch, expect_grid=303):
    monkeypatch.setenv("DV_GRID", "1")
    G = native.SparseMatrix(ctx, A, "duvi", prec)
    assert G.info()["kernel_variant"] == expect_grid
    monkeypatch.setenv("DV_GRID", "0")
    Pm = native.SparseMatrix(ctx, A, "duvi", prec)
    assert Pm.info()["kernel_variant"] == 203
    dt = np.float32 if prec == "f32" else np.float64
    return _device_product(ctx, G, x, dt), _device_product(ctx, Pm, x, dt)


@pytest.mark.parametrize("ne", [(8, 8, 8), (33, 9, 20), (64, 17, 10)])
def test_grid_stencil_f32_equals_pattern_kernel(ctx, native, rng, ne, monkeypatch):
    # FP32 products on device vectors: the grid stencil (hex value classes, structural zeros
    # skipped) and the node-pattern kernel give the same floats (the same fused multiply-adds in
    # the same order; the skipped terms add exact zeros).
    monkeypatch.setenv("DV_AUTOTUNE", "0")
    A = native.hex_stiffness(ne, scale=2.0)
    x = rng.standard_normal(A.shape[1])
    yg, yp = _grid_vs_patterns(native, ctx, A, x, "f32", monkeypatch)
    np.testing.assert_array_equal(yg, yp)


def test_grid_stencil_general_coefficients(ctx, native, oracle, rng, monkeypatch):
    # An operator with the 27-neighbour interior pattern but without the hex value classes (one
    # coupling changed by the same amount in every row of dof 0 with a +x neighbour): FP32 runs
    # the general stencil (all 243 coefficients) and equals the pattern kernel; FP64 keeps the
    # node patterns (variant 203) and equals the oracle's walk.
    ne = (20, 11, 9)
    A = native.hex_stiffness(ne).tolil()
    lx = ne[0]
    for i in range(A.shape[0] // 3):
        if (i % lx) < lx - 1:
            A[3 * i, 3 * (i + 1)] += 1e-3
    A = A.tocsr()
    A.sort_indices()
    x = rng.standard_normal(A.shape[1])
    yg, yp = _grid_vs_patterns(native, ctx, A, x, "f32", monkeypatch)
    np.testing.assert_array_equal(yg, yp)
    monkeypatch.setenv("DV_GRID", "1")
    M = native.SparseMatrix(ctx, A, "duvi", "f64")
    assert M.info()["kernel_variant"] == 203
    np.testing.assert_array_equal(M.Multiply(x), oracle.DuVi(oracle.Csr.from_scipy(A)).spmv(x))


def test_grid_stencil_interior_nodes_of_other_patterns(ctx, native, oracle, rng, monkeypatch):
    # A few elements with other moduli: the interior nodes around them get their own patterns
    # and run from their records inside the grid launch; FP64 stays bit-exact with the oracle,
    # the residual r = b - A x too.
    import torch
    monkeypatch.setenv("DV_GRID", "1")
    ne = (24, 10, 12)
    E = np.ones(int(np.prod(ne)))
    E[rng.choice(E.size, 7, replace=False)] = 2.0
    A = native.hex_stiffness(ne, E)
    x = rng.standard_normal(A.shape[1])
    M = native.SparseMatrix(ctx, A, "duvi", "f64")
    assert M.info()["kernel_variant"] == 303
    ref = oracle.DuVi(oracle.Csr.from_scipy(A)).spmv(x)
    np.testing.assert_array_equal(M.Multiply(x), ref)
    b = rng.standard_normal(A.shape[0])
    db, dx = torch.from_numpy(b).cuda(), torch.from_numpy(x).cuda()
    dr = torch.empty_like(db)
    torch.cuda.synchronize()
    M.residual_device(db.data_ptr(), dx.data_ptr(), dr.data_ptr(), "f64")
    ctx.synchronize()
    np.testing.assert_array_equal(dr.cpu().numpy(), b - ref)


@pytest.mark.parametrize("k", [5, 40, 130])
def test_spmm_transfers_bit_exact(ctx, native, oracle, rng, k):
    # Block products of P and R = P^T on the node-pattern layout (offsets from each node's
    # first column, row d reading column + d): every column equals the oracle's product.
    P = native.hex_trilinear((8, 6, 6))
    for M0 in (P, P.T.tocsr()):
        M0.sort_indices()
        M = native.SparseMatrix(ctx, M0, "duvi", "f64")
        assert M.info()["kernel_variant"] == 203
        X = rng.standard_normal((M0.shape[1], k))
        Y = _spmm(native, M, X, np.float64)
        ref = oracle.DuVi(oracle.Csr.from_scipy(M0))
        for j in (0, k // 2, k - 1):
            np.testing.assert_array_equal(Y[:, j], ref.spmv(X[:, j]))


@pytest.mark.parametrize("ne", [(1, 1, 1), (8, 8, 8), (40, 21, 13), (33, 9, 20)])
@pytest.mark.parametrize("moduli", ["uniform", "log_uniform"])
def test_matrix_free_hex_operator(ctx, native, rng, ne, moduli):
    # The element kernel (format "hex") applies K = sum_e (scale E_e) Ke without storing it:
    # FP64 products within 1e-12 relative per row of the assembled matrix (another summation
    # order), FP32 within 1e-5; y += A x and r = b - A x through the same kernel.
    import torch
    E = None if moduli == "uniform" else 10.0 ** rng.uniform(-2.0, 0.0, int(np.prod(ne)))
    A = native.hex_stiffness(ne, E, scale=2.0)
    x = rng.standard_normal(A.shape[1])
    ref = A @ x
    H = native.SparseMatrix.hex_operator(ctx, ne, E, scale=2.0)
    assert H.info()["kernel_variant"] == 400 and H.info()["format"] == 2
    assert rowwise_rel(H.Multiply(x), ref, A, x) <= REL64
    y0 = rng.standard_normal(A.shape[0])
    assert rowwise_rel(H.Multiply(x, y0.copy(), clear=False), y0 + ref, A, x) <= REL64
    b = rng.standard_normal(A.shape[0])
    db, dx = torch.from_numpy(b).cuda(), torch.from_numpy(x).cuda()
    dr = torch.empty_like(db)
    torch.cuda.synchronize()
    H.residual_device(db.data_ptr(), dx.data_ptr(), dr.data_ptr(), "f64")
    ctx.synchronize()
    assert rowwise_rel(dr.cpu().numpy(), b - ref, A, x) <= REL64
    F = native.SparseMatrix.hex_operator(ctx, ne, E, scale=2.0, precision="f32")
    assert rowwise_rel(_device_product(ctx, F, x, np.float32).astype(np.float64), ref, A, x) <= REL32
    with pytest.raises(native.DuviError):
        H.multiply_many_device(2, dx.data_ptr(), dr.data_ptr(), "f64")


@pytest.mark.parametrize("ne", [(2, 2, 2), (8, 6, 6), (16, 10, 14), (4, 8, 2)])
def test_matrix_free_trilinear_transfers_bit_exact(ctx, native, oracle, rng, ne):
    # Format "trilinear" applies the prolongation P = hex_trilinear(ne) and the restriction P^T
    # from the grid indices alone, summing each row's columns in increasing order with the
    # stored kernels' multiply-add: FP64 products equal the oracle's walk of the assembled
    # matrix bit for bit, FP32 products equal the FP32 DuVi kernel's, and block products
    # equal the oracle column by column.
    P = native.hex_trilinear(ne)
    P.sort_indices()
    for restriction, M0 in ((False, P), (True, P.T.tocsr())):
        M0.sort_indices()
        T = native.SparseMatrix.trilinear_transfer(ctx, ne, restriction=restriction)
        assert T.shape == M0.shape
        assert T.info()["kernel_variant"] == 500 and T.info()["format"] == 3
        x = rng.standard_normal(M0.shape[1])
        ref = oracle.DuVi(oracle.Csr.from_scipy(M0))
        np.testing.assert_array_equal(T.Multiply(x), ref.spmv(x))
        T32 = native.SparseMatrix.trilinear_transfer(ctx, ne, restriction=restriction, precision="f32")
        D32 = native.SparseMatrix(ctx, M0, "duvi", "f32")
        np.testing.assert_array_equal(_device_product(ctx, T32, x, np.float32), _device_product(ctx, D32, x, np.float32))
        X = rng.standard_normal((M0.shape[1], 5))
        Y = _spmm(native, T, X, np.float64)
        for j in range(5):
            np.testing.assert_array_equal(Y[:, j], ref.spmv(X[:, j]))
    with pytest.raises(native.DuviError):
        native.SparseMatrix.trilinear_transfer(ctx, (8, 7, 6))
