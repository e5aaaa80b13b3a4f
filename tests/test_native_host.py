"""libduvigpu.so without a GPU: symbol exports and the host-side setup code.

The structured assembly, the trilinear and the reference Cartesian transfer
operators run on the host inside the product library; they must equal the
oracle's restatement bit for bit, because they feed identical inputs to the
GPU-vs-oracle parity tests.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "duvi_gpu.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"DV_API\s+[^;(]*?\b(dv_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(native):
    lib = native._native.lib()
    syms = declared_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(lib, s), s
    # and the Python binding declares a signature for each of them
    assert set(syms) <= set(native._native.exported_symbols()), set(syms) - set(native._native.exported_symbols())


def test_status_strings(native):
    lib = native._native.lib()
    assert lib.dv_status_string(0) == b"ok"
    assert lib.dv_status_string(-7) == b"no CUDA device"
    assert lib.dv_version() >= 10000


def test_context_without_device_fails_loudly(native):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(native.NoDeviceError):
        native.CudaContext(0)


@pytest.mark.parametrize("ne", [(4, 2, 2), (5, 3, 4), (8, 8, 8)])
def test_hex_assembly_bit_exact(native, oracle, ne):
    A = native.hex_stiffness(ne)
    B = oracle.hex_stiffness(ne).arrays()
    np.testing.assert_array_equal(A.indptr, B[0])
    np.testing.assert_array_equal(A.indices, B[1])
    np.testing.assert_array_equal(A.data, B[2])


def test_hex_assembly_with_moduli_bit_exact(native, oracle, rng):
    ne = (6, 4, 4)
    E = 10.0 ** rng.uniform(-2, 0, size=int(np.prod(ne)))
    A = native.hex_stiffness(ne, E, 2.0)
    B = oracle.hex_stiffness(ne, E, 2.0).arrays()
    np.testing.assert_array_equal(A.data, B[2])
    # and equals the DOK restatement of FemCantileverBase.AssembleGlobalMatrix with densities
    M = oracle.Model(ne, (6, 4, 4), densities=E * 2.0).kff.arrays()
    np.testing.assert_array_equal(A.data, M[2])


@pytest.mark.parametrize("ne", [(4, 4, 4), (8, 4, 2), (5, 3, 4), (7, 9, 1)])
def test_trilinear_bit_exact(native, oracle, ne):
    P = native.hex_trilinear(ne)
    Q = oracle.hex_trilinear(ne).arrays()
    np.testing.assert_array_equal(P.indptr, Q[0])
    np.testing.assert_array_equal(P.indices, Q[1])
    np.testing.assert_array_equal(P.data, Q[2])


@pytest.mark.parametrize("fine,coarse", [((8, 4, 4), (4, 2, 2)), ((6, 2, 2), (3, 1, 1)), ((5, 3, 2), (2, 1, 1)),
                                         ((16, 1, 2), (8, 1, 1))])
def test_cartesian_transfer_bit_exact(native, oracle, fine, coarse):
    mf = native.FemCantilever3D(fine)
    mc = native.FemCantilever3D(coarse)
    R, P = native.cartesian_transfer(3, fine, coarse, 3, mf.FindFreeDofs(), mc.FindFreeDofs())
    Ro, Po = oracle.transfer(fine, coarse)
    for M, O in ((R, Ro), (P, Po)):
        a = O.arrays()
        np.testing.assert_array_equal(M.indptr, a[0])
        np.testing.assert_array_equal(M.indices, a[1])
        np.testing.assert_array_equal(M.data, a[2])


def test_cantilever_model_matches_oracle(native, oracle):
    m = native.FemCantilever3D((8, 2, 2), (20, 1, 1))
    o = oracle.Model((8, 2, 2), (20, 1, 1))
    np.testing.assert_array_equal(m.FindFreeDofs(), o.free_dofs())
    np.testing.assert_allclose(m.free_displacements(), o.uf(), rtol=0, atol=1e-15 * np.abs(o.uf()).max())
    A, b = m.CreateLinearSystem()
    np.testing.assert_allclose(b, o.rhs(), rtol=1e-12, atol=1e-12 * np.abs(o.rhs()).max())


def test_traction_rhs_matches_oracle(native, oracle):
    ne = (6, 4, 2)
    np.testing.assert_array_equal(native.traction_rhs(ne), oracle.traction_rhs(ne, ne, (0, 0, -1.0)))


def test_hierarchy_shapes(native):
    A, P = native.hex_hierarchy((16, 16, 16), coarse_ne=4)
    assert [a.shape[0] for a in A] == [3 * n * (n + 1) ** 2 for n in (16, 8, 4)]
    for l, p in enumerate(P):
        assert p.shape == (A[l].shape[0], A[l + 1].shape[0])


def test_make_path_matches_oracle(native, oracle):
    for ld in ([1, 1, 0, 0], [1, 1, 0], [1, 0, 1, 0], [1, 1, 1, 0, 0, 0]):
        assert native.make_path(ld) == oracle.make_path(ld)


@pytest.mark.parametrize("ne", [(4, 4, 4), (5, 3, 4), (7, 9, 5)])
def test_galerkin_bit_exact(native, oracle, ne):
    # P^T A P summed in the oracle's order (entries of P^T, then A, then P)
    A = native.hex_stiffness(ne)
    P = native.hex_trilinear(ne)
    G = native.galerkin(A, P)
    H = oracle.galerkin(oracle.Csr.from_scipy(A), oracle.hex_trilinear(ne)).arrays()
    np.testing.assert_array_equal(G.indptr, H[0])
    np.testing.assert_array_equal(G.indices, H[1])
    np.testing.assert_array_equal(G.data, H[2])


def test_galerkin_hierarchy_odd_sizes(native):
    A, P = native.galerkin_hierarchy((37, 11, 23), max_coarse_dofs=1000)
    assert [a.shape[0] for a in A] == [31968, 5187, 840]
    for l, p in enumerate(P):
        assert p.shape == (A[l].shape[0], A[l + 1].shape[0])
        d = A[l + 1] - (p.T @ A[l] @ p)
        assert abs(d).max() <= 1e-12 * abs(A[l + 1]).max()
        assert abs(A[l + 1] - A[l + 1].T).max() <= 1e-12 * abs(A[l + 1]).max()


def test_cantilever_batch_is_seeded(native):
    d1, m1, r1 = native.cantilever_batch(4, seed=7)
    d2, m2, r2 = native.cantilever_batch(4, seed=7)
    assert d1 == d2 and all(8 <= v <= 48 for d in d1 for v in d)
    assert all(np.array_equal(a, b) for a, b in zip(r1, r2))
    assert [m[0][0].shape[0] for m in m1] == [3 * d[0] * (d[1] + 1) * (d[2] + 1) for d in d1]


def _encode_matches_oracle(native, oracle, A, tol=1e-10, bits=0):
    got = native.duvi_encode(A, bits, tol)
    ref = oracle.DuVi(oracle.Csr.from_scipy(A), tol, bits)
    exp = ref.arrays()
    assert got["vi_bits"] == ref.vi_bits
    for k in ("row_to_col", "row_to_dist", "col_idx", "dist", "vidx"):
        np.testing.assert_array_equal(got[k], exp[k], err_msg=k)
    np.testing.assert_array_equal(got["values"].view(np.uint64), exp["values"].view(np.uint64))


def _random_csr(rng, n, per_row, values):
    import scipy.sparse as sp
    rows = np.repeat(np.arange(n), per_row)
    cols = np.concatenate([np.sort(rng.choice(n, per_row, replace=False)) for _ in range(n)])
    A = sp.csr_matrix((np.ones(rows.size), (rows, cols)), shape=(n, n))
    A.sort_indices()
    A.data = np.asarray(values, np.float64)[: A.nnz].copy()
    return A


@pytest.mark.parametrize("case", ["hex", "hex_log_moduli", "small"])
def test_duvi_host_encoder_matches_oracle(native, oracle, rng, case):
    # The library's encoder numbers values in parallel chunks (exact-bit local tables,
    # then the chunks' distinct values through the .NET Dictionary semantics in order);
    # its arrays must equal the oracle's sequential FromDokRowMajor bit for bit.
    if case == "hex":
        A = native.hex_stiffness((12, 12, 12))                    # 28 values, 460k entries
    elif case == "hex_log_moduli":
        E = 10.0 ** rng.uniform(-2.0, 0.0, 8 * 8 * 8)
        A = native.hex_stiffness((8, 8, 8), E)                    # nearly every value distinct
    else:
        A = native.hex_stiffness((2, 2, 2))                       # below the parallel threshold
    assert case == "small" or A.nnz >= 1 << 16
    _encode_matches_oracle(native, oracle, A)
    if case != "hex":
        _encode_matches_oracle(native, oracle, A, bits=32)


def test_duvi_host_encoder_near_tolerance_values(native, oracle, rng):
    # Values -0.9, -0.1 and +0.5 x 1e-10 around multiples of 2e-10 share a hash cell;
    # -0.9 and +0.5 are two keys (1.4e-10 apart) and -0.1 lies within the tolerance of
    # both, so its key depends on which one was inserted last: the encoder must detect
    # this and number the values exactly as the sequential walk does.
    n, per_row = 3000, 40
    m = rng.integers(1, 50, n * per_row) * 2e-10
    d = rng.choice([-0.9e-10, -0.1e-10, 0.5e-10], n * per_row)
    _encode_matches_oracle(native, oracle, _random_csr(rng, n, per_row, m + d))


@pytest.mark.parametrize("tol", [1e-10, 0.0])
def test_duvi_host_encoder_special_values(native, oracle, rng, tol):
    # NaN and infinities (under a tolerance they equal nothing, not even themselves, so
    # every occurrence is a new value) and signed zeros, in a matrix large enough for
    # the parallel path.
    n, per_row = 2000, 40
    pool = np.array([0.0, -0.0, 1.5, -2.25, np.inf, -np.inf, np.nan, 3.0])
    vals = pool[rng.integers(0, pool.size, n * per_row)]
    vals[rng.random(vals.size) < 0.995] = 1.5   # keep the special values rare
    _encode_matches_oracle(native, oracle, _random_csr(rng, n, per_row, vals), tol=tol, bits=32)


@pytest.mark.parametrize("kind", ["unsorted", "column_range", "rowptr_down", "rowptr_past_nnz"])
def test_host_encoder_rejects_bad_csr(native, kind):
    # The CSR checks run over the rows in parallel and report the first bad row's fault.
    import ctypes as C
    N = native._native
    rp = np.array([0, 2, 4, 6], np.int32)
    ci = np.array([0, 1, 1, 2, 0, 2], np.int32)
    va = np.ones(6)
    if kind == "unsorted":
        ci[2:4] = [2, 1]
    elif kind == "column_range":
        ci[5] = 3
    elif kind == "rowptr_down":
        rp[2] = 1          # row 0 is valid, row 1 ends before it starts
    else:
        rp[1:3] = [2, 9]   # row 1 would read past nnz
    ah, keep = N.csr_host(rp, ci, va, (3, 3))
    nb, nu, bits = C.c_int64(), C.c_int64(), C.c_int32()
    st = N.lib().dv_duvi_encode(C.byref(ah), 0, 1e-10, C.byref(nb), C.byref(nu), C.byref(bits),
                                None, None, None, None, None, None)
    assert st == N.DV_ERR_FORMAT
    msg = N.lib().dv_last_error().decode()
    assert {"unsorted": "increasing", "column_range": "out of range", "rowptr_down": "monotone",
            "rowptr_past_nnz": "monotone"}[kind] in msg, msg


def _units_match_oracle(native, oracle, A, tol=1e-10):
    got = native.units_encode(A, tol)
    exp = oracle.Units.from_csr(oracle.Csr.from_scipy(A), tol).arrays()
    np.testing.assert_array_equal(got["bytes"], exp["bytes"])
    np.testing.assert_array_equal(got["unit_offsets"], exp["offsets"])
    np.testing.assert_array_equal(got["vidx"], exp["vidx"])
    np.testing.assert_array_equal(got["values"].view(np.uint64), exp["values"].view(np.uint64))
    return got


def test_units_kat_matches_oracle_and_reference_product(native, oracle):
    # CompressedSparseMatrixTests.cs:15-39: 2 x 1024 from CSR; y = A x with x = row 0 is [11, 0]
    import scipy.sparse as sp
    w = 1024
    A = sp.csr_matrix(([1, 1, 1, 2, 2, 3, 3.0], [5, 6, 8, w - 24, w - 1, 50, w - 4], [0, 5, 7]), shape=(2, w))
    got = _units_match_oracle(native, oracle, A)
    B = native.units_decode(A.shape, got)
    assert (B != A).nnz == 0
    x = A.toarray()[0]
    np.testing.assert_array_equal(B @ x, [11.0, 0.0])


def test_units_every_width_and_gap_length(native, oracle):
    # steps of 1, 2 and 4 bytes in every order, gaps in each of the four prefix-code lengths
    # (< 128, < 16,512, < 2,113,664, above), width changes on empty and non-empty units
    import scipy.sparse as sp
    rng = np.random.default_rng(20261203)
    n, m = 60, 6_000_000
    rows, cols = [], []
    for i in range(n):
        c, cs = int(rng.integers(0, 3_000_000)) if i % 4 == 3 else int(rng.integers(0, 20000)), []
        for _ in range(int(rng.integers(1, 40))):
            if c >= m:
                break
            cs.append(c)
            c += int(rng.choice([1, 2, 200, 255, 256, 300, 65535, 65536, 70000]))
        rows += [i] * len(cs)
        cols += cs
    A = sp.csr_matrix((rng.integers(1, 6, len(rows)).astype(float), (rows, cols)), shape=(n, m))
    A.sort_indices()
    got = _units_match_oracle(native, oracle, A)
    b, off = got["bytes"], got["unit_offsets"][:-1]
    assert set(b[off] >> 1) == {0, 1, 2}                                       # step widths 1, 2, 4 bytes
    g = b[off + 2]
    kinds = np.where(g < 0x80, 1, np.where(g < 0xC0, 2, np.where(g < 0xE0, 3, 4)))
    assert set(kinds) == {1, 2, 3, 4}                                          # every gap code length
    B = native.units_decode(A.shape, got)
    assert (B != A).nnz == 0 and np.array_equal(B.indptr, A.indptr)


def test_units_empty_rows_and_hex_operator(native, oracle, rng):
    import scipy.sparse as sp
    # empty rows: one unit of gap 0 numbered as the value 0.0; decoded as an explicit zero
    A = sp.csr_matrix(np.array([[0, 2.0, 0], [0, 0, 0], [1.0, 0, 3.0], [0, 0, 0]]))
    got = _units_match_oracle(native, oracle, A)
    B = native.units_decode(A.shape, got)
    assert B.nnz == A.nnz + 2 and B[1, 0] == 0.0 and B[3, 0] == 0.0
    np.testing.assert_array_equal(B.toarray(), A.toarray())
    # a 12^3 hex operator (460k entries: the parallel value numbering), round trip
    H = native.hex_stiffness((12, 12, 12))
    got = _units_match_oracle(native, oracle, H)
    B = native.units_decode(H.shape, got)
    assert (B != H).nnz == 0


def test_units_reject_unrepresentable_rows_and_malformed_streams(native):
    import scipy.sparse as sp
    # 300 one-byte steps in one unit: the reference's count byte would wrap
    A = sp.csr_matrix((np.ones(301), (np.zeros(301, int), np.arange(301))), shape=(1, 400))
    with pytest.raises(native.DuviError) as e:
        native.units_encode(A)
    assert e.value.status == native._native.DV_ERR_FORMAT and "255" in str(e.value)
    H = native.hex_stiffness((2, 2, 2))
    u = native.units_encode(H)
    bad = dict(u, bytes=u["bytes"][:-1])   # truncated inside the last unit
    with pytest.raises(native.DuviError):
        native.units_decode(H.shape, bad)
    with pytest.raises(native.DuviError):   # one row too few
        native.units_decode((H.shape[0] + 1, H.shape[1]), u)
    # a zero column step (the first unit of row 0 has steps of one byte after its 3 header bytes)
    b = u["bytes"].copy()
    assert b[0] == 1 and b[1] > 0 and b[2] < 0x80
    b[3] = 0
    with pytest.raises(native.DuviError) as e:
        native.units_decode(H.shape, dict(u, bytes=b))
    assert "increasing" in str(e.value)


def test_host_encoders_reproduce_golden_vectors(native):
    # tests/golden/oracle_small.npz (committed, made by tests/golden/make_golden.py): the
    # product's DuVi SoA encoder and Unit-stream encoder on the fixture's stiffness matrix
    # give the committed arrays byte for byte.
    import scipy.sparse as sp
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "oracle_small.npz"))
    n = g["kff_rowptr"].size - 1
    K = sp.csr_matrix((g["kff_val"], g["kff_col"], g["kff_rowptr"]), shape=(n, n))
    d = native.duvi_encode(K)
    for k in ("row_to_col", "row_to_dist", "col_idx", "dist", "vidx", "values"):
        np.testing.assert_array_equal(d[k], g["duvi_" + k], err_msg=k)
    u = native.units_encode(K)
    np.testing.assert_array_equal(u["bytes"], g["units_bytes"])
    np.testing.assert_array_equal(u["vidx"], g["units_vidx"])


def test_duvi_host_encoder_index_widths(native, oracle, rng):
    # value_index_bits 0 picks the narrowest width; a wider forced width keeps the same
    # indices; a width too narrow for the distinct values is a format error
    import scipy.sparse as sp
    A = _random_csr(rng, 400, 20, np.round(rng.standard_normal(8000), 3))   # ~2,000 distinct values
    auto = native.duvi_encode(A)
    assert auto["vi_bits"] == 16
    wide = native.duvi_encode(A, 32)
    assert wide["vi_bits"] == 32
    np.testing.assert_array_equal(wide["vidx"], auto["vidx"])
    _encode_matches_oracle(native, oracle, A, bits=16)
    with pytest.raises(native.DuviError) as e:
        native.duvi_encode(A, 8)
    assert e.value.status == native._native.DV_ERR_FORMAT
    with pytest.raises(native.DuviError) as e:
        native.duvi_encode(A, 12)
    assert e.value.status == native._native.DV_ERR_ARG
