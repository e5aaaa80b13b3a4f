"""On-device assembly of the structured hexahedral stiffness against the host assembler.

dv_hex_assemble_device writes the sorted CSR arrays of K = sum_e (scale E_e) Ke on the
device, one thread per node, with the reference's per-entry summation order
(FemCantileverBase.cs:87-104 into DokRowMajor.cs:182-207): row offsets, columns and
values must equal dv_hex_assemble's bit for bit, which the CPU tests pin against the
oracle's DOK assembly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ne", [(1, 1, 1), (4, 3, 5), (8, 8, 8), (17, 6, 9)])
@pytest.mark.parametrize("moduli", ["uniform", "per_element"])
def test_device_assembly_bit_exact(ctx, native, rng, ne, moduli):
    import torch
    E = None if moduli == "uniform" else 10.0 ** rng.uniform(-2.0, 0.0, int(np.prod(ne)))
    ref = native.hex_stiffness(ne, E, scale=2.0, nu=0.3)
    n, nnz = native.hex_csr_size(ne)
    rp = torch.full((n + 1,), -1, dtype=torch.int32, device="cuda")
    ci = torch.full((nnz,), -1, dtype=torch.int32, device="cuda")
    va = torch.full((nnz,), float("nan"), dtype=torch.float64, device="cuda")
    dE = None if E is None else torch.from_numpy(E).cuda()
    torch.cuda.synchronize()
    native.hex_assemble_device(ctx, ne, rp.data_ptr(), ci.data_ptr(), va.data_ptr(),
                               None if dE is None else dE.data_ptr(), scale=2.0, nu=0.3)
    np.testing.assert_array_equal(rp.cpu().numpy(), ref.indptr)
    np.testing.assert_array_equal(ci.cpu().numpy(), ref.indices)
    np.testing.assert_array_equal(va.cpu().numpy().view(np.uint64), ref.data.view(np.uint64))


def _device_csr(A):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(v)).cuda() for v in (A.indptr.astype(np.int32),
                                                                        A.indices.astype(np.int32),
                                                                        A.data.astype(np.float64))]


def _export(M):
    e = M.export_duvi()
    return {k: v for k, v in e.items() if isinstance(v, np.ndarray)}


@pytest.mark.parametrize("case", ["hex_uniform", "hex_per_element", "hex_scaled_odd", "random", "transfer",
                                  "near_tolerance"])
def test_device_duvi_encoder_equals_host_encoder(ctx, native, rng, case):
    # dv_matrix_create_duvi_device encodes device CSR on the device: the exported SoA arrays,
    # the value table, the index width, the launch shape (node patterns / grid stencil where the
    # host encoder finds them) and the FP64 products equal the host-encoded matrix's bit for bit.
    import scipy.sparse as sp
    import torch
    if case == "hex_uniform":
        A = native.hex_stiffness((12, 9, 7))
    elif case == "hex_per_element":
        A = native.hex_stiffness((8, 6, 5), 10.0 ** rng.uniform(-2.0, 0.0, 240))
    elif case == "hex_scaled_odd":
        A = native.hex_stiffness((13, 5, 11), scale=4.0)
    elif case == "random":
        A = sp.random(500, 700, density=0.02, random_state=np.random.RandomState(3), format="csr")
        A.data = np.round(rng.standard_normal(A.nnz), 1)   # repeated values
        A.sort_indices()
    elif case == "transfer":
        A = native.hex_trilinear((8, 6, 6))
        A.sort_indices()
    else:   # values within the dictionary tolerance of each other
        A = native.hex_stiffness((6, 6, 6)).tocsr()
        A.data = A.data + rng.choice([0.0, 3e-11, -4e-11], A.nnz)
    n, m = A.shape
    for prec in ("f64", "f32"):
        H = native.SparseMatrix(ctx, A, "duvi", prec)
        rp, ci, va = _device_csr(A)
        torch.cuda.synchronize()
        D = native.SparseMatrix.duvi_from_device_csr(ctx, n, m, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), prec)
        eh, ed = _export(H), _export(D)
        assert eh.keys() == ed.keys()
        for k in eh:
            np.testing.assert_array_equal(eh[k].view(np.uint8), ed[k].view(np.uint8), err_msg=k)
        ih, idv = H.info(), D.info()
        for k in ("nblocks", "nuniq", "value_index_bits", "device_bytes"):
            assert ih[k] == idv[k], k
        if ih["kernel_variant"] in (203, 303):
            assert idv["kernel_variant"] == ih["kernel_variant"]
        x = rng.standard_normal(m)
        if prec == "f64":
            np.testing.assert_array_equal(D.Multiply(x), H.Multiply(x))
        H.release()
        D.release()
