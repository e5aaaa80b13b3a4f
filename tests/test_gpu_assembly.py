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
