"""Structured cantilever models feeding the solvers (3-D hexa, 3 dofs/node).

Restates the model contract the reference's solvers consume,
IGeometricMultigridModel (src/MGroup.Solvers/Multigrid/IGeometricMultigridModel.cs:7-65),
for the hexahedral cantilever of FemCantilever3D
(tests/MGroup.LinearAlgebra.Tests/TestData/SparseLinearSystems/FemCantilever3D.cs):
unit-cube top3d element stiffness regardless of element size, density-scaled
assembly in element order, all nodes with x index 0 clamped, node ids
x-fastest, manufactured right-hand side b = K u_EB from the Euler-Bernoulli
beam field (FemCantileverBase.cs:53-82).  Assembly, transfers and the
trilinear hierarchy are computed by the native library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from . import _native as N


def hex_stiffness(ne, elem_E=None, scale=1.0, E=1.0, nu=0.3):
    """Free-dof stiffness of an ne[0] x ne[1] x ne[2] hexa grid as scipy CSR."""
    ne = np.ascontiguousarray(ne, np.int32)
    nr, nnz = C.c_int32(), C.c_int64()
    N.check(N.lib().dv_hex_csr_size(N.ptr(ne), C.byref(nr), C.byref(nnz)))
    rp = np.empty(nr.value + 1, np.int32)
    ci = np.empty(nnz.value, np.int32)
    va = np.empty(nnz.value, np.float64)
    e = None if elem_E is None else np.ascontiguousarray(elem_E, np.float64)
    N.check(N.lib().dv_hex_assemble(N.ptr(ne), N.ptr(e), scale, E, nu, N.ptr(rp), N.ptr(ci), N.ptr(va)))
    return sp.csr_matrix((va, ci, rp), shape=(nr.value, nr.value))


def hex_assemble_device(ctx, ne, d_rowptr, d_col, d_val, d_elem_E=None, scale=1.0, E=1.0, nu=0.3):
    """The same free-dof stiffness assembled on the device into caller-owned device arrays
    (pointers; sizes from hex_csr_size), bit for bit equal to hex_stiffness."""
    ne = np.ascontiguousarray(ne, np.int32)
    N.check(N.lib().dv_hex_assemble_device(ctx.h, N.ptr(ne), d_elem_E, scale, E, nu, d_rowptr, d_col, d_val))


def hex_csr_size(ne):
    """(rows, stored entries) of the free-dof hexa stiffness."""
    ne = np.ascontiguousarray(ne, np.int32)
    nr, nnz = C.c_int32(), C.c_int64()
    N.check(N.lib().dv_hex_csr_size(N.ptr(ne), C.byref(nr), C.byref(nnz)))
    return nr.value, nnz.value


def hex_trilinear(ne_fine):
    """Trilinear prolongation of the factor-2 vertex coarsening (coarse nodes at the even
    fine nodes and the last one, so odd element counts coarsen to ceil(n/2))."""
    ne = np.ascontiguousarray(ne_fine, np.int32)
    nr, nc, nnz = C.c_int32(), C.c_int32(), C.c_int64()
    N.check(N.lib().dv_hex_trilinear_size(N.ptr(ne), C.byref(nr), C.byref(nc), C.byref(nnz)))
    rp = np.empty(nr.value + 1, np.int32)
    ci = np.empty(nnz.value, np.int32)
    va = np.empty(nnz.value, np.float64)
    N.check(N.lib().dv_hex_trilinear(N.ptr(ne), N.ptr(rp), N.ptr(ci), N.ptr(va)))
    return sp.csr_matrix((va, ci, rp), shape=(nr.value, nc.value))


def galerkin(A, P):
    """Galerkin coarse operator P^T A P (native, sorted rows)."""
    ah, ka = _host(A)
    ph, kp = _host(P)
    n, nnz = C.c_int32(), C.c_int64()
    N.check(N.lib().dv_galerkin_size(C.byref(ah), C.byref(ph), C.byref(n), C.byref(nnz)))
    rp = np.empty(n.value + 1, np.int32)
    ci = np.empty(nnz.value, np.int32)
    va = np.empty(nnz.value, np.float64)
    N.check(N.lib().dv_galerkin(C.byref(ah), C.byref(ph), N.ptr(rp), N.ptr(ci), N.ptr(va)))
    del ka, kp
    return sp.csr_matrix((va, ci, rp), shape=(n.value, n.value))


def duvi_encode(A, value_index_bits=0, dedup_tol=1e-10):
    """DuVi SoA arrays of a CSR matrix on the host (FromDokRowMajor), no device needed:
    dict of row_to_col, row_to_dist, col_idx, dist, vidx (uint32), values, vi_bits."""
    ah, ka = _host(A)
    nb, nu, bits = C.c_int64(), C.c_int64(), C.c_int32()
    N.check(N.lib().dv_duvi_encode(C.byref(ah), value_index_bits, dedup_tol, C.byref(nb), C.byref(nu), C.byref(bits),
                                   None, None, None, None, None, None))
    n, nnz = A.shape[0], A.nnz
    out = dict(row_to_col=np.empty(n + 1, np.uint32), row_to_dist=np.empty(n + 1, np.uint32),
               col_idx=np.empty(nb.value, np.uint32), dist=np.empty(nnz, np.uint8), vidx=np.empty(nnz, np.uint32),
               values=np.empty(nu.value, np.float64))
    N.check(N.lib().dv_duvi_encode(C.byref(ah), value_index_bits, dedup_tol, C.byref(nb), C.byref(nu), C.byref(bits),
                                   *(N.ptr(out[k]) for k in ("row_to_col", "row_to_dist", "col_idx", "dist", "vidx",
                                                             "values"))))
    del ka
    out["vi_bits"] = bits.value
    return out


def units_encode(A, dedup_tol=1e-10):
    """CPU DuVi Unit stream of a CSR matrix (DuViCompressedSparseMatrix's units, flat):
    dict of bytes (uint8), unit_offsets (int64, n_units + 1), vidx (int32), values."""
    ah, ka = _host(A)
    nu_, nb, ni, nq = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
    N.check(N.lib().dv_units_encode(C.byref(ah), dedup_tol, C.byref(nu_), C.byref(nb), C.byref(ni), C.byref(nq),
                                    None, None, None, None))
    out = dict(bytes=np.empty(nb.value, np.uint8), unit_offsets=np.empty(nu_.value + 1, np.int64),
               vidx=np.empty(ni.value, np.int32), values=np.empty(nq.value, np.float64))
    N.check(N.lib().dv_units_encode(C.byref(ah), dedup_tol, C.byref(nu_), C.byref(nb), C.byref(ni), C.byref(nq),
                                    *(N.ptr(out[k]) for k in ("bytes", "unit_offsets", "vidx", "values"))))
    del ka
    return out


def units_decode(shape, units):
    """CSR matrix (scipy) of a Unit stream produced by units_encode (or the reference)."""
    n, m = shape
    b, vi, va = (np.ascontiguousarray(units[k]) for k in ("bytes", "vidx", "values"))
    b = b.astype(np.uint8, copy=False)
    vi = vi.astype(np.int32, copy=False)
    va = va.astype(np.float64, copy=False)
    nnz = C.c_int64()
    args = (n, m, N.ptr(b), b.size, N.ptr(vi), vi.size, N.ptr(va), va.size, C.byref(nnz))
    N.check(N.lib().dv_units_decode(*args, None, None, None))
    rp = np.empty(n + 1, np.int32)
    ci = np.empty(nnz.value, np.int32)
    vv = np.empty(nnz.value, np.float64)
    N.check(N.lib().dv_units_decode(*args, N.ptr(rp), N.ptr(ci), N.ptr(vv)))
    return sp.csr_matrix((vv, ci, rp), shape=(n, m))


def _host(a):
    from .sparse import _csr_arrays
    rp, ci, va, shape = _csr_arrays(a)
    return N.csr_host(rp, ci, va, shape)


def galerkin_hierarchy(ne, max_coarse_dofs=1000, elem_E=None, E=1.0, nu=0.3):
    """Hierarchy of an arbitrary ne[0] x ne[1] x ne[2] cantilever: vertex-based factor-2
    coarsening (odd counts coarsen to ceil(n/2)), trilinear P, Galerkin A_{l+1} = P^T A_l P,
    until the coarsest level has at most max_coarse_dofs dofs.  Returns (A_levels, P_levels)."""
    ne = [int(n) for n in ne]
    A = [hex_stiffness(ne, elem_E, 1.0, E, nu)]
    P = []
    while A[-1].shape[0] > max_coarse_dofs and max(ne) > 1:
        P.append(hex_trilinear(ne))
        A.append(galerkin(A[-1], P[-1]))
        ne = [(n + 1) // 2 for n in ne]
    return A, P


def cartesian_transfer(dim, ne_fine, ne_coarse, dofs_per_node, fine_free, coarse_free):
    """Restriction and interpolation of IGeometricMultigridModel.cs:76-194 (free-dof submatrices)."""
    f = np.array(list(ne_fine) + [1] * (3 - len(ne_fine)), np.int32)
    c = np.array(list(ne_coarse) + [1] * (3 - len(ne_coarse)), np.int32)
    ff = np.ascontiguousarray(fine_free, np.int32)
    cf = np.ascontiguousarray(coarse_free, np.int32)
    nr, npp = C.c_int64(), C.c_int64()
    N.check(N.lib().dv_cartesian_transfer_size(dim, N.ptr(f), N.ptr(c), dofs_per_node, len(ff), N.ptr(ff), len(cf),
                                               N.ptr(cf), C.byref(nr), C.byref(npp)))
    rrp = np.empty(len(cf) + 1, np.int32)
    rci = np.empty(nr.value, np.int32)
    rva = np.empty(nr.value)
    prp = np.empty(len(ff) + 1, np.int32)
    pci = np.empty(npp.value, np.int32)
    pva = np.empty(npp.value)
    N.check(N.lib().dv_cartesian_transfer(dim, N.ptr(f), N.ptr(c), dofs_per_node, len(ff), N.ptr(ff), len(cf),
                                          N.ptr(cf), N.ptr(rrp), N.ptr(rci), N.ptr(rva), N.ptr(prp), N.ptr(pci),
                                          N.ptr(pva)))
    R = sp.csr_matrix((rva, rci, rrp), shape=(len(cf), len(ff)))
    P = sp.csr_matrix((pva, pci, prp), shape=(len(ff), len(cf)))
    return R, P


class FemCantilever3D:
    """Hexahedral cantilever model (the IGeometricMultigridModel of the reference tests)."""

    NumDofsPerNode = 3

    def __init__(self, numElementsPerAxis, lengthPerAxis=(20.0, 1.0, 1.0), ElasticityModulus=1.0, PoissonRatio=0.3,
                 DistributedLoad=1.0, ElementDensities=None):
        self.NumElements = tuple(int(v) for v in numElementsPerAxis)
        self.Length = tuple(float(v) for v in lengthPerAxis)
        self.ElasticityModulus = ElasticityModulus
        self.PoissonRatio = PoissonRatio
        self.DistributedLoad = DistributedLoad
        self.ElementDensities = ElementDensities
        nn = [n + 1 for n in self.NumElements]
        self.NumNodes = tuple(nn)
        self.NumDofsAll = 3 * nn[0] * nn[1] * nn[2]
        self.NumDofsFree = self.NumDofsAll - self.NumDofsAll // nn[0]
        L1, L2 = self.Length[1], self.Length[2]
        self.MomentOfInertia = L1 * L2 / 12 * L2 * L2

    def FindFreeDofs(self):
        nx = self.NumNodes[0]
        nodes = np.arange(self.NumDofsAll // 3)
        free_nodes = nodes[nodes % nx != 0]
        return (3 * free_nodes[:, None] + np.arange(3)).ravel().astype(np.int32)

    def stiffness(self):
        return hex_stiffness(self.NumElements, self.ElementDensities, 1.0, self.ElasticityModulus, self.PoissonRatio)

    def free_displacements(self):
        """Euler-Bernoulli displacements on the free dofs (FemCantileverBase.cs:70-82, 160-182)."""
        nx, ny, nz = self.NumNodes
        ex, ey, ez = self.NumElements
        Lx, Ly, Lz = self.Length
        k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(1, nx), indexing="ij")
        x = i.ravel() * (Lx / ex)
        z = k.ravel() * (Lz / ez) - Lz / 2
        q, E, I, L = self.DistributedLoad, self.ElasticityModulus, self.MomentOfInertia, Lx
        w = -q / (24 * E * I) * (x ** 4 - 4 * L * x ** 3 + 6 * L * L * x * x)
        rot = -q / (6 * E * I) * (x ** 3 - 3 * L * x * x + 3 * L * L * x)
        u = -rot * z
        out = np.zeros((x.size, 3))
        out[:, 0] = u
        out[:, 2] = w
        return out.ravel()

    def CreateLinearSystem(self):
        A = self.stiffness()
        b = A @ self.free_displacements()
        return A, b

    def CreateCoarserModel(self):
        ne = [n >> 1 if n > 1 else n for n in self.NumElements]   # MakeCartesianCoarserElementsPerAxis
        return FemCantilever3D(ne, self.Length, self.ElasticityModulus, self.PoissonRatio, self.DistributedLoad)

    def transfer_to(self, coarser):
        return cartesian_transfer(3, self.NumElements, coarser.NumElements, 3, self.FindFreeDofs(),
                                  coarser.FindFreeDofs())


def traction_rhs(ne, t=(0.0, 0.0, -1.0)):
    """Consistent nodal loads of a uniform traction t on the face x = ne[0] (unit cubes)."""
    nx, ny, nz = ne[0] + 1, ne[1] + 1, ne[2] + 1
    wy = np.ones(ny)
    wy[0] = wy[-1] = 0.5
    wz = np.ones(nz)
    wz[0] = wz[-1] = 0.5
    w = np.outer(wz, wy)   # (k, j)
    b = np.zeros((nz, ny, nx - 1, 3))
    for d in range(3):
        b[:, :, -1, d] = w * t[d]
    return b.ravel()


def random_face_loads(ne, k, seed=0):
    """k load cases with i.i.d. N(0, 1) nodal forces (all 3 components) on the free face x = ne[0].

    Returns an n_free x k array (column j = load case j), dofs ordered as traction_rhs.
    """
    nx, ny, nz = ne[0] + 1, ne[1] + 1, ne[2] + 1
    rng = np.random.default_rng(seed)
    B = np.zeros((nz, ny, nx - 1, 3, k))
    B[:, :, -1, :, :] = rng.standard_normal((nz, ny, 3, k))
    return B.reshape(-1, k)


def coarsen_moduli(ne, elem_E):
    """Average of the 8 children of every coarse element (factor-2 grids)."""
    e = np.asarray(elem_E, np.float64).reshape(ne[2], ne[1], ne[0])
    return e.reshape(ne[2] // 2, 2, ne[1] // 2, 2, ne[0] // 2, 2).mean(axis=(1, 3, 5)).ravel()


def hex_hierarchy(ne, coarse_ne=8, elem_E=None, E=1.0, nu=0.3):
    """Factor-2 hierarchy down to coarse_ne elements along the shortest axis.

    Level l is the grid with element size 2^l re-discretised: K_l = 2^l * sum_e E_e Ke
    (the stiffness of 3-D linear elasticity scales with the element size), with
    coarse moduli averaged over children.  With uniform moduli this equals the
    Galerkin product P^T K P of trilinear interpolation.  Returns (A_levels, P_levels).
    """
    ne = list(ne)
    A, P = [], []
    scale = 1.0
    e = elem_E
    while True:
        A.append(hex_stiffness(ne, e, scale, E, nu))
        if min(ne) <= coarse_ne or any(n % 2 for n in ne):
            break
        P.append(hex_trilinear(ne))
        if e is not None:
            e = coarsen_moduli(ne, e)
        ne = [n // 2 for n in ne]
        scale *= 2.0
    return A, P


def cantilever_batch(n_meshes=32, lo=8, hi=48, seed=0, max_coarse_dofs=1000):
    """n_meshes independent cantilevers whose three edge lengths are drawn uniformly from
    lo..hi elements (seeded), each with its Galerkin hierarchy and the unit traction load
    on its free face.  Returns (dims, meshes, rhs) with meshes = [(A_levels, P_levels)]."""
    rng = np.random.default_rng(seed)
    dims = [tuple(int(v) for v in rng.integers(lo, hi + 1, size=3)) for _ in range(n_meshes)]
    meshes = [galerkin_hierarchy(ne, max_coarse_dofs) for ne in dims]
    rhs = [traction_rhs(ne) for ne in dims]
    return dims, meshes, rhs
