"""Slab decomposition of a structured hexahedral operator over several GPUs.

The operator of an nx x ny x nz element cantilever (free nodes numbered x-fastest, then y,
then z) is split into contiguous runs of z node planes, one run per rank.  A rank owns the
rows of its planes; their columns reach one node plane below and one above (the 27-point
coupling of trilinear hexahedra), so a product needs the neighbouring ranks' boundary planes:

    x_ext = [ghost plane below | owned planes | ghost plane above]   (contiguous, global order)
    y_own = A_loc x_ext,   A_loc = rows of the owned planes, columns shifted to x_ext

One halo exchange per product (send the first owned plane down, the last up; receive the
ghosts), then the local product on the device (the library's SpMV through the C ABI).  The
Jacobi-PCG built on it all-reduces its three dot products and the max-norm stop test per
iteration.  Communication goes through torch.distributed: NCCL between GPUs, gloo on CPU for
the host-logic tests.  The reference solves on one device; this layer has no counterpart
there.
"""
from __future__ import annotations

import scipy.sparse as sp

from .replicas import shard


def plane_dofs(ne):
    """Free dofs of one z node plane (3 per node, x index 0 clamped)."""
    return 3 * int(ne[0]) * (int(ne[1]) + 1)


def slab_planes(ne, rank, world):
    """Node planes [z0, z1) owned by this rank (a balanced split of the nz + 1 planes)."""
    nz1 = int(ne[2]) + 1
    if world > nz1:
        raise ValueError("more ranks than node planes")
    return shard(nz1, rank, world)


def local_operator(A, ne, rank, world):
    """Rows of the owned planes of the global operator A (scipy CSR), columns renumbered to x_ext:
    column 0 is the first dof of the ghost plane below (or of the first owned plane on rank 0).
    Returns (A_loc, lo, hi, g_lo, g_hi): owned rows [lo, hi) of the global numbering and the
    ghost plane sizes below and above (0 at the ends)."""
    pd = plane_dofs(ne)
    z0, z1 = slab_planes(ne, rank, world)
    lo, hi = z0 * pd, z1 * pd
    g_lo = pd if rank > 0 else 0
    g_hi = pd if rank < world - 1 else 0
    c0 = lo - g_lo
    A = sp.csr_matrix(A)
    rows = A[lo:hi]
    cols = rows.indices
    if cols.size and (cols.min() < c0 or cols.max() >= hi + g_hi):
        raise ValueError("the operator couples planes further apart than one")
    A_loc = sp.csr_matrix((rows.data, cols - c0, rows.indptr), shape=(hi - lo, g_lo + (hi - lo) + g_hi))
    return A_loc, lo, hi, g_lo, g_hi


def exchange_halos(x_ext, g_lo, n_own, g_hi, rank, world, group=None):
    """Fills the ghost parts of x_ext (a 1-D torch tensor [ghost below | owned | ghost above]) from
    the neighbouring ranks: every rank sends its first owned plane down and its last owned plane
    up.  Point-to-point, all sends and receives posted before any wait."""
    if world == 1:
        return
    import torch.distributed as dist
    own = x_ext[g_lo:g_lo + n_own]
    ops = []
    if rank > 0:
        ops.append(dist.P2POp(dist.isend, own[:g_lo].contiguous(), rank - 1, group))
        ops.append(dist.P2POp(dist.irecv, x_ext[:g_lo], rank - 1, group))
    if rank < world - 1:
        ops.append(dist.P2POp(dist.isend, own[n_own - g_hi:].contiguous(), rank + 1, group))
        ops.append(dist.P2POp(dist.irecv, x_ext[g_lo + n_own:], rank + 1, group))
    for req in dist.batch_isend_irecv(ops):
        req.wait()


def all_reduce_sum(values, world, group=None, op="sum"):
    """Sum (or max) of a few float64 scalars over ranks (one collective)."""
    if world == 1:
        return values
    import torch
    import torch.distributed as dist
    t = values if isinstance(values, torch.Tensor) else torch.tensor(values, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM, group=group)
    return t


class SlabOperator:
    """The owned rows of a slab-decomposed operator as a device matrix (CSR or DuVi, FP64)
    and its extended vector; apply() exchanges the halos and runs the local product."""

    def __init__(self, ctx, A, ne, rank, world, fmt="csr", group=None):
        import torch
        from .sparse import SparseMatrix
        self.rank, self.world, self.group = rank, world, group
        A_loc, self.lo, self.hi, self.g_lo, self.g_hi = local_operator(A, ne, rank, world)
        self.n_own = self.hi - self.lo
        self.ctx = ctx
        self.M = SparseMatrix(ctx, A_loc, fmt, "f64")
        dev = f"cuda:{ctx.device}" if hasattr(ctx, "device") else "cuda"
        self.x_ext = torch.zeros(A_loc.shape[1], dtype=torch.float64, device=dev)
        diag = A_loc[:, self.g_lo:self.g_lo + self.n_own].diagonal()
        self.inv_diag = torch.from_numpy(1.0 / diag).to(dev)

    def apply(self, x_own, y_own):
        """y_own = (A x)_own for the owned part x_own of x (device tensors)."""
        import torch
        torch.cuda.current_stream().synchronize()
        self.x_ext[self.g_lo:self.g_lo + self.n_own].copy_(x_own)
        exchange_halos(self.x_ext, self.g_lo, self.n_own, self.g_hi, self.rank, self.world, self.group)
        torch.cuda.synchronize()
        self.M.multiply_device(self.x_ext.data_ptr(), y_own.data_ptr(), "f64")
        self.ctx.synchronize()

    def release(self):
        self.M.release()


def slab_pcg(op: SlabOperator, b_own, max_iterations=20000, tol=1e-8, rel_l2=True):
    """Jacobi PCG on a slab-decomposed operator (the iteration of dv_pcg_solve: the same stop
    test after the x / r update, max |r_i| <= tol or ||r||_2 <= tol ||b||_2), every rank holding
    its owned part.  Returns (x_own, iterations, converged)."""
    import torch
    w, g = op.world, op.group
    x = torch.zeros_like(b_own)
    r = b_own.clone()
    z = op.inv_diag * r
    p = z.clone()
    ap = torch.empty_like(b_own)

    def red(*vals):   # sums over ranks, on the data's device (NCCL needs device tensors)
        if w == 1:
            return list(vals)
        t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=b_own.device)
        return all_reduce_sum(t, w, g).tolist()

    bb, rz = red(float(b_own @ b_own), float(r @ z))
    for it in range(max_iterations + 1):
        op.apply(p, ap)
        (pap,) = red(float(p @ ap))
        a = rz / pap
        x += a * p
        r -= a * ap
        rr, rmax_local = float(r @ r), float(r.abs().max()) if r.numel() else 0.0
        (rr,) = red(rr)
        rmax = all_reduce_sum(torch.tensor([rmax_local], dtype=torch.float64, device=b_own.device), w, g,
                              op="max")[0].item() if w > 1 else rmax_local
        if (rr <= tol * tol * bb) if rel_l2 else (rmax <= tol):
            return x, it, True
        z = op.inv_diag * r
        (rz_new,) = red(float(r @ z))
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x, max_iterations, False
