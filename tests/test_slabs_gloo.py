"""Slab decomposition host logic on CPU with gloo (world sizes 2 and 3): the owned rows of each
rank, renumbered to [ghost plane below | owned | ghost plane above], times x_ext after the halo
exchange reproduce the global product; the slab Jacobi-PCG (all-reduced dot products and stop
test) reproduces the oracle's single-domain PCG.  The device product itself is the library's
SpMV (SlabOperator), covered on one GPU in the GPU tests."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _CpuSlab:
    """The slab operator's host logic with the local product done by scipy (test side)."""

    def __init__(self, A, ne, rank, world):
        import torch
        from compressiontests_b200 import slabs
        self.rank, self.world, self.group = rank, world, None
        self.A_loc, self.lo, self.hi, self.g_lo, self.g_hi = slabs.local_operator(A, ne, rank, world)
        self.n_own = self.hi - self.lo
        self.x_ext = torch.zeros(self.A_loc.shape[1], dtype=torch.float64)
        self.inv_diag = torch.from_numpy(1.0 / self.A_loc[:, self.g_lo:self.g_lo + self.n_own].diagonal())

    def apply(self, x_own, y_own):
        import torch
        from compressiontests_b200 import slabs
        self.x_ext[self.g_lo:self.g_lo + self.n_own] = x_own
        slabs.exchange_halos(self.x_ext, self.g_lo, self.n_own, self.g_hi, self.rank, self.world)
        y_own.copy_(torch.from_numpy(self.A_loc @ self.x_ext.numpy()))


def _worker(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import compressiontests_b200 as cb
    from compressiontests_b200 import replicas, slabs
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        ne = (4, 3, 5)
        A = cb.hex_stiffness(ne)
        x = np.random.default_rng(7).standard_normal(A.shape[0])
        op = _CpuSlab(A, ne, rank, world)
        y = torch.empty(op.n_own, dtype=torch.float64)
        op.apply(torch.from_numpy(x[op.lo:op.hi].copy()), y)
        prod = replicas.gather_to_root((op.lo, y.numpy()), world, rank)
        b = cb.traction_rhs(ne)
        xs, its, conv = slabs.slab_pcg(op, torch.from_numpy(b[op.lo:op.hi].copy()), 2000, 1e-10, rel_l2=True)
        sol = replicas.gather_to_root((op.lo, xs.numpy(), its, conv), world, rank)
        q.put((rank, prod, sol, None))
    except Exception as e:
        q.put((rank, None, None, f"{type(e).__name__}: {e}"))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_product_and_pcg_match_single_domain(world, oracle):
    import compressiontests_b200 as cb
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, prod, sol, err = q.get(timeout=120)
        assert err is None, err
        out[r] = (prod, sol)
    for p in procs:
        p.join(timeout=60)
    ne = (4, 3, 5)
    A = cb.hex_stiffness(ne)
    x = np.random.default_rng(7).standard_normal(A.shape[0])
    prod, sol = out[0]
    y = np.concatenate([v for _, v in sorted(prod, key=lambda t: t[0])])
    np.testing.assert_allclose(y, A @ x, rtol=0, atol=1e-12 * np.max(np.abs(A) @ np.abs(x)))
    xs = np.concatenate([v for _, v, _, _ in sorted(sol, key=lambda t: t[0])])
    its = {i for _, _, i, _ in sol}
    assert all(c for _, _, _, c in sol) and len(its) == 1
    b = cb.traction_rhs(ne)
    x_ref, it_ref = oracle.pcg_jacobi(oracle.Csr.from_scipy(A), b, 2000, 1e-10, rel_l2=True)
    assert abs(its.pop() - it_ref) <= 1
    assert np.max(np.abs(xs - x_ref)) <= 1e-7 * np.max(np.abs(x_ref))


def test_slab_planes_cover_the_mesh():
    from compressiontests_b200 import slabs
    ne = (6, 5, 9)
    for world in (1, 2, 3, 10):
        spans = [slabs.slab_planes(ne, r, world) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == ne[2] + 1
        assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
    with pytest.raises(ValueError):
        slabs.slab_planes(ne, 0, 11)
