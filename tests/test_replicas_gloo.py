"""Multi-process host logic of replica runs (CPU, gloo, world_size 2): sharding of
independent units, max-over-ranks timing and gathering, plus a failing rank that the
other ranks see as an error instead of a hang."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q, fail_rank):
    import datetime
    import torch.distributed as dist
    from compressiontests_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        lo, hi = replicas.shard(37, rank, world)
        mine = list(range(lo, hi))
        allu = replicas.gather_to_root(mine, world, rank)
        t = replicas.max_over_ranks(1.0 + rank, world)
        if rank == fail_rank:
            raise RuntimeError("planted failure on this rank")
        dist.barrier()   # the healthy rank waits here for the failed one
        q.put((rank, allu, t, None))
    except Exception as e:   # report, do not hang
        q.put((rank, None, None, type(e).__name__))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(res, key=lambda r: r[0])


def test_shard_partitions_units():
    from compressiontests_b200 import replicas
    for n, w in ((37, 2), (8, 8), (5, 8), (0, 3)):
        got = [replicas.shard(n, r, w) for r in range(w)]
        assert got[0][0] == 0 and got[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
        sizes = [h - l for l, h in got]
        assert max(sizes) - min(sizes) <= 1


def test_weighted_shard_balances_meshes(native):
    from compressiontests_b200 import replicas
    dims = [tuple(int(v) for v in d) for d in np.random.default_rng(20261203).integers(8, 49, (32, 3))]
    dofs = [3 * a * (b + 1) * (c + 1) for a, b, c in dims]
    parts = replicas.shard_weighted(dofs, 4)
    assert sorted(i for p in parts for i in p) == list(range(32))
    loads = [sum(dofs[i] for i in p) for p in parts]
    assert max(loads) <= 1.15 * np.mean(loads)
    assert parts == replicas.shard_weighted(dofs, 4)   # deterministic


def test_two_gloo_ranks_shard_and_max():
    res = _run(2)
    assert [r[3] for r in res] == [None, None]
    units = [u for part in res[0][1] for u in part]
    assert units == list(range(37))
    assert res[0][2] == res[1][2] == 2.0


def test_failing_rank_is_seen_not_hung():
    res = _run(2, fail_rank=1)
    assert res[1][3] == "RuntimeError"
    assert res[0][3] is not None   # the healthy rank's barrier ends with an error (peer gone or timeout)
