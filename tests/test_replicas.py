"""The replica (multi-process) path on CPU with gloo, world size 2: disjoint
shards covering every unit, host-side gather in rank order, max-over-ranks
timing -- the plumbing bench.py uses across GPUs."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from ket_b200 import replicas
    r, w, _ = replicas.init("gloo", timeout_s=60)
    units = list(range(11))
    mine = replicas.shard(units, r, w)
    done = [u * u for u in mine]  # each rank's independent work
    allres = replicas.gather(done)
    m = replicas.max_over_ranks(float(10 * (r + 1)))
    replicas.barrier()
    import torch.distributed as dist
    dist.destroy_process_group()
    q.put((r, mine, allres, m))


def test_two_rank_replicas_on_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    from ket_b200.replicas import unshard
    (r0, m0, all0, mx0), (r1, m1, all1, mx1) = res
    assert sorted(m0 + m1) == list(range(11)) and not set(m0) & set(m1)
    assert all0 == all1
    assert unshard(all0) == [u * u for u in range(11)]
    assert mx0 == mx1 == 20.0
