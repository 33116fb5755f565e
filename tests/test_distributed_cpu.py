"""The N>1 bench path on CPU: two gloo ranks on 127.0.0.1.  Each rank
builds its own seeded batch (weak scaling, no collective on the data path);
the whole-job value is all ranks' queries over the slowest rank's time."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    secs = [2.0, 3.0][rank]
    v = bench.weak_scaling_value(dist, 100 * (rank + 1), secs, None)
    mx = bench.max_over_ranks(dist, float(rank + 7), None)
    g, qs = bench.make_workload(rank, 4)
    q.put((rank, v, mx, [x.n for x in qs], int(qs[0].src.sum())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=300) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, v0, m0, n0, s0), (r1, v1, m1, n1, s1) = out
    assert v0 == v1 == pytest.approx(300 / 3.0)
    assert m0 == m1 == 8.0
    # each rank draws its own queries from the same data graph
    assert (n0, s0) != (n1, s1)
