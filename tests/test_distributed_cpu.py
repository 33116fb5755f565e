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


def _partition_rank(rank, world, port, q):
    """One rank of the root partition, on the CPU: the rank's degree-balanced
    part of the data graph's CCSR rows (gfsm_partition_rows, the cut the
    matcher applies to every root window) counted by the oracle, then the
    per-query counts summed over the ranks with an all-reduce."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import numpy as np
    import torch

    import gfsm_b200
    from oracle import oracle as O
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    d = O.Graph(path=os.path.join(gold, "data", "ba300.g"))
    deg = O.row_degrees(d)
    rowptr = np.zeros(len(deg) + 1, np.uint32)
    np.cumsum(deg, out=rowptr[1:])
    bounds = gfsm_b200.partition_rows(rowptr, 0, len(deg), world)
    mine = []
    for qn in ("_3_triangle", "_4_square", "_5_road5"):
        oq = O.Graph(path=os.path.join(gold, "queries", qn + ".g"))
        mine.append(O.ffs_count_rows(oq, O.Plan(oq), d, int(bounds[rank]), int(bounds[rank + 1]), threads=2))
    t = torch.tensor(mine, dtype=torch.int64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    q.put((rank, [int(x) for x in bounds], mine, t.tolist(), int(rowptr[-1])))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_root_partition_gloo_ranks(world):
    import json
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    counts = json.load(open(os.path.join(gold, "counts.json")))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_partition_rank, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=300) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = [counts[qn + "|ba300"]["count"] for qn in ("_3_triangle", "_4_square", "_5_road5")]
    bounds = out[0][1]
    for r, b, mine, total, entries in out:
        assert b == bounds                      # every rank cuts the same way
        assert total == want                    # the parts add up to the whole count
    assert sum(sum(m) for _, _, m, _, _ in out) == sum(want)
    assert all(b0 < b1 for b0, b1 in zip(bounds, bounds[1:]))  # no empty part on this graph
