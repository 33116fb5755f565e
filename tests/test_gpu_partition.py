"""GPU parity of the root partition: the counts of the nparts parts of every
query's root window (gfsm_batch_count_part) add up to the whole count, with
vertex labels ignored and matched, for single queries and for a batch that
shares query prefixes; and the cut the matcher applies is gfsm_partition_rows
over the device CCSR's row pointer."""
import numpy as np
import pytest

import gfsm_b200
from gfsm_b200 import synth

pytestmark = pytest.mark.gpu


def _batch(ctx, g, ks, seed):
    qs = [synth.rw_query(g, k, tree=(i % 2 == 0), seed=seed + i)[0] for i, k in enumerate(ks)]
    return ctx.prepare_queries([(q.n,) + tuple(q.directed()) + (None, q.vlabel) for q in qs])


@pytest.mark.parametrize("vl", [False, True])
def test_parts_add_up(gpu_ctx, gpu_ctx_vl, vl):
    ctx = gpu_ctx_vl if vl else gpu_ctx
    g = synth.ba(20000, 4, seed=11)
    g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=12)
    s, d = g.directed()
    data = ctx.graph_from_edges(g.n, s, d, None, g.vlabel).to_device()
    plans = _batch(ctx, g, [3, 4, 4, 3, 4, 3, 4, 4] if not vl else [3, 4, 5, 6, 7, 5, 4, 6], seed=40)
    whole, _ = ctx.batch_count(plans, data)
    assert whole.sum() > 0
    for nparts in (2, 3, 7):
        tot = np.zeros_like(whole)
        for part in range(nparts):
            c, _ = ctx.batch_count_part(plans, data, part, nparts)
            tot += c
        assert tot.tolist() == whole.tolist(), nparts
        # one query at a time gives the same parts
        single = [ctx.batch_count_part([plans[0]], data, part, nparts)[0][0] for part in range(nparts)]
        assert sum(int(x) for x in single) == int(whole[0])


def test_cut_is_partition_rows_over_the_device_ccsr(gpu_ctx):
    g = synth.rmat(12, 40000, seed=5)
    s, d = g.directed()
    data = gpu_ctx.graph_from_edges(g.n, s, d).to_device()
    rowptr, _, _, _ = data.download()
    q = synth.shape("4-cycle")
    plan = gpu_ctx.pre_process_query(gpu_ctx.graph_from_edges(q.n, *q.directed()))
    lo, bounds = gpu_ctx.root_partition(plan, data, 5)
    n = int(bounds[-1])
    assert bounds[0] == 0 and n > 0
    assert bounds.tolist() == gfsm_b200.partition_rows(rowptr, lo, lo + n, 5).tolist()
    # each part holds about a fifth of the window's entries (within one row)
    w = int(rowptr[lo + n]) - int(rowptr[lo])
    maxdeg = int(np.max(np.diff(rowptr[lo:lo + n + 1])))
    for k in range(5):
        got = int(rowptr[lo + int(bounds[k + 1])]) - int(rowptr[lo + int(bounds[k])])
        assert abs(got - w / 5) <= maxdeg
    # the parts' counts add up
    whole, _ = gpu_ctx.match_count(plan, data)
    assert sum(int(gpu_ctx.batch_count_part([plan], data, p, 5)[0][0]) for p in range(5)) == whole
