"""Full-size, memory-stressing parity: Barabasi-Albert n=4M, m=4 (~16M
edges), 16 Zipf(1.0) vertex labels, random-walk queries of 8-12 vertices
(trees and induced-cyclic), vertex labels matched.  Their frontiers exceed
MEMLIMIT, so the memory-bounded chunking path runs at full size.

No CPU enumerator reaches these counts (10^7 to 10^10 embeddings), so parity
is checked through properties that must hold whatever the size: the count is
the same under the default MEMLIMIT and a 2 GB one (many more chunks and
retries), under the host-driven and the graph-driven schedule, batched and
one at a time, and -- for the smaller ones -- through the 64 MiB
no-allocation path."""
import ctypes as C

import pytest

import gfsm_b200
from gfsm_b200 import synth

pytestmark = pytest.mark.gpu

# (walk seed, size, tree) of queries whose search finishes in seconds; chosen
# from the workload's random-walk stream by running it under a candidate cap.
QUERIES = [(8, 10, False), (11, 8, True), (14, 11, False), (12, 9, False)]


@pytest.fixture(scope="module")
def ba4m():
    g = synth.ba(4_000_000, 4, seed=0)
    g.vlabel = synth.vlabels(g.n, 16, 1.0, seed=100)
    return g


def _plans(ctx, g):
    out = []
    for seed, k, tree in QUERIES:
        qg, _ = synth.rw_query(g, k, tree=tree, seed=seed)
        qs, qd = qg.directed()
        out.append(ctx.pre_process_query(ctx.graph_from_edges(qg.n, qs, qd, None, qg.vlabel)))
    return out


def test_chunking_invariance_full_size(ba4m, monkeypatch):
    g = ba4m
    s, d = g.directed()
    results = {}
    for name, kw, drv in (("default", {}, "host"), ("2GB", dict(mem_limit=2_000_000_000), "host"),
                          ("graph", {}, "graph")):
        monkeypatch.setenv("GFSM_DRIVER", drv)
        ctx = gfsm_b200.GFSM(device=0, vertex_labels=1, **kw)
        data = ctx.graph_from_edges(g.n, s, d, None, g.vlabel)
        plans = _plans(ctx, g)
        single = [ctx.match_count(p, data) for p in plans]
        batch, bst = ctx.batch_count(plans, data)
        results[name] = ([c for c, _ in single], batch.tolist(), [st["steps"] for _, st in single])
        if name == "default":
            # the no-allocation path, on the smaller queries
            for p, (c, st) in list(zip(plans, single))[:2]:
                cnt = C.c_uint64()
                assert ctx._lib.gfsm_match_count_noalloc(p.handle, data.handle, None, C.byref(cnt)) == 0
                assert cnt.value == c
        ctx.close()
    ref = results["default"][0]
    assert all(c > 1_000_000 for c in ref), ref
    for name, (single, batch, steps) in results.items():
        assert single == ref, name
        assert batch == ref, name
    # the 2 GB limit forces more, smaller steps than the default
    assert sum(results["2GB"][2]) > sum(results["default"][2])
