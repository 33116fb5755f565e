"""gfsm_match_count_noalloc: the count path for callers that may not allocate
device memory during a match (a fixed memory budget or pool, or a
latency-critical path that cannot take cudaMalloc/cudaFree's implicit
synchronisation).  Through the C ABI, its counts must equal
gfsm_match_count's exactly, on two calls in a row (the fixed scratch array
keeps the previous call's contents), and device memory must not change
between calls.  This file is collected last on purpose."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

import gfsm_b200
from gfsm_b200 import _lib, synth

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
COUNTS = json.load(open(os.path.join(GOLD, "counts.json")))


def _noalloc_rc(ctx, plan, data):
    cnt = C.c_uint64()
    rc = ctx._lib.gfsm_match_count_noalloc(plan.handle, data.handle, None, C.byref(cnt))
    return rc, cnt.value


def _noalloc(ctx, plan, data):
    rc, cnt = _noalloc_rc(ctx, plan, data)
    assert rc == 0, gfsm_b200.GFSMError(rc)
    return cnt


def test_noalloc_matches_match_count():
    import torch
    ctx = gfsm_b200.GFSM(device=0)
    vctx = gfsm_b200.GFSM(device=0, vertex_labels=1)
    cases = []
    d1 = ctx.file_parse(os.path.join(GOLD, "data", "er200.g")).to_device()
    for qn in ("_3_triangle", "_4_square", "_5_road5", "_5_plus"):
        cases.append((ctx, ctx.pre_process_query(ctx.file_parse(os.path.join(GOLD, "queries", qn + ".g"))), d1))
    # a larger graph whose frontier must be chunked through the fixed scratch
    g = synth.ba(20000, 4, seed=3)
    s, d = g.directed()
    d2 = ctx.graph_from_edges(g.n, s, d).to_device()
    for qn in ("_4_road4", "_5_road5", "_4_square"):
        cases.append((ctx, ctx.pre_process_query(ctx.file_parse(os.path.join(GOLD, "queries", qn + ".g"))), d2))
    # vertex labels
    gv = synth.rmat(12, 30000, seed=4)
    gv.vlabel = synth.vlabels(gv.n, 4, 0.0, seed=5)
    sv, dv = gv.directed()
    d3 = vctx.graph_from_edges(gv.n, sv, dv, None, gv.vlabel).to_device()
    for i in range(6):
        qg, _ = synth.rw_query(gv, 4 + i % 3, tree=i % 2 == 0, seed=i)
        qs, qd = qg.directed()
        cases.append((vctx, vctx.pre_process_query(vctx.graph_from_edges(qg.n, qs, qd, None, qg.vlabel)), d3))

    first = [_noalloc(c, p, d) for c, p, d in cases]  # the first call on the device may load the module
    # the er200 cases are pinned by the golden counts (FFS restatement == enumerator)
    for (qn, f) in zip(("_3_triangle", "_4_square", "_5_road5", "_5_plus"), first):
        assert f == COUNTS[qn + "|er200"]["count"]
    for rep in range(2):
        for (c, p, d), f in zip(cases, first):
            want, _ = c.match_count(p, d)
            got = _noalloc(c, p, d)
            assert got == want == f, (rep, got, want, f)
    # the no-alloc calls themselves take no device memory (match_count's
    # engines were allocated by the loop above)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(0)[0]
    for c, p, d in cases:
        _noalloc(c, p, d)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free_before
    assert sum(first) > 0
    ctx.close()
    vctx.close()


def test_noalloc_requires_device_graph():
    ctx = gfsm_b200.GFSM(device=0)
    d = ctx.file_parse(os.path.join(GOLD, "data", "er200.g"))  # not built on the device yet
    p = ctx.pre_process_query(ctx.file_parse(os.path.join(GOLD, "queries", "_3_triangle.g")))
    cnt = C.c_uint64()
    assert ctx._lib.gfsm_match_count_noalloc(p.handle, d.handle, None, C.byref(cnt)) == 300
    ctx.close()


def test_noalloc_chunks_through_the_fixed_array(monkeypatch, capfd):
    """A frontier far larger than one level's buffer (the context's
    max_soln_size caps it at 2,048 partial mappings) must be cut into several
    steps per level, with re-runs where a chunk overflowed, and still give
    the golden count; GFSM_TRACE shows the steps."""
    ctx = gfsm_b200.GFSM(device=0, max_soln_size=2048)
    data = ctx.file_parse(os.path.join(GOLD, "data", "ba300.g")).to_device()
    plan = ctx.pre_process_query(ctx.file_parse(os.path.join(GOLD, "queries", "_5_road5.g")))
    monkeypatch.setenv("GFSM_TRACE", "1")
    capfd.readouterr()
    got = _noalloc(ctx, plan, data)
    err = capfd.readouterr().err
    monkeypatch.delenv("GFSM_TRACE")
    assert got == COUNTS["_5_road5|ba300"]["count"]
    steps = [dict(kv.split("=") for kv in line.split()[1:]) for line in err.splitlines()
             if line.startswith("gfsm-noalloc-step")]
    per_depth = {}
    for st in steps:
        per_depth[st["depth"]] = per_depth.get(st["depth"], 0) + 1
    assert max(per_depth.values()) > 1, per_depth          # a level ran as several chunks
    assert any(int(st["children"]) > 0 for st in steps)
    assert _noalloc(ctx, plan, data) == got                # and again, on the array the last call left
    ctx.close()


def test_noalloc_candidate_cap_matches_match_count():
    """The context's candidate cap stops both count paths with the same status."""
    ctx = gfsm_b200.GFSM(device=0, max_candidates=5000)
    data = ctx.file_parse(os.path.join(GOLD, "data", "ba300.g")).to_device()
    plan = ctx.pre_process_query(ctx.file_parse(os.path.join(GOLD, "queries", "_5_road5.g")))
    rc, _ = _noalloc_rc(ctx, plan, data)
    with pytest.raises(gfsm_b200.GFSMError) as e:
        ctx.match_count(plan, data)
    assert rc == e.value.status != 0
    ctx.close()
