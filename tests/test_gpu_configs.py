"""GPU parity on the workload configurations at their stated sizes.

Configuration 1 exactly as specified: Erdos-Renyi n=2,000, average degree 8,
seed 0, vertex labels uniform in {0..3}, edge labels 1, one 5-vertex
random-walk query with all induced edges.  The count is checked against
both the oracle's restatement of the reference FFS and the independent
backtracking enumerator, and the sorted full mappings against the
enumerator's, with vertex labels ignored (the reference's semantics) and
matched."""
import numpy as np
import pytest

from gfsm_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _sorted_rows(r):
    return r[np.lexsort(r.T[::-1])]


@pytest.mark.parametrize("vl", [False, True])
def test_config1_count_and_mappings(gpu_ctx, gpu_ctx_vl, tmp_path, vl):
    g, (q,) = synth.config1()
    ctx = gpu_ctx_vl if vl else gpu_ctx
    dpath, qpath = tmp_path / "d.g", tmp_path / "q.g"
    g.write_text(str(dpath))
    q.write_text(str(qpath))
    od, oq = O.Graph(path=str(dpath)), O.Graph(path=str(qpath))
    ffs = O.ffs_count(oq, O.Plan(oq), od, vlabel_mode=vl, threads=8)
    ds, dd = g.directed()
    qs, qd = q.directed()
    bt, rows_bt = O.bt_count(q.n, qs, qd, None, q.vlabel, g.n, ds, dd, None, g.vlabel, vlabel_mode=vl, threads=8,
                             max_rows=9_000_000)
    assert ffs == bt > 0
    assert len(rows_bt) == bt  # every mapping fits the buffer, so the sets compare whole
    data = ctx.graph_from_edges(g.n, ds, dd, None, g.vlabel)
    plan = ctx.pre_process_query(ctx.graph_from_edges(q.n, qs, qd, None, q.vlabel))
    got, _ = ctx.match_count(plan, data)
    assert got == ffs
    # the text path gives the same count
    tq = ctx.pre_process_query(ctx.file_parse(str(qpath)))
    assert ctx.match_count(tq, ctx.file_parse(str(dpath)))[0] == ffs
    rows, n = ctx.match_mappings(plan, data, max_rows=9_000_000)
    assert n == len(rows) == bt
    assert np.array_equal(_sorted_rows(rows), _sorted_rows(rows_bt))
