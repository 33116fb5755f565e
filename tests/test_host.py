"""CPU tests of the product's host side through the C ABI: the library loads
and exports every symbol include/gfsm.h declares; the multi-threaded parser
and the planner reproduce the reference's front-end (pinned fixtures); error
codes match the reference's exit codes.  No kernel runs here."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import gfsm_b200
from gfsm_b200 import _lib
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
REF = json.load(open(os.path.join(GOLD, "ref_frontend.json")))


def test_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "gfsm.h")).read()
    declared = set(re.findall(r"\b(gfsm_[a-z_]+)\s*\(", hdr))
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (gfsm_[a-z_]+)", out))
    assert declared, "no declarations found"
    assert declared <= exported, declared - exported
    assert declared == set(_lib.SIGNATURES), set(_lib.SIGNATURES) ^ declared
    _lib.load()


def test_cli_binary_links():
    r = subprocess.run(["ldd", os.path.join(ROOT, "gfsm_b200", "GFSM")], capture_output=True, text=True)
    assert "libgfsm.so" in r.stdout and "not found" not in r.stdout


def test_limits_defaults_are_environment_h(monkeypatch):
    for k in ("GFSM_MEMLIMIT", "GFSM_MAXSOLNSIZE", "GFSM_MAXSCANSIZE", "GFSM_CCSRRELSIZE", "GFSM_UPPERMEMLIMIT"):
        monkeypatch.delenv(k, raising=False)
    lim = gfsm_b200.default_limits()
    assert lim.ccsr_rel_size == 8
    assert lim.max_soln_size == 500_000_000 and lim.max_scan_size == 500_000_000
    assert lim.mem_limit == 22_000_000_000 and lim.upper_mem_limit == 44_000_000_000
    assert lim.vertex_labels == 0
    monkeypatch.setenv("GFSM_MEMLIMIT", "1e9")
    assert gfsm_b200.default_limits().mem_limit == 1_000_000_000


@pytest.mark.parametrize("key", sorted(k for k in REF if k.startswith("queries/")))
def test_planner_matches_reference(host_ctx, key):
    r = REF[key]
    q = host_ctx.file_parse(os.path.join(GOLD, key + ".g"))
    t = host_ctx.pre_process_query(q).tables()
    assert t["max_valency"] == r["max_valency"]
    assert t["reqs"].tolist() == r["reqs"]
    assert t["header"].tolist() == r["header"]


def test_planner_matches_oracle_on_random_walks(host_ctx, tmp_path):
    from gfsm_b200 import synth
    g = synth.ba(2000, 3, seed=5)
    for i in range(40):
        k = 3 + i % 10
        qg, _ = synth.rw_query(g, k, tree=i % 3 == 0, seed=i)
        p = tmp_path / f"q{i}.g"
        qg.write_text(str(p))
        mine = host_ctx.pre_process_query(host_ctx.file_parse(str(p))).tables()
        ref = O.Plan(O.Graph(path=str(p))).tables()
        assert mine["reqs"].tolist() == ref["reqs"].tolist()
        assert mine["header"].tolist() == ref["header"].tolist()
        assert mine["order"].tolist() == ref["order"].tolist()


def test_planner_matches_oracle_on_irregular_queries(host_ctx, tmp_path):
    """Queries beyond random walks -- repeated edges, self-loops, one-way
    edges, three edge labels, 1-16 vertices: the planner's tables, or its
    rejection of the query, equal the oracle's restatement of the
    reference planner (HnGPU.cu:749-816, ccsr.cpp:98-219).  A row holding
    one target twice with two labels makes the requirement's relation
    depend on the order the reference's std::sort leaves them in; rows of
    at most 16 entries (kept here) are insertion-sorted by libstdc++, which
    keeps input order, and the oracle restates that."""
    rng = np.random.default_rng(11)
    agree_ok = agree_err = 0
    for i in range(300):
        k = int(rng.integers(1, 17))
        edges = []
        for v in range(1, k):
            u, l = int(rng.integers(v)), int(rng.integers(1, 4))
            edges.append((u, v, l))
            if rng.random() < 0.8:
                edges.append((v, u, l if rng.random() < 0.9 else int(rng.integers(1, 4))))
        for _ in range(int(rng.integers(0, 2 * k + 1))):
            a, b, l = int(rng.integers(k)), int(rng.integers(k)), int(rng.integers(1, 4))
            edges.append((a, b, l))
            if rng.random() < 0.7:
                edges.append((b, a, l))
        if edges and rng.random() < 0.1:
            edges += [edges[int(j)] for j in rng.integers(len(edges), size=3)]
        rng.shuffle(edges)
        if np.bincount(np.array([a for a, _, _ in edges], np.int64), minlength=k).max() > 16:
            continue
        lines = ["t # 0", f"{k} {len(edges)} 1 1"] + [f"v {v} 1" for v in range(k)]
        lines += [f"e {a} {b} {l}" for a, b, l in edges] + ["t # -1"]
        path = tmp_path / f"q{i}.g"
        path.write_text("\n".join(lines) + "\n")
        ref = O.Plan(O.Graph(path=str(path)))
        try:
            mine = host_ctx.pre_process_query(host_ctx.file_parse(str(path))).tables()
        except gfsm_b200.GFSMError:
            mine = None
        if ref.err:
            assert mine is None, (i, k, edges)
            agree_err += 1
            continue
        assert mine is not None, (i, k, edges)
        t = ref.tables()
        for key in ("max_valency",):
            assert mine[key] == t[key], (i, key)
        for key in ("reqs", "header", "order"):
            assert mine[key].tolist() == t[key].tolist(), (i, key, edges)
        agree_ok += 1
    assert agree_ok > 100 and agree_err > 10


def test_parser_error_codes(host_ctx, tmp_path):
    cases = {
        "t # 1\n1 0 1 1\nt # -1": 233,
        "t # 0\n3 2 1 1\nv 0 1\nt # -1": 234,
        "t # 0\n2 4 1 1\nv 0 1\nv 1 1\ne 0 1 1\ne 1 0 1\nt # -1": 234,
        "t # 0\n2 2 1 1\nv 0 1\nx 1 1\nt # -1": 233,
        "t # 0\n2 2 1 1\nv 0 1\ne 0 1 1\nv 1 1\nt # -1": 233,
        "t # 0\n2 2 1 1\nv 0 1\ne 0 5 1\ne 1 0 1\nt # -1": 233,
    }
    for text, code in cases.items():
        with pytest.raises(gfsm_b200.GFSMError) as ei:
            host_ctx.parse_text(text)
        assert ei.value.status == code, text
        p = tmp_path / "x.g"
        p.write_text(text)
        assert O.Graph(path=str(p)).err == code or code == 233
    with pytest.raises(gfsm_b200.GFSMError) as ei:
        host_ctx.file_parse(str(tmp_path / "nope.g"))
    assert ei.value.status == 232


def test_file_parse_from_a_pipe_and_an_empty_file(host_ctx, tmp_path):
    """A regular file is mapped while it is parsed; what cannot be mapped (a
    named pipe) is read whole instead -- the same graph either way.  An empty
    file is invalid data, as for the reference (no "t # 0" line)."""
    import threading
    text = open(os.path.join(GOLD, "data", "er200.g"), "rb").read()
    want = host_ctx.file_parse(os.path.join(GOLD, "data", "er200.g")).info()
    fifo = tmp_path / "pipe.g"
    os.mkfifo(fifo)

    def write():
        with open(fifo, "wb") as f:
            f.write(text)
    writer = threading.Thread(target=write)
    writer.start()
    got = host_ctx.file_parse(str(fifo)).info()
    writer.join()
    assert got == want and got["m"] > 0
    (tmp_path / "empty.g").write_bytes(b"")
    with pytest.raises(gfsm_b200.GFSMError) as ei:
        host_ctx.file_parse(str(tmp_path / "empty.g"))
    assert ei.value.status == 233


def test_parser_large_multichunk_matches_oracle(host_ctx, tmp_path):
    """A file big enough to be split across threads parses to the same edges."""
    from gfsm_b200 import synth
    g = synth.rmat(15, 120_000, seed=3)
    p = tmp_path / "big.g"
    g.write_text(str(p))
    assert os.path.getsize(p) > 3 << 20
    dg = host_ctx.file_parse(str(p))
    info = dg.info()
    og = O.Graph(path=str(p))
    assert info["n"] == og.arrays()["count"] and info["m"] == 2 * g.m
    assert info["rows"] == og.arrays()["rows"]


def test_disconnected_query_is_status_1(host_ctx):
    q = host_ctx.parse_text("t # 0\n4 4 1 1\nv 0 1\nv 1 1\nv 2 1\nv 3 1\ne 0 1 1\ne 1 0 1\ne 2 3 1\ne 3 2 1\nt # -1")
    with pytest.raises(gfsm_b200.GFSMError) as ei:
        host_ctx.pre_process_query(q)
    assert ei.value.status == 1


def test_matching_needs_a_device(host_ctx):
    q = host_ctx.file_parse(os.path.join(GOLD, "queries", "_3_triangle.g"))
    d = host_ctx.file_parse(os.path.join(GOLD, "data", "er200.g"))
    with pytest.raises(gfsm_b200.GFSMError) as ei:
        host_ctx.solve(q, d)
    assert ei.value.status == 305


def test_batch_planning_matches_one_at_a_time(host_ctx):
    """gfsm_query_prepare_batch gives every query the plan gfsm_query_prepare
    gives it (random walks of 3-12 vertices, with and without labels)."""
    from gfsm_b200 import synth
    g = synth.ba(2000, 3, seed=7)
    g.vlabel = synth.vlabels(g.n, 4, 0.0, seed=3)
    qs = []
    for i in range(300):
        qg, _ = synth.rw_query(g, 3 + i % 10, tree=i % 3 == 0, seed=100 + i)
        a, b = qg.directed()
        qs.append((qg.n, a, b, None, qg.vlabel))
    for use_labels in (True, False):
        batch = host_ctx.prepare_queries(q if use_labels else q[:4] + (None,) for q in qs)
        assert len(batch) == len(qs)
        for q, p in zip(qs, batch):
            one = host_ctx.pre_process_query(host_ctx.graph_from_edges(q[0], q[1], q[2], None,
                                                                       q[4] if use_labels else None))
            t, r = p.tables(), one.tables()
            for key in ("order", "header", "reqs"):
                assert t[key].tolist() == r[key].tolist()
            assert p.columns().tolist() == one.columns().tolist()


def test_batch_planning_reports_the_failing_query(host_ctx):
    """A disconnected query fails the whole batch with its own status (1) and
    index; an edge endpoint out of range is invalid data."""
    import ctypes as C
    tri = (3, [0, 1, 1, 2, 2, 0], [1, 0, 2, 1, 0, 2], None, None)
    split = (4, [0, 1, 2, 3], [1, 0, 3, 2], None, None)
    with pytest.raises(gfsm_b200.GFSMError) as ei:
        host_ctx.prepare_queries([tri, tri, split, tri])
    assert ei.value.status == 1
    lib = host_ctx._lib
    nv = np.array([3, 4], np.uint32)
    eoff = np.array([0, 6, 10], np.uint64)
    src = np.array(tri[1] + split[1], np.uint32)
    dst = np.array(tri[2] + split[2], np.uint32)
    out = (C.c_void_p * 2)()
    failed = C.c_int(7)
    rc = lib.gfsm_query_prepare_batch(host_ctx._h, 2, nv.ctypes.data_as(_lib.u32p), eoff.ctypes.data_as(_lib.u64p),
                                      src.ctypes.data_as(_lib.u32p), dst.ctypes.data_as(_lib.u32p), None, None,
                                      None, out, C.byref(failed))
    assert rc == 1 and failed.value == 1 and out[0] is None and out[1] is None
    bad = (3, [0, 1, 5], [1, 0, 0], None, None)
    with pytest.raises(gfsm_b200.GFSMError) as ei:
        host_ctx.prepare_queries([tri, bad])
    assert ei.value.status == 233  # GFSM_ERR_INVALID_DATA
    assert len(host_ctx.prepare_queries([])) == 0


@pytest.mark.parametrize("nq", [50, 3000])
def test_flat_batch_planning_and_plan_batch(host_ctx, nq):
    """prepare_queries_flat over flat arrays gives the per-query plans; a
    PlanBatch indexes as Plan views and closes every plan once.  3,000
    queries plan and free on several host threads."""
    from gfsm_b200 import synth
    g = synth.grid(30, 0.05, 0.02, seed=2)
    g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=4)
    qs = [synth.rw_query(g, 3 + i % 6, seed=300 + i)[0] for i in range(nq)]
    dirs = [q.directed() for q in qs]
    nv = np.array([q.n for q in qs], np.uint32)
    eoff = np.zeros(len(qs) + 1, np.uint64)
    np.cumsum([len(a) for a, _ in dirs], out=eoff[1:])
    src = np.concatenate([a for a, _ in dirs])
    dst = np.concatenate([b for _, b in dirs])
    vl = np.concatenate([q.vlabel for q in qs])
    batch = host_ctx.prepare_queries_flat(nv, eoff, src, dst, None, vl)
    assert len(batch) == len(qs)
    for q, (a, b), p in zip(qs, dirs, batch):
        one = host_ctx.pre_process_query(host_ctx.graph_from_edges(q.n, a, b, None, q.vlabel))
        assert p.tables()["order"].tolist() == one.tables()["order"].tolist()
        assert p.tables()["reqs"].tolist() == one.tables()["reqs"].tolist()
        assert p.symmetry() == one.symmetry()
        p.close()  # a view: does not destroy the batch's plan
    assert batch[-1].tables()["k"] == qs[-1].n
    batch.close()
    assert len(batch) == 0


def test_symmetry_group_orders_and_limits(host_ctx):
    """|Aut(Q)| of known shapes (found without listing the group: K_16 has
    16! elements), restricted by self-loops and edge labels; a directed query
    (count depends on the order) gets none."""
    import math
    import time

    def plan(n, edges, labels=None):
        s = np.array([a for a, b in edges] + [b for a, b in edges if a != b], np.uint32)
        d = np.array([b for a, b in edges] + [a for a, b in edges if a != b], np.uint32)
        el = None if labels is None else np.array(list(labels) + [l for (a, b), l in zip(edges, labels) if a != b],
                                                   np.uint32)
        return host_ctx.pre_process_query(host_ctx.graph_from_edges(n, s, d, el, None))

    t = time.perf_counter()
    for n in (5, 8, 12, 16):
        aut, cond = plan(n, [(a, b) for a in range(n) for b in range(a + 1, n)]).symmetry()
        assert aut == math.factorial(n) and len(cond) == n * (n - 1) // 2
    assert time.perf_counter() - t < 5.0
    assert plan(6, [(i, (i + 1) % 6) for i in range(6)]).symmetry()[0] == 12       # C6: dihedral
    assert plan(5, [(0, i) for i in range(1, 5)]).symmetry()[0] == 24              # K_{1,4}
    assert plan(4, [(0, 1), (1, 2), (2, 3)]).symmetry()[0] == 2                    # path
    # a self-loop on one end of a path breaks its reversal
    assert plan(4, [(0, 1), (1, 2), (2, 3), (0, 0)]).symmetry()[0] == 1
    # edge labels: a triangle with one edge of another label keeps one swap
    assert plan(3, [(0, 1), (1, 2), (2, 0)], [1, 1, 2]).symmetry()[0] == 2
    # an edge without its reverse: not order-invariant, no symmetry breaking
    s = np.array([0, 1, 2, 1], np.uint32)
    d = np.array([1, 2, 0, 0], np.uint32)
    p = host_ctx.pre_process_query(host_ctx.graph_from_edges(3, s, d))
    assert p.info()["order_invariant"] is False and p.symmetry() == (1, [])


def test_partition_rows_edges():
    """gfsm_partition_rows: monotone bounds covering the window, parts of
    near-equal CCSR entries, empty windows, more parts than rows, rows
    without entries."""
    import numpy as np
    import gfsm_b200
    deg = np.array([9, 7, 7, 5, 3, 3, 2, 1, 1, 1, 0, 0], np.uint32)
    rowptr = np.zeros(len(deg) + 1, np.uint32)
    np.cumsum(deg, out=rowptr[1:])
    for lo, hi in ((0, 12), (2, 9), (5, 5), (10, 12)):
        for nparts in (1, 2, 3, 5, 16):
            b = gfsm_b200.partition_rows(rowptr, lo, hi, nparts).astype(np.int64)
            assert b[0] == 0 and b[-1] == hi - lo and len(b) == nparts + 1
            assert np.all(np.diff(b) >= 0)
            w = int(rowptr[hi]) - int(rowptr[lo])
            if w:
                parts = [int(rowptr[lo + b[k + 1]]) - int(rowptr[lo + b[k]]) for k in range(nparts)]
                assert sum(parts) == w
                # each part ends at the first row reaching its share
                for k in range(1, nparts):
                    target = -(-k * w // nparts)
                    reach = int(rowptr[lo + b[k]]) - int(rowptr[lo])
                    assert reach >= target
                    assert b[k] == b[k - 1] or int(rowptr[lo + b[k] - 1]) - int(rowptr[lo]) < target
    with pytest.raises(gfsm_b200.GFSMError):
        gfsm_b200.partition_rows(rowptr, 5, 2, 2)
