"""GPU parity: the sm_100a kernels through the C ABI against the oracle.

Bit-exact integer counts (and, for small cases, identical sorted mapping
sets) on: the golden fixtures; seeded random graphs and random-walk queries
(trees and cyclic, edge labels, vertex labels); edge cases (no match, absent
labels, query larger than data, duplicate entries, self-loops); forced
chunking with tiny MEMLIMIT / MAXSCANSIZE / MAXSOLNSIZE; batched == one at a
time; and size-independent closed forms at the full R-MAT 2^20 size."""
import json
import os

import numpy as np
import pytest

import gfsm_b200
from gfsm_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
COUNTS = json.load(open(os.path.join(GOLD, "counts.json")))


def _g(key):
    return os.path.join(GOLD, key + ".g")


@pytest.mark.parametrize("key", sorted(COUNTS))
def test_golden_counts(gpu_ctx, gpu_ctx_vl, key):
    qn, dn = key.split("|")
    for ctx, field in ((gpu_ctx, "count"), (gpu_ctx_vl, "count_vlabels")):
        q = ctx.file_parse(_g("queries/" + qn))
        d = ctx.file_parse(_g("data/" + dn))
        assert ctx.solve(q, d) == COUNTS[key][field]


def _labelled_query(g, lab, qg, visited):
    if lab is None:
        return None
    key = {(int(a), int(b)): int(l) for a, b, l in zip(g.src, g.dst, lab)}
    return np.array([key[(min(visited[a], visited[b]), max(visited[a], visited[b]))]
                     for a, b in zip(qg.src, qg.dst)], np.uint32)


def _both_dirs(ug, lab=None):
    s, d = ug.directed()
    l = None if lab is None else np.concatenate([lab, lab])
    return s, d, l


# Sizes chosen so that the CPU oracle finishes every case in well under a
# second: unlabelled queries up to 5 vertices, vertex-labelled up to 7.
GENS = [
    ("er", lambda s: synth.er(300, 5.0, seed=s)),
    ("ba", lambda s: synth.ba(300, 2, seed=s)),
    ("rmat", lambda s: synth.rmat(9, 1200, seed=s)),
    ("grid", lambda s: synth.grid(16, 0.05, 0.03, seed=s)),
]


@pytest.mark.parametrize("gen", range(len(GENS)))
@pytest.mark.parametrize("labelled", [False, True])
def test_random_walk_queries(gpu_ctx, gpu_ctx_vl, tmp_path, gen, labelled):
    name, fn = GENS[gen]
    g = fn(gen + 1)
    g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=gen + 40)
    lab = ((np.arange(g.m, dtype=np.uint64) * 2654435761 + gen) % 3 + 1).astype(np.uint32) if labelled else None
    dpath = tmp_path / "d.g"
    g.write_text(str(dpath), lab)
    od = O.Graph(path=str(dpath))
    ds, dd, dl = _both_dirs(g, lab)
    dev = {c: c.graph_from_edges(g.n, ds, dd, dl, g.vlabel) for c in (gpu_ctx, gpu_ctx_vl)}
    text_graph = gpu_ctx.file_parse(str(dpath))
    for i, k in enumerate((3, 4, 5, 6, 7)):
        for tree in (False, True):
            qg, visited = synth.rw_query(g, k, tree=tree, seed=1000 * gen + 10 * i + tree)
            ql = _labelled_query(g, lab, qg, visited)
            qpath = tmp_path / "q.g"
            qg.write_text(str(qpath), ql)
            oq = O.Graph(path=str(qpath))
            op = O.Plan(oq)
            cases = [(gpu_ctx_vl, O.ffs_count(oq, op, od, vlabel_mode=True, threads=8))]
            if k <= 5:
                cases.append((gpu_ctx, O.ffs_count(oq, op, od, threads=8)))
            for ctx, expect in cases:
                plan = ctx.pre_process_query(ctx.file_parse(str(qpath)))
                got, st = ctx.match_count(plan, dev[ctx])
                assert got == expect, (name, k, tree, ctx is gpu_ctx_vl, got, expect)
            if k <= 5:
                # the text-parsed data graph gives the same count
                plan = gpu_ctx.pre_process_query(gpu_ctx.file_parse(str(qpath)))
                assert gpu_ctx.match_count(plan, text_graph)[0] == cases[-1][1]


def test_mappings_match_backtracking(gpu_ctx, tmp_path):
    g = synth.er(120, 5.0, seed=9)
    ds, dd, _ = _both_dirs(g)
    data = gpu_ctx.graph_from_edges(g.n, ds, dd)
    for qn in ("_3_triangle", "_4_square", "_5_plus", "_5_road5"):
        oq = O.Graph(path=_g("queries/" + qn))
        qs, qd, ql = oq.edges()
        k = oq.arrays()["count"]
        c2, r2 = O.bt_count(k, qs, qd, ql, None, g.n, ds, dd, None, None, threads=8, max_rows=2_000_000)
        plan = gpu_ctx.pre_process_query(gpu_ctx.file_parse(_g("queries/" + qn)))
        rows, c1 = gpu_ctx.match_mappings(plan, data, max_rows=2_000_000)
        assert c1 == c2 == len(rows) == len(r2)
        s1 = rows[np.lexsort(rows.T[::-1])]
        s2 = r2[np.lexsort(r2.T[::-1])]
        assert np.array_equal(s1, s2)


def test_edge_cases(gpu_ctx, gpu_ctx_vl, tmp_path):
    tri = gpu_ctx.file_parse(_g("queries/_3_triangle"))
    # a tree has no triangle
    path = synth.UGraph(6, np.arange(5, dtype=np.uint32), np.arange(1, 6, dtype=np.uint32))
    s, d, _ = _both_dirs(path)
    assert gpu_ctx.solve(tri, gpu_ctx.graph_from_edges(6, s, d)) == 0
    # query larger than the data graph
    big = gpu_ctx.file_parse(_g("queries/_5_plus"))
    k3 = synth.UGraph(3, np.array([0, 0, 1], np.uint32), np.array([1, 2, 2], np.uint32))
    s, d, _ = _both_dirs(k3)
    assert gpu_ctx.solve(big, gpu_ctx.graph_from_edges(3, s, d)) == 0
    # isolated vertices in the data graph
    s, d, _ = _both_dirs(k3)
    assert gpu_ctx.solve(tri, gpu_ctx.graph_from_edges(50, s, d)) == 6
    # an edge label the data does not have
    q = gpu_ctx.parse_text("t # 0\n3 6 1 1\nv 0 1\nv 1 1\nv 2 1\ne 0 1 2\ne 1 0 2\ne 1 2 2\ne 2 1 2\ne 2 0 2\ne 0 2 2\nt # -1")
    assert gpu_ctx.solve(q, gpu_ctx.graph_from_edges(3, s, d)) == 0
    # a vertex label the data does not have (vertex-label mode)
    qv = gpu_ctx_vl.parse_text("t # 0\n3 6 1 1\nv 0 9\nv 1 9\nv 2 9\ne 0 1 1\ne 1 0 1\ne 1 2 1\ne 2 1 1\ne 2 0 1\ne 0 2 1\nt # -1")
    assert gpu_ctx_vl.solve(qv, gpu_ctx_vl.graph_from_edges(3, s, d)) == 0


def test_duplicate_entries_and_self_loops(gpu_ctx, tmp_path):
    """Duplicate data entries yield duplicate embeddings and data self-loops
    are rejected by injectivity -- the reference's semantics (HnGPU.cu:168-175,
    223-236), checked against the oracle's restatement."""
    rng = np.random.default_rng(5)
    g = synth.er(80, 6.0, seed=21)
    s, d = g.directed()
    extra = rng.integers(0, len(s), 40)
    loops = rng.integers(0, g.n, 10).astype(np.uint32)
    s = np.concatenate([s, s[extra], loops]).astype(np.uint32)
    d = np.concatenate([d, d[extra], loops]).astype(np.uint32)
    lines = ["t # 0", f"{g.n} {len(s)} 1 1"] + [f"v {i} 1" for i in range(g.n)]
    lines += [f"e {a} {b} 1" for a, b in zip(s, d)]
    p = tmp_path / "dup.g"
    p.write_text("\n".join(lines) + "\nt # -1")
    od = O.Graph(path=str(p))
    dev = gpu_ctx.file_parse(str(p))
    assert dev.to_device().info()["multi_edges"] == 1
    for qn in ("_3_triangle", "_4_square", "_4_roadY"):
        oq = O.Graph(path=_g("queries/" + qn))
        want = O.ffs_count(oq, O.Plan(oq), od, threads=8)
        assert gpu_ctx.solve(gpu_ctx.file_parse(_g("queries/" + qn)), dev) == want


def test_device_ccsr_matches_reference_layout(gpu_ctx):
    """The device builder reproduces the reference CCSR (row order, rows sorted
    by target, staggers) recorded from the reference's own fileParse."""
    ref = json.load(open(os.path.join(GOLD, "ref_frontend.json")))
    for name in ("data/er200", "data/ba300", "data/grid15", "data/er150_lab3"):
        r = ref[name]
        g = gpu_ctx.file_parse(_g(name))
        rowptr, adj, elab, order = g.download()
        # rebuild the packed reference segments from the device arrays
        rows = int(np.count_nonzero(np.diff(rowptr.astype(np.int64))))
        deg = np.diff(rowptr.astype(np.int64))
        rowoff = np.concatenate([[0], np.cumsum(deg[:rows] + 1)])[:rows]
        seg = []
        for i in range(rows):
            seg.append(int(deg[i]))
            for j in range(rowptr[i], rowptr[i + 1]):
                seg.append(int(rowoff[adj[j]]) | (int(elab[j]) << 24))
        assert seg == r["segments"]
        assert order.tolist() == r["inv"]


@pytest.mark.parametrize("limits", [
    dict(mem_limit=64 << 20),
    dict(max_scan_size=4096),
    dict(max_soln_size=2048, max_scan_size=8192),
])
def test_forced_chunking(tmp_path, limits):
    """MEMLIMIT-bounded chunking: tiny limits force many steps and retries
    and must not change any count."""
    ctx = gfsm_b200.GFSM(device=0, **limits)
    g = synth.ba(3000, 4, seed=2)
    s, d, _ = _both_dirs(g)
    data = ctx.graph_from_edges(g.n, s, d)
    dpath = tmp_path / "d.g"
    g.write_text(str(dpath))
    od = O.Graph(path=str(dpath))
    deg = np.bincount(np.concatenate([g.src, g.dst]), minlength=g.n).astype(object)
    steps = []
    for qn in ("_3_triangle", "_4_square", "_4_road4", "_5_road5", "_5_plus"):
        if qn == "_5_plus":  # a 4-leaf star: closed form of the degree sequence
            want = int(sum(x * (x - 1) * (x - 2) * (x - 3) for x in deg))
        else:
            oq = O.Graph(path=_g("queries/" + qn))
            want = O.ffs_count(oq, O.Plan(oq), od, threads=8)
        plan = ctx.pre_process_query(ctx.file_parse(_g("queries/" + qn)))
        got, st = ctx.match_count(plan, data)
        assert got == want
        steps.append(st["steps"])
    # the 5-vertex queries cannot fit one step per level under these limits
    assert max(steps) > 10, steps
    ctx.close()


def test_batch_equals_one_at_a_time(gpu_ctx_vl):
    g = synth.rmat(12, 30000, seed=4)
    g.vlabel = synth.vlabels(g.n, 4, 0.0, seed=5)
    s, d, _ = _both_dirs(g)
    data = gpu_ctx_vl.graph_from_edges(g.n, s, d, None, g.vlabel)
    plans = []
    for i in range(64):
        qg, _ = synth.rw_query(g, 3 + i % 4, tree=i % 2 == 0, seed=i)
        qs, qd = qg.directed()
        q = gpu_ctx_vl.graph_from_edges(qg.n, qs, qd, None, qg.vlabel)
        plans.append(gpu_ctx_vl.pre_process_query(q))
    batch, st = gpu_ctx_vl.batch_count(plans, data)
    single = [gpu_ctx_vl.match_count(p, data)[0] for p in plans]
    assert batch.tolist() == single
    assert sum(single) > 0


def test_full_size_rmat(gpu_ctx):
    """Size-independent properties at the R-MAT 2^20 (~16M edges) size: the
    counts of an edge and of a 3-path are closed forms of the degree sequence,
    and the triangle count is 6x the triangles found by an independent
    orientation-and-intersection counter."""
    g = synth.rmat(20, 16 << 20, seed=0)
    s, d, _ = _both_dirs(g)
    data = gpu_ctx.graph_from_edges(g.n, s, d)
    deg = np.bincount(np.concatenate([g.src, g.dst]), minlength=g.n).astype(object)
    q2 = gpu_ctx.file_parse(_g("queries/_2_road2"))
    assert gpu_ctx.solve(q2, data) == 2 * g.m
    q3 = gpu_ctx.file_parse(_g("queries/_3_road3"))
    assert gpu_ctx.solve(q3, data) == int(sum(x * (x - 1) for x in deg))
    tri = gpu_ctx.file_parse(_g("queries/_3_triangle"))
    assert gpu_ctx.solve(tri, data) == 6 * O.triangles(g.n, g.src, g.dst)


def test_triangles_medium_rmat(gpu_ctx):
    g = synth.rmat(14, 200_000, seed=1)
    s, d, _ = _both_dirs(g)
    data = gpu_ctx.graph_from_edges(g.n, s, d)
    tri = gpu_ctx.file_parse(_g("queries/_3_triangle"))
    assert gpu_ctx.solve(tri, data) == 6 * O.triangles(g.n, g.src, g.dst)


@pytest.mark.parametrize("tile", ["0", "2"])
def test_device_and_host_drivers_agree(monkeypatch, tile):
    """The graph-driven schedule (one CUDA graph launch, decisions on the
    device) and the host-driven step loop do the same work: identical counts,
    candidates and expansions, for both tile geometries the graph is
    instantiated for."""
    monkeypatch.setenv("GFSM_TILE", tile)
    ctx = gfsm_b200.GFSM(device=0, vertex_labels=1, mem_limit=256 << 20)
    g = synth.grid(300, 0.05, 0.02, seed=8)
    g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=9)
    s, d = g.directed()
    data = ctx.graph_from_edges(g.n, s, d, None, g.vlabel)
    plans = []
    for i in range(40):
        qg, _ = synth.rw_query(g, 3 + i % 8, tree=i % 2 == 0, seed=50 + i)
        qs, qd = qg.directed()
        plans.append(ctx.pre_process_query(ctx.graph_from_edges(qg.n, qs, qd, None, qg.vlabel)))
    monkeypatch.setenv("GFSM_DRIVER", "host")
    host_counts, host_st = ctx.batch_count(plans, data)
    host_single = [ctx.match_count(p, data) for p in plans[:8]]
    monkeypatch.setenv("GFSM_DRIVER", "graph")
    dev_counts, dev_st = ctx.batch_count(plans, data)
    dev_single = [ctx.match_count(p, data) for p in plans[:8]]
    assert dev_counts.tolist() == host_counts.tolist()
    # the work is the same; the chunking is not: children land in tile
    # completion order, so the survivor ratios each driver observes -- and
    # with them the number of steps and re-runs under this tight MEMLIMIT --
    # may differ between runs
    for key in ("candidates", "expansions"):
        assert dev_st[key] == host_st[key], key
    # kernels launched: partition + step per step (+ count commits) on the
    # host loop; the graph's first controller, then partition, root step,
    # level step and controller nodes per step
    assert 2 * host_st["steps"] <= host_st["launches"] <= 3 * host_st["steps"]
    assert dev_st["launches"] == 1 + 4 * dev_st["steps"]
    assert (host_st["driver"], dev_st["driver"]) == (0, 1)
    assert dev_st["tile_variant"] == int(tile) and dev_st["graph_error"] == 0
    for (c1, s1), (c2, s2) in zip(host_single, dev_single):
        assert c1 == c2 and s1["candidates"] == s2["candidates"]
    assert host_st["steps"] > 20
    ctx.close()


@pytest.mark.parametrize("driver", ["host", "graph"])
def test_repeated_call_takes_larger_first_steps(monkeypatch, driver):
    """A depth's first step is capped until its next-level rate is known; a
    repeated call of the same workload class starts from the rates its
    predecessor saw, so it needs no more steps, and counts, candidates and
    expansions do not change."""
    monkeypatch.setenv("GFSM_DRIVER", driver)
    monkeypatch.setenv("GFSM_TILE", "0")
    ctx = gfsm_b200.GFSM(device=0, vertex_labels=1)
    g = synth.grid(700, 0.05, 0.02, seed=8)
    g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=9)
    s, d = g.directed()
    data = ctx.graph_from_edges(g.n, s, d, None, g.vlabel)
    plans = []
    for i in range(64):
        qg, _ = synth.rw_query(g, 4 + i % 4, tree=i % 2 == 0, seed=700 + i)
        qs, qd = qg.directed()
        plans.append(ctx.pre_process_query(ctx.graph_from_edges(qg.n, qs, qd, None, qg.vlabel)))
    c1, s1 = ctx.batch_count(plans, data)
    c2, s2 = ctx.batch_count(plans, data)
    assert c1.tolist() == c2.tolist() and c1.sum() > 0
    for key in ("candidates", "expansions"):
        assert s1[key] == s2[key], key
    assert s2["steps"] <= s1["steps"] and s2["retries"] == 0
    ctx.close()


def test_default_driver_policy(monkeypatch):
    """Without GFSM_DRIVER a call whose first level (the CCSR entries of its
    queries' root windows) holds at most 2^22 candidates runs on the graph,
    a heavier one on the host loop; both count what the other driver counts."""
    monkeypatch.delenv("GFSM_DRIVER", raising=False)
    monkeypatch.setenv("GFSM_TILE", "0")
    ctx = gfsm_b200.GFSM(device=0, vertex_labels=1)
    g = synth.grid(300, 0.05, 0.02, seed=8)
    g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=9)
    s, d = g.directed()
    data = ctx.graph_from_edges(g.n, s, d, None, g.vlabel).to_device()
    rowptr = data.download()[0]
    plans = []
    for i in range(96):
        qg, _ = synth.rw_query(g, 3 + i % 6, tree=i % 2 == 0, seed=300 + i)
        qs, qd = qg.directed()
        plans.append(ctx.pre_process_query(ctx.graph_from_edges(qg.n, qs, qd, None, qg.vlabel)))

    def first_level(ps):
        tot = 0
        for p in ps:
            lo, bounds = ctx.root_partition(p, data, 1)
            tot += int(rowptr[lo + int(bounds[-1])]) - int(rowptr[lo])
        return tot

    light, heavy = plans[:1], plans
    assert first_level(light) <= 1 << 22 < first_level(heavy)
    for ps, want in ((light, 1), (heavy, 0)):
        c, st = ctx.batch_count(ps, data)
        assert st["driver"] == want
        monkeypatch.setenv("GFSM_DRIVER", "host" if want else "graph")
        c2, st2 = ctx.batch_count(ps, data)
        monkeypatch.delenv("GFSM_DRIVER")
        assert st2["driver"] == 1 - want and c2.tolist() == c.tolist()
    ctx.close()


@pytest.mark.parametrize("variant", ["0", "1", "2", "3"])
def test_tile_geometries_agree(monkeypatch, variant):
    """Every tile geometry the autotuner can pick gives the same counts,
    candidates and expansions (hub rows, vertex labels and chunking)."""
    monkeypatch.setenv("GFSM_TILE", variant)
    ctx = gfsm_b200.GFSM(device=0, vertex_labels=1, mem_limit=512 << 20)
    g = synth.rmat(12, 25000, seed=6)
    g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=7)
    s, d = g.directed()
    data = ctx.graph_from_edges(g.n, s, d, None, g.vlabel)
    dpath_plans = []
    for i in range(24):
        qg, _ = synth.rw_query(g, 3 + i % 4, tree=i % 2 == 0, seed=300 + i)
        qs, qd = qg.directed()
        dpath_plans.append(ctx.pre_process_query(ctx.graph_from_edges(qg.n, qs, qd, None, qg.vlabel)))
    counts, st = ctx.batch_count(dpath_plans, data)
    assert st["tile_variant"] == int(variant)
    ref = gfsm_b200.GFSM(device=0, vertex_labels=1)
    monkeypatch.setenv("GFSM_TILE", "0")
    rdata = ref.graph_from_edges(g.n, s, d, None, g.vlabel)
    rplans = []
    for i in range(24):
        qg, _ = synth.rw_query(g, 3 + i % 4, tree=i % 2 == 0, seed=300 + i)
        qs, qd = qg.directed()
        rplans.append(ref.pre_process_query(ref.graph_from_edges(qg.n, qs, qd, None, qg.vlabel)))
    rcounts, rst = ref.batch_count(rplans, rdata)
    assert counts.tolist() == rcounts.tolist() and counts.sum() > 0
    tri = ctx.pre_process_query(ctx.file_parse(_g("queries/_3_triangle")))
    udata = gfsm_b200.GFSM(device=0)
    monkeypatch.setenv("GFSM_TILE", variant)
    ud = udata.graph_from_edges(g.n, s, d)
    assert udata.solve(udata.file_parse(_g("queries/_3_triangle")), ud) == 6 * O.triangles(g.n, g.src, g.dst)
    ctx.close()
    ref.close()
    udata.close()


def test_autotuner_choice_is_exact(monkeypatch):
    monkeypatch.delenv("GFSM_TILE", raising=False)
    ctx = gfsm_b200.GFSM(device=0)
    g = synth.ba(5000, 4, seed=12)
    s, d = g.directed()
    data = ctx.graph_from_edges(g.n, s, d)
    tri = ctx.pre_process_query(ctx.file_parse(_g("queries/_3_triangle")))
    c, st = ctx.match_count(tri, data)
    assert 0 <= st["tile_variant"] < 4
    assert c == 6 * O.triangles(g.n, g.src, g.dst)
    ctx.close()


def test_mixed_batch_retries_count_once(monkeypatch):
    """A batch mixing query sizes under tight MEMLIMITs re-runs steps that
    overflow their level buffer; queries that end at such a step must still be
    counted once (per-step count scratch, committed on acceptance).  Children
    are written in tile-completion order, so the chunking of later levels (and
    whether a step overflows) varies from run to run; a survivor guess of 0.1%
    makes every depth's first chunk far larger than its buffer, so steps do
    overflow and are re-run.  Counts must equal the unconstrained run's,
    shared and unshared."""
    monkeypatch.setenv("GFSM_TILE", "0")
    monkeypatch.setenv("GFSM_SURVIVOR_GUESS", "0.001")
    g = synth.grid(200, 0.05, 0.05, seed=21)
    g.vlabel = synth.vlabels(g.n, 2, 0.0, seed=22)
    s, d = g.directed()
    results = []
    for share, mem in [(sh, m) for sh in ("0", "1") for m in (None, 24 << 20, 16 << 20, 12 << 20, 10 << 20)]:
        monkeypatch.setenv("GFSM_SHARE", share)
        kw = {} if mem is None else dict(mem_limit=mem, max_scan_size=1 << 20)
        ctx = gfsm_b200.GFSM(device=0, vertex_labels=1, **kw)
        data = ctx.graph_from_edges(g.n, s, d, None, g.vlabel)
        plans = []
        for i in range(60):
            qg, _ = synth.rw_query(g, 3 + i % 6, tree=i % 3 == 0, seed=700 + i)
            qs, qd = qg.directed()
            plans.append(ctx.pre_process_query(ctx.graph_from_edges(qg.n, qs, qd, None, qg.vlabel)))
        counts, st = ctx.batch_count(plans, data)
        results.append((counts.tolist(), st["retries"], st["steps"]))
        ctx.close()
    ref = results[0][0]
    assert sum(ref) > 0
    for counts, retries, steps in results[1:]:
        assert counts == ref
    assert min(r for _, r, _ in results[1:5]) > 0, [(r, st) for _, r, st in results]


def test_shared_prefix_batches(monkeypatch):
    """Queries whose plans coincide up to some depth share those levels (one
    tuple per shared partial mapping, fanned out to the child prefixes where
    they part); the counts must equal unshared batching and one-at-a-time
    matching, on both drivers, including members that end at a shared depth."""
    ctx = gfsm_b200.GFSM(device=0, vertex_labels=1)
    g = synth.grid(150, 0.05, 0.03, seed=31)
    g.vlabel = synth.vlabels(g.n, 2, 0.0, seed=32)
    s, d = g.directed()
    data = ctx.graph_from_edges(g.n, s, d, None, g.vlabel)
    plans = []
    for i in range(200):
        qg, _ = synth.rw_query(g, 2 + i % 7, tree=i % 4 == 0, seed=900 + i)
        qs, qd = qg.directed()
        plans.append(ctx.pre_process_query(ctx.graph_from_edges(qg.n, qs, qd, None, qg.vlabel)))
    single = [ctx.match_count(p, data)[0] for p in plans]
    monkeypatch.setenv("GFSM_SHARE", "0")
    unshared, st0 = ctx.batch_count(plans, data)
    monkeypatch.setenv("GFSM_SHARE", "1")
    shared, st1 = ctx.batch_count(plans, data)
    monkeypatch.setenv("GFSM_DRIVER", "graph")
    shared_g, st2 = ctx.batch_count(plans, data)
    assert unshared.tolist() == single == shared.tolist() == shared_g.tolist()
    assert st1["candidates"] < st0["candidates"]  # levels 0 and 1 ran once per class
    assert sum(single) > 0
    ctx.close()


@pytest.mark.parametrize("gen", range(len(GENS)))
def test_data_aware_order(gpu_ctx_vl, tmp_path, gen):
    """Plans with the data-aware matching order (gfsm_query_prepare_for, Zipf
    vertex labels so label windows differ) count exactly what the reference
    order counts -- on the device, and in the oracle run over the same plan
    tables; the batch planner with a data graph gives the same plans."""
    name, fn = GENS[gen]
    g = fn(gen + 11)
    g.vlabel = synth.vlabels(g.n, 5, 1.0, seed=gen + 60)
    dpath = tmp_path / "d.g"
    g.write_text(str(dpath))
    od = O.Graph(path=str(dpath))
    ds, dd = g.directed()
    data = gpu_ctx_vl.graph_from_edges(g.n, ds, dd, None, g.vlabel)
    qd, differ = [], 0
    for i, k in enumerate((3, 4, 5, 6, 7, 5, 6, 7)):
        qg, _ = synth.rw_query(g, k, tree=i % 3 == 1, seed=700 * gen + i)
        qpath = tmp_path / "q.g"
        qg.write_text(str(qpath))
        q = gpu_ctx_vl.file_parse(str(qpath))
        ref, mine = gpu_ctx_vl.pre_process_query(q), gpu_ctx_vl.plan_for(q, data)
        assert mine.info() == {"planner": 1, "order_invariant": True}
        oq = O.Graph(path=str(qpath))
        expect = O.ffs_count(oq, O.Plan(oq), od, vlabel_mode=True, threads=8)
        assert O.ffs_count(oq, O.TablePlan(oq, mine.tables()), od, vlabel_mode=True, threads=8) == expect
        assert gpu_ctx_vl.match_count(ref, data)[0] == expect
        assert gpu_ctx_vl.match_count(mine, data)[0] == expect, (name, k, i)
        differ += mine.tables()["order"].tolist() != ref.tables()["order"].tolist()
        qs, qt = qg.directed()
        qd.append((qg.n, qs, qt, None, qg.vlabel))
    assert differ > 0
    batch = gpu_ctx_vl.prepare_queries(qd, data)
    singles = [gpu_ctx_vl.plan_for(gpu_ctx_vl.graph_from_edges(*q), data) for q in qd]
    for a, b in zip(batch, singles):
        assert a.tables()["order"].tolist() == b.tables()["order"].tolist()
    c1, _ = gpu_ctx_vl.batch_count(batch, data)
    c2, _ = gpu_ctx_vl.batch_count(gpu_ctx_vl.prepare_queries(qd), data)
    assert c1.tolist() == c2.tolist()


def test_data_aware_order_falls_back_on_directed_data(gpu_ctx):
    """Where the count could depend on the order (a data edge without its
    reverse), gfsm_query_prepare_for keeps the reference's order."""
    g = synth.er(200, 4.0, seed=9)
    s, d = g.src.astype(np.uint32), g.dst.astype(np.uint32)   # one direction only
    data = gpu_ctx.graph_from_edges(g.n, s, d)
    q = gpu_ctx.file_parse(_g("queries/_3_triangle"))
    mine, ref = gpu_ctx.plan_for(q, data), gpu_ctx.pre_process_query(q)
    assert mine.info()["planner"] == 0
    assert mine.tables()["order"].tolist() == ref.tables()["order"].tolist()
    assert gpu_ctx.match_count(mine, data)[0] == gpu_ctx.match_count(ref, data)[0]


def test_shared_prefixes_identical_queries_on_a_hub():
    """900 identical triangle queries on a graph with a 40,000-entry row (a
    star) and a K5: one trie path for all of them, counted once and copied to
    every member -- each count equals the single-query count (60: the
    ordered triangles of a K5)."""
    ctx = gfsm_b200.GFSM(device=0)
    m = 40000
    src = list(np.zeros(m, np.uint32)) + list(range(1, m + 1))
    dst = list(range(1, m + 1)) + list(np.zeros(m, np.uint32))
    k5 = [m + 1 + i for i in range(5)]
    for a in k5:
        for b in k5:
            if a != b:
                src.append(a)
                dst.append(b)
    data = ctx.graph_from_edges(m + 6, np.array(src, np.uint32), np.array(dst, np.uint32))
    tri = ctx.pre_process_query(ctx.file_parse(_g("queries/_3_triangle")))
    one = ctx.match_count(tri, data)[0]
    assert one == 60
    counts, st = ctx.batch_count([tri] * 900, data)
    assert counts.tolist() == [one] * 900
    ctx.close()


def test_trie_too_wide_for_row_size_runs_unshared():
    """With a 2^24-entry row (a star), a trie node may not branch at all
    (its fan-out times the row must fit 32-bit slice sums with 128 per warp);
    three queries with the same root level but different depth-1 plans (their
    depth-2 windows differ) would make the root node branch, so the call runs
    unshared, and the counts equal one-at-a-time matching and the oracle."""
    ctx = gfsm_b200.GFSM(device=0, vertex_labels=1)
    m = 1 << 24
    leaves = np.arange(1, m + 1, dtype=np.uint32)
    hub = np.zeros(m, np.uint32)
    # a labelled grid component (labels 1..3) beside the label-0 star
    comp = synth.grid(20, 0.0, 0.05, seed=41)
    off = m + 1
    cs, cd = comp.directed()
    src = np.concatenate([hub, leaves, cs.astype(np.uint32) + off])
    dst = np.concatenate([leaves, hub, cd.astype(np.uint32) + off])
    vl = np.concatenate([np.zeros(m + 1, np.uint32), 1 + synth.vlabels(comp.n, 3, 0.0, seed=42)])
    data = ctx.graph_from_edges(m + 1 + comp.n, src, dst, None, vl)
    # paths a-b-c, planned b, a, c: b labelled 1, a 2, and c 1, 2 or 3
    qs = []
    for l3 in (1, 2, 3):
        qvl = np.array([2, 1, l3], np.uint32)
        qs.append((3, np.array([0, 1, 1, 2], np.uint32), np.array([1, 0, 2, 1], np.uint32), None, qvl))
    plans = [ctx.pre_process_query(ctx.graph_from_edges(*q)) for q in qs]
    alone = [ctx.match_count(p, data) for p in plans]
    single = [c for c, _ in alone]
    batch, st = ctx.batch_count(plans, data)
    assert batch.tolist() == single and sum(single) > 0
    # unshared: the batch processes exactly the candidates of the three calls
    # (shared, the common root level would run once)
    assert st["candidates"] == sum(s["candidates"] for _, s in alone)
    # the oracle on the component alone (the star has no labels 1-3)
    ccs, ccd = comp.directed()
    cvl = vl[off:]
    for (n, a, b, _, qvl), c in zip(qs, single):
        assert c == O.bt_count(n, a, b, None, qvl, comp.n, ccs, ccd, None, cvl, vlabel_mode=True)
    ctx.close()
