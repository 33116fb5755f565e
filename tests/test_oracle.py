"""CPU tests of the oracle: pinned to the reference's own front-end output
(tests/golden/ref_frontend.json, produced by the reference's fileParse /
preProcessQuery), to closed-form counts, and to agreement between the FFS
restatement and the independent backtracking enumerator."""
import glob
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from gfsm_b200 import synth

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REF = json.load(open(os.path.join(GOLD, "ref_frontend.json")))
COUNTS = json.load(open(os.path.join(GOLD, "counts.json")))


def _gfile(key):
    return os.path.join(GOLD, key + ".g")


@pytest.mark.parametrize("key", sorted(REF))
def test_oracle_parse_matches_reference(key):
    r = REF[key]
    g = O.Graph(path=_gfile(key))
    assert g.err == 0
    a = g.arrays()
    assert a["count"] == r["count"] and a["size"] == r["size"]
    assert g.packed().tolist() == r["segments"]
    assert a["vlocs"].tolist() == r["vlocs"]
    assert a["inv"].tolist() == r["inv"]
    assert a["staggers"].tolist() == r["staggers"]
    assert a["sinfo"].tolist() == r["sinfo"]


@pytest.mark.parametrize("key", sorted(k for k in REF if k.startswith("queries/")))
def test_oracle_plan_matches_reference(key):
    r = REF[key]
    t = O.Plan(O.Graph(path=_gfile(key))).tables()
    assert t["max_valency"] == r["max_valency"]
    assert t["reqs"].tolist() == r["reqs"]
    assert t["header"].tolist() == r["header"]


@pytest.mark.parametrize("key", sorted(COUNTS))
def test_oracle_golden_counts(key):
    qn, dn = key.split("|")
    q = O.Graph(path=_gfile("queries/" + qn))
    d = O.Graph(path=_gfile("data/" + dn))
    p = O.Plan(q)
    assert O.ffs_count(q, p, d, threads=4) == COUNTS[key]["count"]
    assert O.ffs_count(q, p, d, vlabel_mode=True, threads=4) == COUNTS[key]["count_vlabels"]


def _complete(n):
    s, d = np.triu_indices(n, 1)
    return synth.UGraph(n, s.astype(np.uint32), d.astype(np.uint32))


def _text(g, tmp_path, name, lab=None):
    p = tmp_path / name
    g.write_text(str(p), lab)
    return O.Graph(path=str(p))


def test_closed_forms(tmp_path):
    # triangle on K_n: n(n-1)(n-2); K_{1,4} ("plus") on a star K_{1,m}: m(m-1)(m-2)(m-3);
    # a k-vertex path on the cycle C_n: 2n
    tri = O.Graph(path=_gfile("queries/_3_triangle"))
    for n in (3, 4, 7, 10):
        d = _text(_complete(n), tmp_path, f"k{n}.g")
        assert O.ffs_count(tri, O.Plan(tri), d) == n * (n - 1) * (n - 2)
    plus = O.Graph(path=_gfile("queries/_5_plus"))
    for m in (4, 6, 9):
        star = synth.UGraph(m + 1, np.zeros(m, np.uint32), np.arange(1, m + 1, dtype=np.uint32))
        d = _text(star, tmp_path, f"s{m}.g")
        assert O.ffs_count(plus, O.Plan(plus), d) == m * (m - 1) * (m - 2) * (m - 3)
    for k, qn in ((2, "_2_road2"), (3, "_3_road3"), (4, "_4_road4"), (5, "_5_road5")):
        q = O.Graph(path=_gfile("queries/" + qn))
        for n in (k if k > 2 else 3, 8, 13):
            if n < k:
                continue
            cyc = synth.UGraph(n, np.arange(n, dtype=np.uint32), (np.arange(n, dtype=np.uint32) + 1) % n)
            cyc.src, cyc.dst = np.minimum(cyc.src, cyc.dst), np.maximum(cyc.src, cyc.dst)
            d = _text(cyc, tmp_path, f"c{n}.g")
            expect = 2 * n if not (k == n == 3) else 6
            assert O.ffs_count(q, O.Plan(q), d) == expect


@pytest.mark.parametrize("seed", range(6))
def test_ffs_matches_backtracking(seed, tmp_path):
    gen = [lambda: synth.er(120, 5.0, seed=seed), lambda: synth.ba(150, 2, seed=seed),
           lambda: synth.grid(10, 0.1, 0.05, seed=seed)][seed % 3]
    g = gen()
    g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=seed + 50)
    lab = (np.arange(g.m, dtype=np.uint32) * 7 + seed) % 2 + 1 if seed % 2 else None
    d = _text(g, tmp_path, "d.g", lab)
    ds, dd, dl = d.edges()
    for k in (3, 4, 5):
        for tree in (False, True):
            qg, visited = synth.rw_query(g, k, tree=tree, seed=100 * seed + k)
            qlab = None
            if lab is not None:
                key = {(int(a), int(b)): int(l) for a, b, l in zip(g.src, g.dst, lab)}
                qlab = np.array([key[(min(visited[a], visited[b]), max(visited[a], visited[b]))]
                                 for a, b in zip(qg.src, qg.dst)], np.uint32)
            q = _text(qg, tmp_path, "q.g", qlab)
            p = O.Plan(q)
            assert p.err == 0
            qs, qd, ql = q.edges()
            for vl in (False, True):
                c1 = O.ffs_count(q, p, d, vlabel_mode=vl, threads=2)
                c2 = O.bt_count(k, qs, qd, ql, q.arrays()["vlabel"], g.n, ds, dd, dl, d.arrays()["vlabel"],
                                vlabel_mode=vl, threads=2)
                assert c1 == c2 and c1 >= (1 if not vl else 0)


def test_mappings_agree(tmp_path):
    g = synth.er(60, 5.0, seed=3)
    d = _text(g, tmp_path, "d.g")
    q = O.Graph(path=_gfile("queries/_4_square"))
    p = O.Plan(q)
    c1, r1 = O.ffs_count(q, p, d, max_rows=100000)
    qs, qd, ql = q.edges()
    ds, dd, dl = d.edges()
    c2, r2 = O.bt_count(4, qs, qd, ql, None, g.n, ds, dd, dl, None, max_rows=100000)
    assert c1 == c2 == len(r1) == len(r2)
    s1 = r1[np.lexsort(r1.T[::-1])]
    s2 = r2[np.lexsort(r2.T[::-1])]
    assert np.array_equal(s1, s2)


def test_parser_error_codes(tmp_path):
    (tmp_path / "bad.g").write_text("t # 1\n1 0 1 1\nt # -1")
    assert O.Graph(path=str(tmp_path / "bad.g")).err == 233
    assert O.Graph(path=str(tmp_path / "missing.g")).err == 232
    (tmp_path / "few.g").write_text("t # 0\n3 2 1 1\nv 0 1\nt # -1")
    assert O.Graph(path=str(tmp_path / "few.g")).err == 234
    (tmp_path / "fewe.g").write_text("t # 0\n2 4 1 1\nv 0 1\nv 1 1\ne 0 1 1\ne 1 0 1\nt # -1")
    assert O.Graph(path=str(tmp_path / "fewe.g")).err == 234
    (tmp_path / "junk.g").write_text("t # 0\n2 2 1 1\nv 0 1\nx 1 1\nt # -1")
    assert O.Graph(path=str(tmp_path / "junk.g")).err == 233


def test_disconnected_query_rejected(tmp_path):
    (tmp_path / "dq.g").write_text("t # 0\n4 4 1 1\nv 0 1\nv 1 1\nv 2 1\nv 3 1\n"
                                   "e 0 1 1\ne 1 0 1\ne 2 3 1\ne 3 2 1\nt # -1")
    q = O.Graph(path=str(tmp_path / "dq.g"))
    assert O.Plan(q).err == 1


@pytest.mark.skipif(not os.path.exists(O.REF_FRONTEND), reason="reference front-end not built here")
def test_reference_frontend_live(tmp_path):
    """Live comparison with the reference's own parser/planner on fresh inputs,
    including its parser's error exits."""
    for seed in range(4):
        g = synth.ba(80 + seed * 30, 2 + seed % 3, seed=seed)
        p = tmp_path / f"g{seed}.g"
        g.write_text(str(p))
        rc, r = O.ref_frontend_dump(str(p))
        d = O.Graph(path=str(p))
        assert rc == 0 and d.packed().tolist() == r["segments"].tolist()
        assert d.arrays()["sinfo"].tolist() == r["sinfo"].tolist()
        qg, _ = synth.rw_query(g, 6, tree=seed % 2 == 0, seed=seed)
        qp = tmp_path / f"q{seed}.g"
        qg.write_text(str(qp))
        rc, r = O.ref_frontend_dump(str(qp), plan=True)
        t = O.Plan(O.Graph(path=str(qp))).tables()
        assert rc == 0 and t["reqs"].tolist() == r["reqs"].tolist() and t["header"].tolist() == r["header"].tolist()
    (tmp_path / "few.g").write_text("t # 0\n3 2 1 1\nv 0 1\nt # -1")
    assert O.ref_frontend_dump(str(tmp_path / "few.g"))[0] == 234
    (tmp_path / "bad.g").write_text("t # 1\n1 0 1 1\nt # -1")
    assert O.ref_frontend_dump(str(tmp_path / "bad.g"))[0] == 233
    # the reference's shipped sample queries (kept as fixtures) parse and plan
    # in the reference's own front-end exactly as recorded
    for f in glob.glob(os.path.join(GOLD, "queries", "*.g")):
        name = os.path.basename(f)[:-2]
        rc, r = O.ref_frontend_dump(f, plan=True)
        assert rc == 0
        assert r["segments"].tolist() == REF["queries/" + name]["segments"]
        assert r["reqs"].tolist() == REF["queries/" + name]["reqs"]


@pytest.mark.skipif(not os.path.exists(O.REF_FRONTEND), reason="reference front-end not built here")
def test_reference_frontend_live_irregular_queries(tmp_path):
    """The reference's own planner on queries with repeated edges (one pair
    under two labels), self-loops, one-way edges and three edge labels: where
    it plans the query, the product's planner and the oracle give its
    requirement table bit for bit; where it exits, both reject the query.
    Every vertex has a row (the reference walks past its CCSR otherwise) and
    no row holds more than 16 entries."""
    import gfsm_b200
    ctx = gfsm_b200.GFSM(device=-1)
    rng = np.random.default_rng(23)
    planned = rejected = 0
    for i in range(120):
        k = int(rng.integers(2, 13))
        edges = []
        for v in range(1, k):
            u, l = int(rng.integers(v)), int(rng.integers(1, 4))
            edges.append((u, v, l))
            edges.append((v, u, l if rng.random() < 0.8 else int(rng.integers(1, 4))))
        for _ in range(int(rng.integers(0, k + 1))):
            a, b, l = int(rng.integers(k)), int(rng.integers(k)), int(rng.integers(1, 4))
            edges.append((a, b, l))
            if rng.random() < 0.6:
                edges.append((b, a, l))
        rng.shuffle(edges)
        out = np.bincount(np.array([a for a, _, _ in edges], np.int64), minlength=k)
        if out.min() == 0 or out.max() > 16:
            continue
        lines = ["t # 0", f"{k} {len(edges)} 1 1"] + [f"v {v} 1" for v in range(k)]
        lines += [f"e {a} {b} {l}" for a, b, l in edges] + ["t # -1"]
        path = tmp_path / f"q{i}.g"
        path.write_text("\n".join(lines) + "\n")
        rc, r = O.ref_frontend_dump(str(path), plan=True)
        orc = O.Plan(O.Graph(path=str(path)))
        try:
            mine = ctx.pre_process_query(ctx.file_parse(str(path))).tables()
        except gfsm_b200.GFSMError:
            mine = None
        if rc != 0:
            assert mine is None and orc.err, (i, rc, edges)
            rejected += 1
            continue
        assert mine is not None and not orc.err, (i, edges)
        t = orc.tables()
        assert t["reqs"].tolist() == r["reqs"].tolist() and t["header"].tolist() == r["header"].tolist(), (i, edges)
        assert mine["reqs"].tolist() == r["reqs"].tolist() and mine["header"].tolist() == r["header"].tolist(), (i, edges)
        planned += 1
    ctx.close()
    assert planned > 40


@pytest.mark.parametrize("vl", [False, True])
def test_data_aware_order_counts_the_same(tmp_path, vl):
    """Plans from gfsm_query_prepare_for (data-aware matching order), run by
    the oracle's level semantics, count what the reference order counts and
    what the independent backtracking enumerator counts."""
    import gfsm_b200
    from gfsm_b200 import synth
    ctx = gfsm_b200.GFSM(device=-1, vertex_labels=int(vl))
    gens = [synth.er(300, 5, seed=3), synth.ba(300, 2, seed=4), synth.grid(16, 0.05, 0.02, seed=5)]
    differ = 0
    for gi, g in enumerate(gens):
        g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=6 + gi)
        dpath = tmp_path / f"d{gi}.g"
        g.write_text(str(dpath))
        data = ctx.file_parse(str(dpath))
        od = O.Graph(path=str(dpath))
        for i in range(12):
            k = 3 + i % 4 if not vl else 3 + i % 5
            qg, _ = synth.rw_query(g, k, tree=i % 3 == 0, seed=50 * gi + i)
            qpath = tmp_path / f"q{gi}_{i}.g"
            qg.write_text(str(qpath))
            q = ctx.file_parse(str(qpath))
            mine = ctx.plan_for(q, data)
            ref = ctx.pre_process_query(q)
            assert mine.info()["order_invariant"]
            oq = O.Graph(path=str(qpath))
            c_ref = O.ffs_count(oq, O.Plan(oq), od, vlabel_mode=vl)
            c_mine = O.ffs_count(oq, O.TablePlan(oq, mine.tables()), od, vlabel_mode=vl)
            qs, qd = qg.directed()
            ds, dd = g.directed()
            c_bt = O.bt_count(qg.n, qs, qd, None, qg.vlabel, g.n, ds, dd, None, g.vlabel, vlabel_mode=vl)
            assert c_mine == c_ref == c_bt, (gi, i, c_mine, c_ref, c_bt)
            differ += mine.tables()["order"].tolist() != ref.tables()["order"].tolist()
    if vl:  # unlabelled, both orders take high-degree rows first and mostly agree
        assert differ > 0


@pytest.mark.parametrize("vl", [False, True])
def test_symmetry_breaking_counts_one_embedding_per_orbit(vl):
    """gfsm_plan_symmetry: of every embedding the independent enumerator
    lists, those meeting the conditions f(a) < f(b) (original vertex ids --
    any fixed order works) number exactly total / |Aut(Q)|."""
    import gfsm_b200
    from gfsm_b200 import synth
    ctx = gfsm_b200.GFSM(device=-1, vertex_labels=int(vl))
    nontrivial = 0
    for gi, g in enumerate([synth.er(60, 6.0, seed=5), synth.grid(9, 0.0, 0.1, seed=6),
                            synth.ba(80, 3, seed=7)]):
        g.vlabel = synth.vlabels(g.n, 2, 0.0, seed=8 + gi)
        ds, dd = g.directed()
        qs = [synth.rw_query(g, 3 + i % 4, tree=i % 2 == 0, seed=40 * gi + i)[0] for i in range(10)]
        # plus small symmetric shapes: triangle, 4-cycle, star, 4-clique
        shapes = [(3, [(0, 1), (1, 2), (2, 0)]), (4, [(0, 1), (1, 2), (2, 3), (3, 0)]),
                  (4, [(0, 1), (0, 2), (0, 3)]), (4, [(a, b) for a in range(4) for b in range(a + 1, 4)])]
        cases = [(q.n, *q.directed(), q.vlabel) for q in qs]
        for n, ed in shapes:
            s_ = np.array([a for a, b in ed] + [b for a, b in ed], np.uint32)
            d_ = np.array([b for a, b in ed] + [a for a, b in ed], np.uint32)
            cases.append((n, s_, d_, np.zeros(n, np.uint32)))
        for n, qs_, qd_, qvl in cases:
            plan = ctx.pre_process_query(ctx.graph_from_edges(n, qs_, qd_, None, qvl))
            aut, cond = plan.symmetry()
            total, rows = O.bt_count(n, qs_, qd_, None, qvl, g.n, ds, dd, None, g.vlabel, vlabel_mode=vl,
                                     max_rows=1 << 22)
            assert len(rows) == total
            keep = np.ones(len(rows), bool)
            for a, b in cond:
                keep &= rows[:, a] < rows[:, b]
            assert int(keep.sum()) * aut == total, (gi, n, aut, cond)
            nontrivial += aut > 1
    assert nontrivial >= 6


@pytest.mark.parametrize("vl", [False, True])
def test_config1_ffs_matches_backtracking(vl, tmp_path):
    """Configuration 1 at its stated size (ER n=2,000, average degree 8, seed
    0, 4 uniform vertex labels, one 5-vertex random-walk query): the FFS
    restatement and the independent enumerator agree."""
    g, (q,) = synth.config1()
    g.write_text(str(tmp_path / "d.g"))
    q.write_text(str(tmp_path / "q.g"))
    od, oq = O.Graph(path=str(tmp_path / "d.g")), O.Graph(path=str(tmp_path / "q.g"))
    ffs = O.ffs_count(oq, O.Plan(oq), od, vlabel_mode=vl, threads=8)
    ds, dd = g.directed()
    qs, qd = q.directed()
    bt = O.bt_count(q.n, qs, qd, None, q.vlabel, g.n, ds, dd, None, g.vlabel, vlabel_mode=vl, threads=8)
    assert ffs == bt > 0


def test_three_vertex_closed_forms_match_backtracking():
    """The exact methods the large-configuration fixtures use for 3-vertex
    queries -- the labelled 2-path closed form and the labelled triangle
    histogram -- equal the independent enumerator on every label pattern."""
    g = synth.er(300, 6.0, seed=3)
    g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=4)
    H = O.triangle_label_hist(g.n, g.src, g.dst, g.vlabel, 3)
    P = O.path3_label_counts(g.n, g.src, g.dst, g.vlabel, 3)
    ds, dd = g.directed()
    tri = (np.array([0, 1, 0, 1, 2, 2], np.uint32), np.array([1, 0, 2, 2, 0, 1], np.uint32))
    path = (np.array([0, 1, 1, 2], np.uint32), np.array([1, 0, 2, 1], np.uint32))
    for a in range(3):
        for b in range(3):
            for c in range(3):
                qvl = np.array([a, b, c], np.uint32)
                assert O.bt_count(3, *tri, None, qvl, g.n, ds, dd, None, g.vlabel, vlabel_mode=True) == H[a, b, c]
                assert O.bt_count(3, *path, None, qvl, g.n, ds, dd, None, g.vlabel, vlabel_mode=True) == P[a, b, c]
    assert H.sum() == 6 * O.triangles(g.n, g.src, g.dst)
