"""Generates the golden fixtures under tests/golden/.

    python tests/golden/make_golden.py        (needs oracle/_ref/ref_frontend)

* queries/*.g  -- the eight query shapes the reference ships as its only test
  inputs (path of 2..5 vertices, triangle, square, "Y", "plus"), written by
  our own writer in the `t # / v / e` format with both edge directions;
* data/*.g     -- small seeded data graphs (Erdos-Renyi, Barabasi-Albert,
  grid with shortcuts, and an edge-labelled Erdos-Renyi);
* ref_frontend.json -- for every file above, the CCSR (packed 32-bit
  segments, verticeLocs, invVerticeLocs, staggers, StaggerInfo) and, for
  queries, the plan (requirements, requirement header, maxValency) exactly as
  produced by the reference's own fileParse / preProcessQuery, compiled from
  its sources into oracle/_ref/ref_frontend;
* counts.json  -- embedding count of every (query, data) pair, from the
  oracle's restatement of the reference's FFS semantics, generated only when
  the independent backtracking enumerator gives the same number.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gfsm_b200 import synth  # noqa: E402
from oracle import oracle  # noqa: E402

QUERY_SHAPES = {
    "_2_road2": (2, [(0, 1)]),
    "_3_road3": (3, [(0, 1), (1, 2)]),
    "_3_triangle": (3, [(0, 1), (1, 2), (2, 0)]),
    "_4_road4": (4, [(0, 1), (1, 2), (2, 3)]),
    "_4_roadY": (4, [(0, 1), (0, 2), (0, 3)]),
    "_4_square": (4, [(0, 1), (1, 2), (2, 3), (0, 3)]),
    "_5_plus": (5, [(0, 1), (2, 1), (3, 1), (4, 1)]),
    "_5_road5": (5, [(0, 1), (1, 2), (2, 3), (3, 4)]),
}


def write_shape(path, k, edges):
    lines = ["t # 0", f"{k} {2 * len(edges)} 1 1"]
    lines += [f"v {i} 1" for i in range(k)]
    for a, b in edges:
        lines.append(f"e {a} {b} 1")
        lines.append(f"e {b} {a} 1")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\nt # -1")


def data_graphs():
    out = {}
    g = synth.er(200, 6.0, seed=11)
    g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=12)
    out["er200"] = (g, None)
    g = synth.ba(300, 3, seed=13)
    g.vlabel = synth.vlabels(g.n, 4, 1.0, seed=14)
    out["ba300"] = (g, None)
    g = synth.grid(15, 0.05, 0.05, seed=15)
    g.vlabel = synth.vlabels(g.n, 2, 0.0, seed=16)
    out["grid15"] = (g, None)
    g = synth.er(150, 8.0, seed=17)
    g.vlabel = synth.vlabels(g.n, 3, 0.0, seed=18)
    lab = (np.arange(g.m, dtype=np.uint32) * 2654435761 % 3 + 1).astype(np.uint32)
    out["er150_lab3"] = (g, lab)
    return out


def main():
    qdir = os.path.join(HERE, "queries")
    ddir = os.path.join(HERE, "data")
    os.makedirs(qdir, exist_ok=True)
    os.makedirs(ddir, exist_ok=True)
    if not os.path.exists(oracle.REF_FRONTEND):
        sys.exit("oracle/_ref/ref_frontend not built (make -C oracle ref)")
    ref = {}
    for name, (k, edges) in QUERY_SHAPES.items():
        path = os.path.join(qdir, name + ".g")
        write_shape(path, k, edges)
        rc, d = oracle.ref_frontend_dump(path, plan=True)
        assert rc == 0, (name, rc)
        ref["queries/" + name] = {key: (v.tolist() if hasattr(v, "tolist") else v) for key, v in d.items()}
    for name, (g, lab) in data_graphs().items():
        path = os.path.join(ddir, name + ".g")
        g.write_text(path, lab)
        rc, d = oracle.ref_frontend_dump(path, plan=False)
        assert rc == 0, (name, rc)
        ref["data/" + name] = {key: (v.tolist() if hasattr(v, "tolist") else v) for key, v in d.items()}
    with open(os.path.join(HERE, "ref_frontend.json"), "w") as f:
        json.dump(ref, f, separators=(",", ":"))

    counts = {}
    for dname in sorted(os.listdir(ddir)):
        d = oracle.Graph(path=os.path.join(ddir, dname))
        ds, dd, dl = d.edges()
        for qname in sorted(os.listdir(qdir)):
            q = oracle.Graph(path=os.path.join(qdir, qname))
            p = oracle.Plan(q)
            c1 = oracle.ffs_count(q, p, d, threads=8)
            qs, qd, ql = q.edges()
            c2 = oracle.bt_count(q.arrays()["count"], qs, qd, ql, None, d.arrays()["count"], ds, dd, dl, None,
                                 threads=8)
            assert c1 == c2, (qname, dname, c1, c2)
            # vertex-label mode: the query's v-line labels must match
            c3 = oracle.ffs_count(q, p, d, vlabel_mode=True, threads=8)
            c4 = oracle.bt_count(q.arrays()["count"], qs, qd, ql, q.arrays()["vlabel"], d.arrays()["count"], ds, dd,
                                 dl, d.arrays()["vlabel"], vlabel_mode=True, threads=8)
            assert c3 == c4, (qname, dname, c3, c4)
            counts[f"{qname[:-2]}|{dname[:-2]}"] = {"count": c1, "count_vlabels": c3}
    with open(os.path.join(HERE, "counts.json"), "w") as f:
        json.dump(counts, f, indent=1, sort_keys=True)
    print(f"wrote {len(ref)} front-end dumps and {len(counts)} counts")


if __name__ == "__main__":
    main()
