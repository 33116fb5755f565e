#!/usr/bin/env python
"""Exact counts for the bench's configuration legs, CPU only.

  config 2: R-MAT(0.57, 0.19, 0.19, 0.05), 2^20 vertices, 16M undirected
            edges, unlabelled -- the triangle query's count, 6 x the oracle's
            triangle count (degree-ordered orientation + list intersection);
  config 4: labelled R-MAT 2^22, average degree 16, 8 uniform vertex labels,
            4,096 random-walk queries of 3-12 vertices (vertex labels matched)
            -- every 3-vertex query's count: a path x-y-z by the closed form
            sum_y N_a(y) N_c(y) - [a == c] N_a(y), a triangle by the oracle's
            labelled triangle histogram (oracle.path3_label_counts,
            oracle.triangle_label_hist, both checked against the backtracking
            enumerator in tests/test_oracle.py).

The reference's own FFS restatement is too slow at these sizes (its
requirement check scans a hub row linearly for every candidate), so these
independent exact methods stand in for it.  Writes
tests/golden/config_counts.json; a few minutes on 8 cores.

    python tests/golden/make_config_counts.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "config_counts.json")


def three_vertex_count(q, P, H):
    """Exact count of a 3-vertex query (path or triangle) from the tables."""
    lab = [int(x) for x in q.vlabel]
    if q.m == 3:
        return int(H[lab[0], lab[1], lab[2]])
    deg = np.bincount(np.concatenate([q.src, q.dst]), minlength=3)
    mid = int(np.argmax(deg))
    ends = [v for v in range(3) if v != mid]
    return int(P[lab[ends[0]], lab[mid], lab[ends[1]]])


def main():
    sys.path.insert(0, ROOT)
    from gfsm_b200 import synth
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    t0 = time.time()
    g2, _ = synth.config2()
    tri2 = 6 * O.triangles(g2.n, g2.src, g2.dst, threads=threads)
    print(f"config 2 triangle: {tri2} ({time.time() - t0:.0f} s)", flush=True)
    del g2
    g4, qs = synth.config4(nq=4096)
    H = O.triangle_label_hist(g4.n, g4.src, g4.dst, g4.vlabel, 8, threads=threads)
    P = O.path3_label_counts(g4.n, g4.src, g4.dst, g4.vlabel, 8)
    idx = [i for i, q in enumerate(qs) if q.n == 3]
    counts = [three_vertex_count(qs[i], P, H) for i in idx]
    print(f"config 4: {len(idx)} 3-vertex queries, total {sum(counts)} ({time.time() - t0:.0f} s)", flush=True)
    rec = {
        "config2": {"graph": "R-MAT(0.57,0.19,0.19,0.05) scale 20, 16Mi undirected edges, seed 0, unlabelled",
                    "triangle": tri2, "checker": "6 x oracle triangle count"},
        "config4": {"graph": "R-MAT scale 22, average degree 16, seed 0, 8 uniform vertex labels (seed 100)",
                    "queries": "synth.config4(nq=4096): random walks of U{3..12} vertices, all induced edges",
                    "vertex_labels": True, "indices": idx, "counts": counts,
                    "checker": "3-vertex paths: closed form over labelled neighbour counts; triangles: oracle "
                               "labelled triangle histogram"},
    }
    with open(OUT, "w") as f:
        json.dump(rec, f, separators=(",", ":"))
        f.write("\n")
    print(f"wrote {OUT} ({time.time() - t0:.0f} s)")


if __name__ == "__main__":
    main()
