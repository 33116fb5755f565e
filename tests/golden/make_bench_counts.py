#!/usr/bin/env python
"""Oracle counts for every query of the benchmark's headline batch.

The batch is the one ``bench.py`` times: the 1,400 x 1,400 road-like grid
(5% of edges removed, 2% shortcuts, 4 uniform vertex labels) and 4,096
seeded random-walk queries of 4-10 vertices with all induced edges, vertex
labels matched.  Each query is counted by the oracle's restatement of the
reference FFS (oracle/gfsm_oracle.c, ``orc_ffs_count``), one query per
worker process, and the counts are written to
``tests/golden/bench_cfg5_counts.json`` together with the workload's seeds.

    python tests/golden/make_bench_counts.py [--queries N] [--workers W]

CPU only; about half an hour on 8 cores.  ``bench.py`` checks every batched,
plain and served count of rank 0 against this file.
"""
import argparse
import json
import multiprocessing as mp
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "bench_cfg5_counts.json")

_state = {}


def _init(dpath):
    sys.path.insert(0, ROOT)
    from oracle import oracle
    _state["oracle"] = oracle
    _state["data"] = oracle.Graph(path=dpath)


def _count(item):
    i, text = item
    o = _state["oracle"]
    q = o.Graph(text=text)
    return i, o.ffs_count(q, o.Plan(q), _state["data"], vlabel_mode=True, threads=1)


def query_text(q):
    path = tempfile.mktemp(suffix=".g")
    q.write_text(path)
    with open(path) as f:
        t = f.read()
    os.unlink(path)
    return t


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--queries", type=int, default=4096)
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    sys.path.insert(0, ROOT)
    import bench
    g, qs = bench.make_workload(0, args.queries)
    tmp = tempfile.mkdtemp()
    dpath = os.path.join(tmp, "grid.g")
    g.write_text(dpath)
    items = [(i, query_text(q)) for i, q in enumerate(qs)]
    counts = [None] * len(items)
    t0 = time.time()
    ctx = mp.get_context("spawn")
    with ctx.Pool(args.workers, initializer=_init, initargs=(dpath,)) as pool:
        for n, (i, c) in enumerate(pool.imap_unordered(_count, items, chunksize=4)):
            counts[i] = c
            if (n + 1) % 256 == 0:
                print(f"{n + 1}/{len(items)} queries, {time.time() - t0:.0f} s", flush=True)
    os.unlink(dpath)
    os.rmdir(tmp)
    rec = {
        "workload": bench.WORKLOAD,
        "grid_side": bench.GRID_SIDE, "graph_seed": 0, "vlabel_seed": 100, "query_rng_seed": 11,
        "query_seed": "1 + i", "kmin": bench.KMIN, "kmax": bench.KMAX, "vertex_labels": True,
        "checker": "oracle orc_ffs_count (reference FFS restatement)",
        "queries": len(counts), "counts": counts,
    }
    with open(OUT, "w") as f:
        json.dump(rec, f, separators=(",", ":"))
        f.write("\n")
    print(f"wrote {OUT}: {len(counts)} counts, total {sum(counts)}, {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
