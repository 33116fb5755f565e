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

CPU only; a few minutes on 8 cores.  ``bench.py`` checks every batched,
plain and served count of rank 0 against this file.

    python tests/golden/make_bench_counts.py --refsubset

writes ``tests/golden/bench_cfg5_refsubset_counts.json`` instead: the first 64
queries of the batch with at most 5 vertices, counted with vertex labels
ignored (the reference's semantics) -- the subset on which ``bench.py``
compares the reference GFSM build on the same GPU.
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
OUT_REF = os.path.join(HERE, "bench_cfg5_refsubset_counts.json")
REF_SUBSET_N, REF_SUBSET_KMAX = 64, 5

_state = {}


def _init(dpath):
    sys.path.insert(0, ROOT)
    from oracle import oracle
    _state["oracle"] = oracle
    _state["data"] = oracle.Graph(path=dpath)


def _count(item):
    i, text, vl, threads = item
    o = _state["oracle"]
    q = o.Graph(text=text)
    return i, o.ffs_count(q, o.Plan(q), _state["data"], vlabel_mode=vl, threads=threads)


def ref_subset(qs):
    """Indices of the batch's queries the reference-build comparison uses."""
    return [i for i, q in enumerate(qs) if q.n <= REF_SUBSET_KMAX][:REF_SUBSET_N]


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
    ap.add_argument("--refsubset", action="store_true")
    args = ap.parse_args()
    sys.path.insert(0, ROOT)
    import bench
    g, qs = bench.make_workload(0, args.queries)
    tmp = tempfile.mkdtemp()
    dpath = os.path.join(tmp, "grid.g")
    g.write_text(dpath)
    if args.refsubset:
        # label-off counts are large: fewer workers, each counting with threads
        idx = ref_subset(qs)
        items = [(j, query_text(qs[i]), False, 4) for j, i in enumerate(idx)]
        workers = max(1, args.workers // 4)
    else:
        items = [(i, query_text(q), True, 1) for i, q in enumerate(qs)]
        workers = args.workers
    counts = [None] * len(items)
    t0 = time.time()
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers, initializer=_init, initargs=(dpath,)) as pool:
        for n, (i, c) in enumerate(pool.imap_unordered(_count, items, chunksize=4)):
            counts[i] = c
            if (n + 1) % 256 == 0:
                print(f"{n + 1}/{len(items)} queries, {time.time() - t0:.0f} s", flush=True)
    os.unlink(dpath)
    os.rmdir(tmp)
    if args.refsubset:
        rec = {
            "workload": bench.WORKLOAD, "subset": f"first {REF_SUBSET_N} queries with <= {REF_SUBSET_KMAX} vertices",
            "indices": idx, "vertex_labels": False,
            "checker": "oracle orc_ffs_count (reference FFS restatement), vertex labels ignored",
            "queries": len(counts), "counts": counts,
        }
        with open(OUT_REF, "w") as f:
            json.dump(rec, f, separators=(",", ":"))
            f.write("\n")
        print(f"wrote {OUT_REF}: {len(counts)} counts, total {sum(counts)}, {time.time() - t0:.0f} s")
        return
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
