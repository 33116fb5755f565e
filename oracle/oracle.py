"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py as the checker / CPU baseline.  The product never uses
it.  Restatements and their reference citations are in gfsm_oracle.h.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_FRONTEND = os.path.join(HERE, "_ref", "ref_frontend")

u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)


class OrcGraph(C.Structure):
    _fields_ = [
        ("n", C.c_uint32), ("size", C.c_uint64), ("rows", C.c_uint32),
        ("seg_val", u32p), ("seg_lab", u32p), ("vlocs", u32p), ("inv", u32p),
        ("maxlen", C.c_uint32), ("staggers", u32p), ("sinfo", u32p), ("vlabel", u32p),
        ("n_edges", C.c_uint32), ("e_src", u32p), ("e_dst", u32p), ("e_lab", u32p),
        ("err", C.c_int32),
    ]


class OrcPlan(C.Structure):
    _fields_ = [
        ("k", C.c_uint32), ("max_valency", C.c_uint32), ("rel_bits", C.c_uint32), ("reqs", u32p), ("header", u32p),
        ("order", u32p), ("err", C.c_int32),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        lib.orc_parse_file.argtypes = [C.c_char_p, C.c_uint32, C.POINTER(OrcGraph)]
        lib.orc_parse_buffer.argtypes = [C.c_char_p, C.c_uint64, C.c_uint32, C.POINTER(OrcGraph)]
        lib.orc_graph_free.argtypes = [C.POINTER(OrcGraph)]
        lib.orc_plan.argtypes = [C.POINTER(OrcGraph), C.c_uint32, C.POINTER(OrcPlan)]
        lib.orc_plan_free.argtypes = [C.POINTER(OrcPlan)]
        lib.orc_pack_segments.argtypes = [C.POINTER(OrcGraph), C.c_uint32, u32p]
        lib.orc_ffs_count.argtypes = [C.POINTER(OrcGraph), C.POINTER(OrcPlan), C.POINTER(OrcGraph), C.c_int,
                                      C.c_int, u64p, u32p, C.c_uint64, u64p]
        lib.orc_ffs_count_rows.argtypes = [C.POINTER(OrcGraph), C.POINTER(OrcPlan), C.POINTER(OrcGraph), C.c_int,
                                           C.c_int, C.c_uint32, C.c_uint32, u64p, u32p, C.c_uint64, u64p]
        lib.orc_bt_count.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p, u32p, u32p,
                                     C.c_uint32, C.c_uint64, u32p, u32p, u32p, u32p,
                                     C.c_uint32, C.c_int, C.c_int, u64p, u32p, C.c_uint64, u64p]
        lib.orc_triangles.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int, u64p]
        lib.orc_triangle_label_hist.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, u32p, C.c_uint32, C.c_int,
                                                u64p, u64p]
        for f in ("orc_parse_file", "orc_parse_buffer", "orc_plan", "orc_ffs_count", "orc_ffs_count_rows", "orc_bt_count",
                  "orc_triangle_label_hist",
                  "orc_triangles"):
            getattr(lib, f).restype = C.c_int
        _lib = lib
    return _lib


def _arr(p, n, dtype=np.uint32):
    if n == 0 or not p:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(p, shape=(n,)).astype(dtype, copy=True)


class Graph:
    """Reference-style parse of a text graph (HnHelper.cuh:283 fileParse)."""

    def __init__(self, text=None, path=None, rel_bits=8):
        lib = load()
        self._g = OrcGraph()
        if path is not None:
            lib.orc_parse_file(str(path).encode(), rel_bits, C.byref(self._g))
        else:
            if isinstance(text, str):
                text = text.encode()
            lib.orc_parse_buffer(text, len(text), rel_bits, C.byref(self._g))
        self.rel_bits = rel_bits

    @property
    def err(self):
        return self._g.err

    def arrays(self):
        g = self._g
        return {
            "count": g.n, "size": g.size, "rows": g.rows,
            "seg_val": _arr(g.seg_val, g.size), "seg_lab": _arr(g.seg_lab, g.size),
            "vlocs": _arr(g.vlocs, g.n), "inv": _arr(g.inv, g.n),
            "staggers": _arr(g.staggers, g.maxlen), "sinfo": _arr(g.sinfo, 2 * g.maxlen),
            "vlabel": _arr(g.vlabel, g.n),
        }

    def packed(self):
        out = np.zeros(max(self._g.size, 1), np.uint32)
        load().orc_pack_segments(C.byref(self._g), self.rel_bits, out.ctypes.data_as(u32p))
        return out[: self._g.size]

    def edges(self):
        g = self._g
        return _arr(g.e_src, g.n_edges), _arr(g.e_dst, g.n_edges), _arr(g.e_lab, g.n_edges)

    def __del__(self):
        try:
            load().orc_graph_free(C.byref(self._g))
        except Exception:
            pass


class Plan:
    """Reference planner restatement (HnGPU.cu:749-816, ccsr.cpp:98-219)."""

    def __init__(self, q):
        self._p = OrcPlan()
        load().orc_plan(C.byref(q._g), q.rel_bits, C.byref(self._p))
        self.q = q

    @property
    def err(self):
        return self._p.err

    def tables(self):
        p = self._p
        return {"k": p.k, "max_valency": p.max_valency, "order": _arr(p.order, p.k),
                "header": _arr(p.header, 3 * p.k), "reqs": _arr(p.reqs, 2 * p.max_valency * p.k)}

    def __del__(self):
        try:
            load().orc_plan_free(C.byref(self._p))
        except Exception:
            pass


class TablePlan:
    """A plan given as tables (order, header, reqs in the reference's packed
    layout), e.g. one made with another matching order; ffs_count runs the
    same level semantics over it."""

    def __init__(self, q, tables, rel_bits=8):
        self._keep = [np.ascontiguousarray(tables[k], np.uint32) for k in ("reqs", "header", "order")]
        reqs, header, order = self._keep
        self._p = OrcPlan(k=int(tables["k"]), max_valency=int(tables["max_valency"]), rel_bits=rel_bits,
                          reqs=reqs.ctypes.data_as(u32p), header=header.ctypes.data_as(u32p),
                          order=order.ctypes.data_as(u32p), err=0)
        self.q = q


def ffs_count(q, plan, d, vlabel_mode=False, threads=1, max_rows=0):
    """Reference-semantics count; with max_rows, also the mappings (ids)."""
    cnt = C.c_uint64()
    nr = C.c_uint64()
    rows = np.zeros((max(max_rows, 1), plan._p.k), np.uint32) if max_rows else None
    rc = load().orc_ffs_count(C.byref(q._g), C.byref(plan._p), C.byref(d._g), int(vlabel_mode), int(threads),
                              C.byref(cnt), rows.ctypes.data_as(u32p) if rows is not None else None,
                              int(max_rows), C.byref(nr))
    if rc:
        raise RuntimeError(f"orc_ffs_count failed ({rc})")
    if max_rows:
        return cnt.value, rows[: nr.value]
    return cnt.value


def ffs_count_rows(q, plan, d, root_begin, root_end, vlabel_mode=False, threads=1):
    """ffs_count over the roots in CCSR rows [root_begin, root_end) only."""
    cnt = C.c_uint64()
    rc = load().orc_ffs_count_rows(C.byref(q._g), C.byref(plan._p), C.byref(d._g), int(vlabel_mode), int(threads),
                                   int(root_begin), int(root_end), C.byref(cnt), None, 0, None)
    if rc:
        raise RuntimeError(f"orc_ffs_count_rows failed ({rc})")
    return cnt.value


def row_degrees(d):
    """Out-degree of every CCSR row of an oracle Graph, in row order."""
    seg = d.arrays()["seg_val"]
    out, off = [], 0
    while off < len(seg):
        out.append(int(seg[off]))
        off += int(seg[off]) + 1
    return np.array(out, np.uint32)


def bt_count(qn, qsrc, qdst, qlab, qvl, dn, dsrc, dst, dlab, dvl, rel_bits=8, vlabel_mode=False, threads=1,
             max_rows=0):
    """Independent backtracking enumerator over directed edge lists."""
    def a(x, n):
        return np.ascontiguousarray(np.ones(n, np.uint32) if x is None else x, np.uint32)
    qsrc, qdst = a(qsrc, 0), a(qdst, 0)
    dsrc, dst = a(dsrc, 0), a(dst, 0)
    qlab, dlab = a(qlab, len(qsrc)), a(dlab, len(dsrc))
    qvl = np.zeros(qn, np.uint32) if qvl is None else np.ascontiguousarray(qvl, np.uint32)
    dvl = np.zeros(dn, np.uint32) if dvl is None else np.ascontiguousarray(dvl, np.uint32)
    cnt, nr = C.c_uint64(), C.c_uint64()
    rows = np.zeros((max(max_rows, 1), qn), np.uint32) if max_rows else None
    p = lambda x: x.ctypes.data_as(u32p)
    rc = load().orc_bt_count(qn, len(qsrc), p(qsrc), p(qdst), p(qlab), p(qvl), dn, len(dsrc), p(dsrc), p(dst),
                             p(dlab), p(dvl), rel_bits, int(vlabel_mode), int(threads), C.byref(cnt),
                             rows.ctypes.data_as(u32p) if rows is not None else None, int(max_rows), C.byref(nr))
    if rc:
        raise RuntimeError(f"orc_bt_count failed ({rc})")
    if max_rows:
        return cnt.value, rows[: nr.value]
    return cnt.value


def triangles(n, src, dst, threads=8):
    """Triangles of an undirected simple graph (edges src[i] < dst[i])."""
    s = np.ascontiguousarray(src, np.uint32)
    d = np.ascontiguousarray(dst, np.uint32)
    cnt = C.c_uint64()
    load().orc_triangles(int(n), len(s), s.ctypes.data_as(u32p), d.ctypes.data_as(u32p), int(threads), C.byref(cnt))
    return cnt.value


def triangle_label_hist(n, src, dst, vlabel, nl, threads=8):
    """hist[a, b, c]: embeddings of the triangle query with vertex labels
    (a, b, c) in an undirected simple graph (edges src[i] < dst[i])."""
    s = np.ascontiguousarray(src, np.uint32)
    d = np.ascontiguousarray(dst, np.uint32)
    vl = np.ascontiguousarray(vlabel, np.uint32)
    h = np.zeros(nl ** 3, np.uint64)
    cnt = C.c_uint64()
    rc = load().orc_triangle_label_hist(int(n), len(s), s.ctypes.data_as(u32p), d.ctypes.data_as(u32p),
                                        vl.ctypes.data_as(u32p), int(nl), int(threads), h.ctypes.data_as(u64p),
                                        C.byref(cnt))
    if rc:
        raise RuntimeError(f"orc_triangle_label_hist failed ({rc})")
    return h.reshape(nl, nl, nl)


def path3_label_counts(n, src, dst, vlabel, nl):
    """cnt[a, b, c]: embeddings of the 3-vertex path query x-y-z with vertex
    labels (a, b, c) in an undirected simple graph, by the closed form
    sum over y with label b of N_a(y) N_c(y) - [a == c] N_a(y), N_l(y) being
    y's neighbours with label l (x != z is the only injectivity constraint
    left: x, z are neighbours of y, so they differ from y)."""
    vl = np.asarray(vlabel, np.int64)
    s = np.asarray(src, np.int64)
    d = np.asarray(dst, np.int64)
    nb = np.zeros((n, nl), np.int64)          # N_l(y)
    np.add.at(nb, (s, vl[d]), 1)
    np.add.at(nb, (d, vl[s]), 1)
    out = np.zeros((nl, nl, nl), np.int64)
    for b in range(nl):
        rows = nb[vl == b]
        prod = rows.T @ rows                   # [a, c] = sum N_a N_c
        prod[np.diag_indices(nl)] -= rows.sum(axis=0)
        out[:, b, :] = prod
    return out


def ref_frontend_dump(path, plan=False):
    """Run the reference's own parser (+ planner) via oracle/_ref/ref_frontend.

    Returns (exit_code, dict or None)."""
    import tempfile
    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
        out = f.name
    try:
        r = subprocess.run([REF_FRONTEND, str(path), out] + (["plan"] if plan else []),
                           capture_output=True, timeout=120)
        if r.returncode != 0:
            return r.returncode, None
        w = np.fromfile(out, np.uint32)
    finally:
        os.unlink(out)
    i = 0

    def take(n):
        nonlocal i
        x = w[i:i + n]
        i += n
        return x
    count = int(take(1)[0])
    size = int(take(1)[0])
    res = {"count": count, "size": size, "segments": take(size), "vlocs": take(count), "inv": take(count)}
    ss = int(take(1)[0])
    res["staggers"] = take(ss)
    res["sinfo"] = take(2 * ss)
    if plan:
        mv = int(take(1)[0])
        res["max_valency"] = mv
        res["reqs"] = take(2 * mv * count)
        res["header"] = take(3 * count)
        res["mapping_after"] = take(count)
    return 0, res
