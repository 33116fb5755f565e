"""gfsm_b200 -- B200-native GFSM subgraph matching.

Python mirror of the reference's host interface (HnGPU.cuh:60-80
``HnSetup::preinit / solve / preProcessQuery``, HnHelper.cuh:283 ``fileParse``)
over the C ABI of ``libgfsm.so`` (include/gfsm.h).  All matching runs in the
library's CUDA kernels; there is no CPU path in this package.

    >>> ctx = GFSM()                         # HnSetup::preinit
    >>> q = ctx.file_parse("query.g")         # fileParse
    >>> d = ctx.file_parse("data.g")
    >>> ctx.solve(q, d)                       # HnSetup::solve -> Function Count
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import GraphInfo, Limits, Result, ServeConfig, Stats

__all__ = ["GFSM", "Graph", "Plan", "Server", "GFSMError", "Limits", "Stats", "default_limits"]


class GFSMError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = int(status)
        text = _lib.load().gfsm_status_str(self.status).decode()
        super().__init__(f"GFSM status {self.status} ({text}){': ' + msg if msg else ''}")


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(_lib.u32p)


def default_limits(**overrides):
    """Environment.h knobs with GFSM_* environment overrides, then kwargs."""
    lib = _lib.load()
    lim = Limits()
    lib.gfsm_limits_default(C.byref(lim))
    for k, v in overrides.items():
        if not hasattr(lim, k):
            raise KeyError(k)
        setattr(lim, k, v)
    return lim


class Graph:
    """A parsed graph; built on the device on first use as a data graph."""

    def __init__(self, ctx, handle):
        self._ctx = ctx
        self._h = C.c_void_p(handle)

    @property
    def handle(self):
        return self._h

    def to_device(self):
        self._ctx._check(self._ctx._lib.gfsm_graph_to_device(self._ctx._h, self._h))
        return self

    def info(self):
        inf = GraphInfo()
        self._ctx._check(self._ctx._lib.gfsm_graph_info_get(self._h, C.byref(inf)))
        return {k: getattr(inf, k) for k, _ in inf._fields_}

    def download(self):
        """Device CCSR in the reference's row order: rowptr, adj (row ids), elab, order."""
        inf = self.info()
        if not inf["on_device"]:
            self.to_device()
            inf = self.info()
        n, m = inf["n"], inf["m"]
        rowptr = np.zeros(n + 1, np.uint32)
        adj = np.zeros(max(m, 1), np.uint32)
        elab = np.zeros(max(m, 1), np.uint8)
        order = np.zeros(max(n, 1), np.uint32)
        self._ctx._check(self._ctx._lib.gfsm_graph_download(
            self._ctx._h, self._h, rowptr.ctypes.data_as(_lib.u32p), adj.ctypes.data_as(_lib.u32p),
            elab.ctypes.data_as(_lib.u8p), order.ctypes.data_as(_lib.u32p)))
        return rowptr, adj[:m], elab[:m], order[:n]

    def close(self):
        if self._h:
            self._ctx._lib.gfsm_graph_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """The reference's matching order + requirement table for one query."""

    def __init__(self, ctx, handle):
        self._ctx = ctx
        self._h = C.c_void_p(handle)
        self._owned = True  # False for a view into a PlanBatch (the batch destroys it)

    @property
    def handle(self):
        return self._h

    def tables(self):
        lib = self._ctx._lib
        k, mv = C.c_uint32(), C.c_uint32()
        self._ctx._check(lib.gfsm_plan_tables(self._h, C.byref(k), C.byref(mv), None, None, None))
        k, mv = k.value, mv.value
        order = np.zeros(k, np.uint32)
        header = np.zeros(3 * k, np.uint32)
        reqs = np.zeros(max(2 * mv * k, 1), np.uint32)
        self._ctx._check(lib.gfsm_plan_tables(self._h, None, None, order.ctypes.data_as(_lib.u32p),
                                              header.ctypes.data_as(_lib.u32p), reqs.ctypes.data_as(_lib.u32p)))
        return {"k": k, "max_valency": mv, "order": order, "header": header, "reqs": reqs[: 2 * mv * k]}

    def symmetry(self):
        """(|Aut(Q)|, [(a, b), ...]): count embeddings with f(a) < f(b) for
        every pair, times |Aut(Q)|, to get the full count."""
        lib = self._ctx._lib
        aut, n = C.c_uint64(), C.c_uint32()
        self._ctx._check(lib.gfsm_plan_symmetry(self._h, C.byref(aut), C.byref(n), None))
        cond = np.zeros(max(2 * n.value, 1), np.uint32)
        self._ctx._check(lib.gfsm_plan_symmetry(self._h, None, None, cond.ctypes.data_as(_lib.u32p)))
        return aut.value, [(int(cond[2 * i]), int(cond[2 * i + 1])) for i in range(n.value)]

    def info(self):
        """{"planner": 0 reference order / 1 data-aware, "order_invariant": bool}"""
        pl, inv = C.c_uint32(), C.c_uint32()
        self._ctx._check(self._ctx._lib.gfsm_plan_info(self._h, C.byref(pl), C.byref(inv)))
        return {"planner": pl.value, "order_invariant": bool(inv.value)}

    def columns(self):
        k = self.tables()["k"]
        cols = np.zeros(k, np.uint32)
        self._ctx._check(self._ctx._lib.gfsm_plan_columns(self._h, cols.ctypes.data_as(_lib.u32p)))
        return cols

    def close(self):
        if self._h and self._owned:
            self._ctx._lib.gfsm_plan_destroy(self._h)
        self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PlanBatch:
    """The plans of a batch as one object: the C handles in one array, passed
    to gfsm_batch_count as they are.  Indexing gives Plan views (owned by the
    batch); close() destroys every plan."""

    def __init__(self, ctx, arr, n):
        self._ctx = ctx
        self._arr = arr
        self._n = n

    def __len__(self):
        return self._n

    def __getitem__(self, i):
        if not -self._n <= i < self._n:
            raise IndexError(i)
        p = Plan.__new__(Plan)
        p._ctx = self._ctx
        p._h = C.c_void_p(self._arr[i % self._n])
        p._owned = False
        return p

    def __iter__(self):
        return (self[i] for i in range(self._n))

    def close(self):
        if self._arr is not None:
            self._ctx._lib.gfsm_plan_destroy_array(self._arr, self._n)
            self._arr = None
            self._n = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Served form: continuous batching over a resident data graph."""

    def __init__(self, ctx, data, slots=2, max_batch=256, queue_capacity=65536, frontier_bytes=0):
        self._ctx = ctx
        self._data = data
        cfg = ServeConfig(slots, max_batch, queue_capacity, frontier_bytes)
        h = C.c_void_p()
        ctx._check(ctx._lib.gfsm_serve_start(ctx._h, data.handle, C.byref(cfg), C.byref(h)))
        self._h = h

    def submit(self, plan, req_id):
        rc = self._ctx._lib.gfsm_serve_submit(self._h, plan.handle, int(req_id))
        if rc:
            raise GFSMError(rc)

    def poll(self, max_results=4096):
        buf = (Result * max_results)()
        n = C.c_int()
        self._ctx._check(self._ctx._lib.gfsm_serve_poll(self._h, buf, max_results, C.byref(n)))
        return [{k: getattr(buf[i], k) for k, _ in Result._fields_} for i in range(n.value)]

    def drain(self, timeout_ms=0.0):
        self._ctx._check(self._ctx._lib.gfsm_serve_drain(self._h, float(timeout_ms)))

    def stop(self):
        if self._h:
            self._ctx._check(self._ctx._lib.gfsm_serve_stop(self._h))
            self._h = None


def partition_rows(rowptr, lo, hi, nparts):
    """gfsm_partition_rows: degree-balanced cut of CCSR rows [lo, hi) into
    nparts consecutive parts (offsets into the window; host only)."""
    rp = np.ascontiguousarray(rowptr, np.uint32)
    b = np.zeros(nparts + 1, np.uint64)
    rc = _lib.load().gfsm_partition_rows(rp.ctypes.data_as(_lib.u32p), int(lo), int(hi), int(nparts),
                                         b.ctypes.data_as(_lib.u64p))
    if rc:
        raise GFSMError(rc)
    return b


class GFSM:
    """One device context (HnSetup::preinit, HnGPU.cu:847-862)."""

    def __init__(self, limits=None, device=0, **overrides):
        self._lib = _lib.load()
        lim = limits if limits is not None else default_limits(**overrides)
        h = C.c_void_p()
        rc = self._lib.gfsm_init(C.byref(h), C.byref(lim), int(device))
        if rc:
            raise GFSMError(rc)
        self._h = h
        self.limits = lim

    def _check(self, rc):
        if rc:
            raise GFSMError(rc, self._lib.gfsm_last_error(self._h).decode(errors="replace"))

    # -- graphs ---------------------------------------------------------------
    def file_parse(self, path):
        """fileParse (HnHelper.cuh:283): text graph -> Graph."""
        h = C.c_void_p()
        self._check(self._lib.gfsm_graph_load_text(self._h, str(path).encode(), C.byref(h)))
        return Graph(self, h.value)

    def parse_text(self, text):
        if isinstance(text, str):
            text = text.encode()
        h = C.c_void_p()
        self._check(self._lib.gfsm_graph_load_buffer(self._h, text, len(text), C.byref(h)))
        return Graph(self, h.value)

    def graph_from_edges(self, n, src, dst, elabel=None, vlabel=None):
        """Directed edge list (give both directions for undirected graphs)."""
        s, sp = _u32(src)
        d, dp = _u32(dst)
        el, elp = (None, None) if elabel is None else _u32(elabel)
        vl, vlp = (None, None) if vlabel is None else _u32(vlabel)
        h = C.c_void_p()
        self._check(self._lib.gfsm_graph_from_edges(self._h, int(n), len(s), sp, dp, elp, vlp, C.byref(h)))
        return Graph(self, h.value)

    # -- planning -------------------------------------------------------------
    def pre_process_query(self, query):
        """HnSetup::preProcessQuery (HnGPU.cu:749): matching order + requirements."""
        h = C.c_void_p()
        self._check(self._lib.gfsm_query_prepare(self._h, query.handle, C.byref(h)))
        return Plan(self, h.value)

    def plan_for(self, query, data):
        """A plan whose matching order is chosen for `data` where the count
        cannot depend on the order (gfsm_query_prepare_for)."""
        h = C.c_void_p()
        self._check(self._lib.gfsm_query_prepare_for(self._h, query.handle, data.handle, C.byref(h)))
        return Plan(self, h.value)

    def prepare_queries(self, queries, data=None):
        """Plans for many queries in one call (gfsm_query_prepare_batch).

        queries: iterable of (n, src, dst, elabel or None, vlabel or None),
        directed edge lists with ids local to each query.  The labels must be
        given for all queries or for none.  With `data`, each plan is
        gfsm_query_prepare_for's (data-aware order where it is allowed).
        Returns a PlanBatch."""
        queries = list(queries)
        nq = len(queries)
        nv = np.fromiter((int(q[0]) for q in queries), np.uint32, nq)
        ne = np.fromiter((len(q[1]) for q in queries), np.uint64, nq)
        eoff = np.zeros(nq + 1, np.uint64)
        np.cumsum(ne, out=eoff[1:])
        cat = lambda i: np.concatenate([np.asarray(q[i], np.uint32) for q in queries]) \
            if nq and queries[0][i] is not None else None
        return self.prepare_queries_flat(nv, eoff, cat(1), cat(2), cat(3), cat(4), data)

    def prepare_queries_flat(self, nv, eoff, src, dst, elabel=None, vlabel=None, data=None):
        """prepare_queries over a batch already in flat arrays: query i has
        nv[i] vertices and the edges eoff[i]:eoff[i+1] of src/dst/elabel; its
        vertex labels are the next nv[i] entries of vlabel."""
        nq = len(nv)
        out = (C.c_void_p * max(nq, 1))()
        if nq == 0:
            return PlanBatch(self, out, 0)
        u32 = lambda a: None if a is None else np.ascontiguousarray(a, np.uint32)
        nv, src, dst, elabel, vlabel = u32(nv), u32(src), u32(dst), u32(elabel), u32(vlabel)
        eoff = np.ascontiguousarray(eoff, np.uint64)
        ptr = lambda a: a.ctypes.data_as(_lib.u32p) if a is not None and len(a) else None
        failed = C.c_int(-1)
        self._check(self._lib.gfsm_query_prepare_batch(
            self._h, nq, nv.ctypes.data_as(_lib.u32p), eoff.ctypes.data_as(_lib.u64p), ptr(src), ptr(dst),
            ptr(elabel), ptr(vlabel), data.handle if data is not None else None, out, C.byref(failed)))
        return PlanBatch(self, out, nq)

    # -- matching -------------------------------------------------------------
    def match_count(self, plan, data):
        cnt = C.c_uint64()
        st = Stats()
        self._check(self._lib.gfsm_match_count(self._h, plan.handle, data.handle, C.byref(cnt), C.byref(st)))
        return cnt.value, st.as_dict()

    def solve(self, query, data):
        """HnSetup::solve (HnGPU.cu:710): the embedding count ("Function Count")."""
        plan = self.pre_process_query(query)
        try:
            return self.match_count(plan, data)[0]
        finally:
            plan.close()

    def match_mappings(self, plan, data, max_rows=1 << 20):
        """Full mappings as original vertex ids, column c = query vertex c."""
        k = plan.tables()["k"]
        rows = np.zeros((max(max_rows, 1), k), np.uint32)
        nr, cnt = C.c_uint64(), C.c_uint64()
        st = Stats()
        self._check(self._lib.gfsm_match_mappings(self._h, plan.handle, data.handle,
                                                  rows.ctypes.data_as(_lib.u32p), int(max_rows),
                                                  C.byref(nr), C.byref(cnt), C.byref(st)))
        return rows[: nr.value], cnt.value

    def batch_count(self, plans, data):
        if isinstance(plans, PlanBatch):
            arr = plans._arr
        else:
            arr = (C.c_void_p * max(len(plans), 1))(*[p.handle.value for p in plans])
        counts = np.zeros(max(len(plans), 1), np.uint64)
        st = Stats()
        self._check(self._lib.gfsm_batch_count(self._h, arr, len(plans), data.handle,
                                               counts.ctypes.data_as(_lib.u64p), C.byref(st)))
        return counts[: len(plans)], st.as_dict()

    def batch_count_part(self, plans, data, part, nparts):
        """batch_count over part `part` of nparts of every query's root window
        (gfsm_batch_count_part): the parts' counts add up to batch_count's."""
        if isinstance(plans, PlanBatch):
            arr = plans._arr
        else:
            arr = (C.c_void_p * max(len(plans), 1))(*[p.handle.value for p in plans])
        counts = np.zeros(max(len(plans), 1), np.uint64)
        st = Stats()
        self._check(self._lib.gfsm_batch_count_part(self._h, arr, len(plans), data.handle, int(part), int(nparts),
                                                    counts.ctypes.data_as(_lib.u64p), C.byref(st)))
        return counts[: len(plans)], st.as_dict()

    def root_partition(self, plan, data, nparts):
        """(window_lo, bounds): the degree-balanced cut of plan's root window."""
        b = np.zeros(nparts + 1, np.uint64)
        lo = C.c_uint32()
        self._check(self._lib.gfsm_root_partition(self._h, plan.handle, data.handle, int(nparts), C.byref(lo),
                                                  b.ctypes.data_as(_lib.u64p)))
        return lo.value, b

    def predict_frontier_bytes(self, plan, data):
        """The served form's admission estimate of plan's peak frontier bytes."""
        b = C.c_double()
        self._check(self._lib.gfsm_predict_frontier_bytes(self._h, plan.handle, data.handle, C.byref(b)))
        return b.value

    def serve(self, data, **kw):
        return Server(self, data, **kw)

    def close(self):
        if self._h:
            self._lib.gfsm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
