"""Seeded synthetic workloads (libgfsm_synth.so).

The reference is benchmarked on SNAP / RDF datasets that are not available
here; these generators stand in for them with the shapes of the five
workload configurations:

  1. Erdos-Renyi n=2,000, average degree 8, 4 uniform vertex labels, one
     5-vertex random-walk query with all induced edges;
  2. R-MAT(0.57, 0.19, 0.19, 0.05), 2^20 vertices, ~16M undirected edges,
     unlabelled; queries triangle, 4-cycle, 4-clique, house;
  3. Barabasi-Albert n=4M, m=4, 16 Zipf(1.0) vertex labels; 8-12 vertex
     random-walk queries, half spanning trees, half all induced edges;
  4. labelled R-MAT 2^22, average degree 16, 8 uniform vertex labels; 4,096
     random-walk queries of 3-12 vertices;
  5. 1,400 x 1,400 grid, 5% of edges removed, 2% random shortcuts, 4 uniform
     vertex labels; random-walk queries of 4-10 vertices.

Every graph is undirected (``src < dst`` per edge, no loops, no duplicates)
with edge label 1; ``directed()`` gives both directions as the matcher and the
reference's text format expect.
"""
import ctypes as C
import os

import numpy as np

from . import _lib

u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)

_synth = None


def _load():
    global _synth
    if _synth is None:
        if not os.path.exists(_lib.SYNTH_PATH):
            raise ImportError(f"libgfsm_synth.so not built at {_lib.SYNTH_PATH} (run: make -C gfsm_b200)")
        s = C.CDLL(_lib.SYNTH_PATH)
        out_arr = C.POINTER(u32p)
        s.syn_er.argtypes = [C.c_uint32, C.c_double, C.c_uint64, u64p, out_arr, out_arr]
        s.syn_rmat.argtypes = [C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_uint64, u64p,
                               out_arr, out_arr]
        s.syn_ba.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, u64p, out_arr, out_arr]
        s.syn_grid.argtypes = [C.c_uint32, C.c_double, C.c_double, C.c_uint64, u64p, out_arr, out_arr]
        s.syn_vlabels.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_uint64, u32p]
        s.syn_csr.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, u64p, u32p]
        s.syn_rw_query.argtypes = [C.c_uint32, u64p, u32p, C.c_uint32, C.c_int, C.c_uint64, u32p,
                                   C.POINTER(C.c_uint32), u32p, u32p]
        s.syn_write_text.argtypes = [C.c_char_p, C.c_uint32, u32p, C.c_uint64, u32p, u32p, u32p]
        s.syn_free.argtypes = [C.c_void_p]
        for f in ("syn_er", "syn_rmat", "syn_ba", "syn_grid", "syn_vlabels", "syn_csr", "syn_rw_query",
                  "syn_write_text"):
            getattr(s, f).restype = C.c_int
        _synth = s
    return _synth


def _take(m, ps, pd):
    s = _load()
    src = np.ctypeslib.as_array(ps, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
    dst = np.ctypeslib.as_array(pd, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
    s.syn_free(C.cast(ps, C.c_void_p))
    s.syn_free(C.cast(pd, C.c_void_p))
    return src, dst


def _gen(fn, *args):
    m = C.c_uint64()
    ps, pd = u32p(), u32p()
    rc = fn(*args, C.byref(m), C.byref(ps), C.byref(pd))
    if rc:
        raise RuntimeError(f"generator failed ({rc})")
    return _take(m.value, ps, pd)


class UGraph:
    """Undirected graph: n vertices, edges (src[i] < dst[i]), vertex labels."""

    def __init__(self, n, src, dst, vlabel=None):
        self.n = int(n)
        self.src = np.asarray(src, np.uint32)
        self.dst = np.asarray(dst, np.uint32)
        self.vlabel = np.zeros(self.n, np.uint32) if vlabel is None else np.asarray(vlabel, np.uint32)
        self._csr = None

    @property
    def m(self):
        return len(self.src)

    def directed(self):
        """Both directions: (src, dst) of length 2m."""
        return np.concatenate([self.src, self.dst]), np.concatenate([self.dst, self.src])

    def csr(self):
        if self._csr is None:
            rowptr = np.zeros(self.n + 1, np.uint64)
            adj = np.zeros(max(2 * self.m, 1), np.uint32)
            _load().syn_csr(self.n, self.m, self.src.ctypes.data_as(u32p), self.dst.ctypes.data_as(u32p),
                            rowptr.ctypes.data_as(u64p), adj.ctypes.data_as(u32p))
            # rows sorted by neighbour id
            for_sort = np.repeat(np.arange(self.n, dtype=np.uint64), np.diff(rowptr).astype(np.int64))
            order = np.lexsort((adj[: 2 * self.m], for_sort))
            adj = adj[: 2 * self.m][order]
            self._csr = (rowptr, adj)
        return self._csr

    def write_text(self, path, elabel=None):
        el = None if elabel is None else np.ascontiguousarray(elabel, np.uint32)
        rc = _load().syn_write_text(str(path).encode(), self.n, self.vlabel.ctypes.data_as(u32p), self.m,
                                    self.src.ctypes.data_as(u32p), self.dst.ctypes.data_as(u32p),
                                    None if el is None else el.ctypes.data_as(u32p))
        if rc:
            raise OSError(f"cannot write {path}")


def er(n, avg_deg, seed=0):
    return UGraph(n, *_gen(_load().syn_er, n, float(avg_deg), seed))


def rmat(scale, undirected_edges, a=0.57, b=0.19, c=0.19, seed=0):
    return UGraph(1 << scale, *_gen(_load().syn_rmat, scale, int(undirected_edges), a, b, c, seed))


def ba(n, m, seed=0):
    return UGraph(n, *_gen(_load().syn_ba, n, m, seed))


def grid(side, remove=0.05, shortcuts=0.02, seed=0):
    return UGraph(side * side, *_gen(_load().syn_grid, side, float(remove), float(shortcuts), seed))


def vlabels(n, nlabels, zipf_s=0.0, seed=0):
    out = np.zeros(max(n, 1), np.uint32)
    _load().syn_vlabels(n, nlabels, float(zipf_s), seed, out.ctypes.data_as(u32p))
    return out[:n]


def rw_query(g, k, tree=False, seed=1):
    """Random-walk query of k vertices from UGraph g.

    Returns a UGraph whose vertex i is the i-th visited data vertex (labels
    copied), plus the visited data vertex ids."""
    rowptr, adj = g.csr()
    visited = np.zeros(k, np.uint32)
    qs = np.zeros(k * k, np.uint32)
    qd = np.zeros(k * k, np.uint32)
    qm = C.c_uint32()
    rc = _load().syn_rw_query(g.n, rowptr.ctypes.data_as(u64p), adj.ctypes.data_as(u32p), k, 1 if tree else 0,
                              seed, visited.ctypes.data_as(u32p), C.byref(qm), qs.ctypes.data_as(u32p),
                              qd.ctypes.data_as(u32p))
    if rc:
        raise RuntimeError("random walk did not reach k vertices")
    m = qm.value
    return UGraph(k, qs[:m], qd[:m], g.vlabel[visited]), visited


# Fixed query shapes (undirected edge lists over 0..k-1).
SHAPES = {
    "triangle": (3, [(0, 1), (1, 2), (0, 2)]),
    "4-cycle": (4, [(0, 1), (1, 2), (2, 3), (0, 3)]),
    "4-clique": (4, [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]),
    "house": (5, [(0, 1), (1, 2), (2, 3), (3, 0), (0, 4), (1, 4)]),
    "path3": (3, [(0, 1), (1, 2)]),
    "star4": (5, [(0, 1), (0, 2), (0, 3), (0, 4)]),
}


def shape(name):
    k, e = SHAPES[name]
    a = np.array(e, np.uint32).reshape(-1, 2)
    return UGraph(k, np.minimum(a[:, 0], a[:, 1]), np.maximum(a[:, 0], a[:, 1]))


# ---------------------------------------------------------------------------
# The five workload configurations
# ---------------------------------------------------------------------------
def config1():
    g = er(2000, 8.0, seed=0)
    g.vlabel = vlabels(g.n, 4, 0.0, seed=100)
    q, _ = rw_query(g, 5, tree=False, seed=1)
    return g, [q]


def config2(scale=20, undirected_edges=16 * (1 << 20) // 1):
    g = rmat(scale, undirected_edges, seed=0)
    return g, [shape(s) for s in ("triangle", "4-cycle", "4-clique", "house")]


def config3(n=4_000_000, nq=8, seed=0):
    g = ba(n, 4, seed=seed)
    g.vlabel = vlabels(g.n, 16, 1.0, seed=100 + seed)
    qs = []
    for i in range(nq):
        k = 8 + (i % 5)
        q, _ = rw_query(g, k, tree=(i % 2 == 0), seed=1 + i)
        qs.append(q)
    return g, qs


def config4(scale=22, avg_deg=16, nq=4096, seed=0, kmin=3, kmax=12):
    n = 1 << scale
    g = rmat(scale, n * avg_deg // 2, seed=seed)
    g.vlabel = vlabels(g.n, 8, 0.0, seed=100 + seed)
    rng = np.random.default_rng(seed + 7)
    qs = []
    for i in range(nq):
        k = int(rng.integers(kmin, kmax + 1))
        q, _ = rw_query(g, k, tree=False, seed=1 + i)
        qs.append(q)
    return g, qs


def config5(side=1400, nq=1000, seed=0, kmin=4, kmax=10):
    g = grid(side, 0.05, 0.02, seed=seed)
    g.vlabel = vlabels(g.n, 4, 0.0, seed=100 + seed)
    rng = np.random.default_rng(seed + 11)
    qs = []
    for i in range(nq):
        k = int(rng.integers(kmin, kmax + 1))
        q, _ = rw_query(g, k, tree=False, seed=1 + i)
        qs.append(q)
    return g, qs
