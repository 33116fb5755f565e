"""ctypes binding of libgfsm.so (declared in include/gfsm.h).

The library is built in-tree (``make -C gfsm_b200``); importing this module
without it raises, there is no fallback path.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgfsm.so")
SYNTH_PATH = os.path.join(_HERE, "libgfsm_synth.so")

u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
u8p = C.POINTER(C.c_uint8)
vp = C.c_void_p

# Every function declared in include/gfsm.h: name -> (restype, argtypes).
SIGNATURES = {
    "gfsm_limits_default": (None, [vp]),
    "gfsm_init": (C.c_int, [C.POINTER(vp), vp, C.c_int]),
    "gfsm_destroy": (None, [vp]),
    "gfsm_status_str": (C.c_char_p, [C.c_int]),
    "gfsm_last_error": (C.c_char_p, [vp]),
    "gfsm_graph_load_text": (C.c_int, [vp, C.c_char_p, C.POINTER(vp)]),
    "gfsm_graph_load_buffer": (C.c_int, [vp, C.c_char_p, C.c_uint64, C.POINTER(vp)]),
    "gfsm_graph_from_edges": (C.c_int, [vp, C.c_uint32, C.c_uint64, u32p, u32p, u32p, u32p, C.POINTER(vp)]),
    "gfsm_graph_to_device": (C.c_int, [vp, vp]),
    "gfsm_graph_info_get": (C.c_int, [vp, vp]),
    "gfsm_graph_download": (C.c_int, [vp, vp, u32p, u32p, u8p, u32p]),
    "gfsm_graph_destroy": (None, [vp]),
    "gfsm_query_prepare": (C.c_int, [vp, vp, C.POINTER(vp)]),
    "gfsm_query_prepare_batch": (C.c_int, [vp, C.c_int, u32p, u64p, u32p, u32p, u32p, u32p, vp, C.POINTER(vp),
                                           C.POINTER(C.c_int)]),
    "gfsm_query_prepare_for": (C.c_int, [vp, vp, vp, C.POINTER(vp)]),
    "gfsm_plan_info": (C.c_int, [vp, u32p, u32p]),
    "gfsm_plan_symmetry": (C.c_int, [vp, u64p, u32p, u32p]),
    "gfsm_plan_destroy_array": (None, [vp, C.c_int]),
    "gfsm_plan_tables": (C.c_int, [vp, u32p, u32p, u32p, u32p, u32p]),
    "gfsm_plan_columns": (C.c_int, [vp, u32p]),
    "gfsm_plan_destroy": (None, [vp]),
    "gfsm_match_count": (C.c_int, [vp, vp, vp, u64p, vp]),
    "gfsm_match_mappings": (C.c_int, [vp, vp, vp, u32p, C.c_uint64, u64p, u64p, vp]),
    "gfsm_batch_count": (C.c_int, [vp, C.POINTER(vp), C.c_int, vp, u64p, vp]),
    "gfsm_match_count_noalloc": (C.c_int, [vp, vp, vp, u64p]),
    "gfsm_partition_rows": (C.c_int, [u32p, C.c_uint32, C.c_uint32, C.c_uint32, u64p]),
    "gfsm_root_partition": (C.c_int, [vp, vp, vp, C.c_uint32, u32p, u64p]),
    "gfsm_batch_count_part": (C.c_int, [vp, C.POINTER(vp), C.c_int, vp, C.c_uint32, C.c_uint32, u64p, vp]),
    "gfsm_predict_frontier_bytes": (C.c_int, [vp, vp, vp, C.POINTER(C.c_double)]),
    "gfsm_serve_start": (C.c_int, [vp, vp, vp, C.POINTER(vp)]),
    "gfsm_serve_submit": (C.c_int, [vp, vp, C.c_uint64]),
    "gfsm_serve_poll": (C.c_int, [vp, vp, C.c_int, C.POINTER(C.c_int)]),
    "gfsm_serve_drain": (C.c_int, [vp, C.c_double]),
    "gfsm_serve_stop": (C.c_int, [vp]),
}


class Limits(C.Structure):
    _fields_ = [
        ("ccsr_rel_size", C.c_uint32),
        ("max_soln_size", C.c_uint64),
        ("max_scan_size", C.c_uint64),
        ("mem_limit", C.c_uint64),
        ("upper_mem_limit", C.c_uint64),
        ("vertex_labels", C.c_int32),
        ("degree_filter", C.c_int32),
        ("max_candidates", C.c_uint64),
    ]


class GraphInfo(C.Structure):
    _fields_ = [
        ("n", C.c_uint32),
        ("m", C.c_uint64),
        ("rows", C.c_uint32),
        ("max_degree", C.c_uint32),
        ("symmetric", C.c_int32),
        ("multi_edges", C.c_int32),
        ("n_edge_labels", C.c_int32),
        ("on_device", C.c_int32),
        ("device_bytes", C.c_uint64),
        ("build_alloc_ms", C.c_double),
        ("build_h2d_ms", C.c_double),
        ("build_kernel_ms", C.c_double),
        ("build_d2h_ms", C.c_double),
        ("build_wall_ms", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("count", C.c_uint64),
        ("expansions", C.c_uint64),
        ("candidates", C.c_uint64),
        ("alg_bytes", C.c_uint64),
        ("steps", C.c_uint64),
        ("retries", C.c_uint64),
        ("peak_frontier_bytes", C.c_uint64),
        ("kernel_ms", C.c_double),
        ("device_ms", C.c_double),
        ("wall_ms", C.c_double),
        ("h2d_bytes", C.c_uint64),
        ("d2h_bytes", C.c_uint64),
        ("tile_variant", C.c_int32),
        ("launches", C.c_uint32),
        ("driver", C.c_int32),
        ("graph_error", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Result(C.Structure):
    _fields_ = [
        ("req_id", C.c_uint64),
        ("count", C.c_uint64),
        ("status", C.c_int32),
        ("submit_ms", C.c_double),
        ("start_ms", C.c_double),
        ("done_ms", C.c_double),
    ]


class ServeConfig(C.Structure):
    _fields_ = [
        ("slots", C.c_int32),
        ("max_batch", C.c_int32),
        ("queue_capacity", C.c_int32),
        ("frontier_bytes", C.c_uint64),
    ]


_lib = None


def load():
    """Load libgfsm.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libgfsm.so not built at {LIB_PATH} (run: make -C gfsm_b200)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
