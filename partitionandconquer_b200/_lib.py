"""ctypes binding of libpc.so (the C ABI declared in include/pc.h).

The library is loaded from this package directory.  There is no fallback:
if libpc.so is missing the import fails with instructions, and every compute
call raises PCError when the library reports an error (including the absence
of a CUDA device).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libpc.so"

PC_OK = 0
STATUS = {
    0: "PC_OK",
    1: "PC_ERR_INVALID_INPUT",
    2: "PC_ERR_OOM",
    3: "PC_ERR_CUDA",
    4: "PC_ERR_TIMEOUT",
    5: "PC_ERR_NO_DEVICE",
    6: "PC_ERR_UNSUPPORTED",
}

METHOD_MERGE = 0
METHOD_GALLOPING = 1
VARIANT_AUTO = -1
VARIANT_HEURISTIC = -2
VARIANTS = {
    "bitmap_warp": 0,
    "bitmap_group8": 1,
    "bitmap_lane": 2,
    "hash_warp": 3,
    "merge_lane": 4,
    "gallop_lane": 5,
    "matrix": 6,
}
NUM_VARIANTS = 7
SELECTOR_FEATURES = 10
MLP_IN, MLP_HIDDEN, MLP_OUT = 12, 64, NUM_VARIANTS


class PCError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class TCStats(C.Structure):
    _fields_ = [
        ("kernel_ms", C.c_double),
        ("launches", C.c_uint64),
        ("scan_bound", C.c_uint64),
        ("partitions", C.c_int32),
        ("variant_hist", C.c_int32 * NUM_VARIANTS),
        ("selector", C.c_int32),
    ]


class BatchStats(C.Structure):
    _fields_ = [
        ("ms", C.c_double),
        ("items", C.c_uint32),
        ("threads", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("order", C.c_int32),
    ]


P = C.c_void_p
i32, u32, i64, u64, f32, f64 = C.c_int32, C.c_uint32, C.c_int64, C.c_uint64, C.c_float, C.c_double
PP = C.POINTER(C.c_void_p)

# name -> (restype, argtypes)
_SIG = {
    "pc_last_error": (C.c_char_p, []),
    "pc_version": (C.c_char_p, []),
    "pc_device_count": (i32, []),
    "pc_set_device": (i32, [i32]),
    "pc_launch_count": (u64, []),
    "pc_host_register": (i32, [P, C.c_size_t]),
    "pc_release_cached_memory": (i32, []),
    "pc_selftest_grid_barrier": (i32, [i32, i32, i32, u32, P]),
    "pc_host_unregister": (i32, [P]),
    "pc_graph_create": (i32, [P, P, P, u64, u64, u32, PP]),
    "pc_graph_destroy": (i32, [P]),
    "pc_graph_info": (i32, [P, P, P, P]),
    "pc_graph_stream": (P, [P]),
    "pc_greedy_partition": (i32, [P, i32, u64, P]),
    "pc_host_greedy_partition": (i32, [P, P, u64, i32, u64, P]),
    "pc_friend_triangle": (i32, [P, i32, P, u64, P]),
    "pc_square_count": (i32, [P, P]),
    "pc_graph_from_edges": (i32, [P, P, u64, u64, u32, P, PP]),
    "pc_graph_rmat": (i32, [u32, u32, u64, u32, PP]),
    "pc_graph_er": (i32, [u32, u64, u64, u32, PP]),
    "pc_graph_add_weights": (i32, [P, u64, i32]),
    "pc_graph_download": (i32, [P, P, P, P]),
    "pc_partition": (i32, [P, P, PP]),
    "pc_pgraph_destroy": (i32, [P]),
    "pc_pgraph_info": (i32, [P, P, P, P]),
    "pc_pgraph_reorder": (i32, [P]),
    "pc_pgraph_vertex_map": (i32, [P, P]),
    "pc_pgraph_layout": (i32, [P, P, P, P]),
    "pc_pgraph_evaluate": (i32, [P, P, P, P]),
    "pc_tc": (i32, [P, i32, P]),
    "pc_tc_ex": (i32, [P, i32, i32, P, P]),
    "pc_lcc": (i32, [P, i32, P]),
    "pc_jaccard_edges": (i32, [P, P]),
    "pc_jaccard_queries": (i32, [P, P, i32, P]),
    "pc_batch_count_pairs": (i32, [P, P, u64, P]),
    "pc_batch_count_sets": (i32, [P, P, P, u64, P]),
    "pc_bfs": (i32, [P, i32, P]),
    "pc_sssp": (i32, [P, i32, P]),
    "pc_sssp_ex": (i32, [P, i32, i32, i32, P]),
    "pc_pagerank": (i32, [P, f32, i32, P, P]),
    "pc_pagerank_f64": (i32, [P, f64, i32, P, P]),
    "pc_kcore": (i32, [P, P, P]),
    "pc_mis": (i32, [P, P]),
    "pc_mis_hashed": (i32, [P, u64, P]),
    "pc_cdlp": (i32, [P, i32, P]),
    "pc_tc_count_noalloc": (i32, [P, P, u64, u64, P, P]),
    "pc_batch_create": (i32, [P, P, u64, u64, P, u32, PP]),
    "pc_batch_destroy": (i32, [P]),
    "pc_batch_run": (i32, [P, u32, P, P, P, P]),
    "pc_batch_set_schedule": (i32, [P, i32, i32, i32]),
    "pc_batch_autotune": (i32, [P, u32, P]),
    "pc_synth_rmat_batch": (i32, [u32, u32, u32, u32, u32, u64, PP, P]),
    "pc_tc_units": (i32, [P, P]),
    "pc_tc_unit_features": (i32, [P, P, i32]),
    "pc_tc_plan": (i32, [P, i32, P, i32]),
    "pc_tc_time_unit": (i32, [P, i32, i32, P, P]),
    "pc_selector_collect": (i32, [P, i32, i32, P]),
    "pc_selector_collect_insitu": (i32, [P, i32, P]),
    "pc_selector_judge": (i32, [P, P]),
    "pc_selector_num_samples": (i32, []),
    "pc_selector_get_samples": (i32, [P, P, P, i32]),
    "pc_selector_add_samples": (i32, [P, P, P, i32]),
    "pc_selector_train": (i32, [i32, f32, u64, P]),
    "pc_selector_predict": (i32, [P, i32, P]),
    "pc_selector_autotune": (i32, [P]),
    "pc_selector_autotune_measured": (i32, [P, i32, i32, i32, P, P]),
    "pc_selector_get_heuristic": (i32, [P]),
    "pc_selector_set_heuristic": (i32, [P]),
    "pc_selector_clear": (i32, []),
    "pc_selector_trained": (i32, []),
    "pc_selector_enable": (i32, [i32]),
    "pc_selector_save": (i32, [C.c_char_p]),
    "pc_selector_load": (i32, [C.c_char_p]),
    "pc_mlp_num_params": (i32, []),
    "pc_mlp_forward": (i32, [P, P, i32, P]),
    "pc_mlp_loss_grad": (i32, [P, P, P, P, i32, P, P]),
    "pc_mlp_loss_grad_weighted": (i32, [P, P, P, P, P, i32, P, P]),
    "pc_mlp_train_steps": (i32, [P, P, P, P, i32, i32, f32, P]),
    "pc_synth_rmat": (i32, [u32, u32, u64, i32, PP]),
    "pc_synth_er": (i32, [u32, u64, u64, i32, PP]),
    "pc_synth_chung_lu": (i32, [u32, u64, f64, u64, u64, i32, PP]),
    "pc_synth_add_weights": (i32, [P, u64, i32]),
    "pc_host_csr_arrays": (i32, [P, P, P, P, P, P]),
    "pc_host_csr_load": (i32, [C.c_char_p, i32, PP]),
    "pc_host_csr_save": (i32, [P, C.c_char_p]),
    "pc_host_csr_from_arrays": (i32, [P, P, P, u64, u64, PP]),
    "pc_host_csr_free": (i32, [P]),
    "pc_synth_vertex_priority": (i32, [u64, u64, P]),
}


def _load():
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `python partitionandconquer_b200/build.py` (needs nvcc)"
        )
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIG.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def exported_symbols():
    """Names of _SIG entries that libpc.so exports."""
    return [n for n in _SIG if hasattr(lib, n)]


def check(status: int):
    if status != PC_OK:
        raise PCError(status, lib.pc_last_error().decode(errors="replace"))


def ptr(a):
    """Pointer to a numpy array's data (None -> NULL)."""
    if a is None:
        return None
    return C.c_void_p(a.ctypes.data)


def as_array(a, dtype):
    return np.ascontiguousarray(np.asarray(a), dtype=dtype)
