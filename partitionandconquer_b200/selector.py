"""Per-partition intersection-kernel selection: features, training data, the
GPU-trained MLP and the autotuned heuristic (thin wrappers over include/pc.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import MLP_IN, MLP_OUT, NUM_VARIANTS, SELECTOR_FEATURES, check, lib, ptr

FEATURE_NAMES = [
    "pivots", "in_edges", "sum_set", "max_set", "max_id_plus1", "sum_scan", "mean_log_deg", "var_log_deg",
    "frac_scan_ge32", "in_per_pivot",
]


def num_units(pg) -> int:
    n = C.c_int32()
    check(lib.pc_tc_units(pg.handle, C.byref(n)))
    return int(n.value)


def unit_features(pg) -> np.ndarray:
    u = num_units(pg)
    out = np.empty((u, SELECTOR_FEATURES), np.float32)
    check(lib.pc_tc_unit_features(pg.handle, ptr(out), u))
    return out


def plan(pg, variant: int) -> np.ndarray:
    u = num_units(pg)
    out = np.empty(u, np.int8)
    check(lib.pc_tc_plan(pg.handle, variant, ptr(out), u))
    return out


def time_unit(pg, unit: int, variant: int):
    ms, cnt = C.c_double(), C.c_uint64()
    check(lib.pc_tc_time_unit(pg.handle, unit, variant, C.byref(ms), C.byref(cnt)))
    return float(ms.value), int(cnt.value)


def collect(pg, max_units: int = 256, repeats: int = 2) -> int:
    """Each feasible variant timed on each sampled unit alone."""
    added = C.c_int32()
    check(lib.pc_selector_collect(pg.handle, max_units, repeats, C.byref(added)))
    return int(added.value)


def collect_insitu(pg, repeats: int = 2) -> int:
    """Each variant run on all units at once; every unit charged its share
    of the run (per-item cycle counters).  One sample per unit with work."""
    added = C.c_int32()
    check(lib.pc_selector_collect_insitu(pg.handle, repeats, C.byref(added)))
    return int(added.value)


def judge():
    """(log margin, held-out gain) of the trained selector's judge."""
    m, g = C.c_double(), C.c_double()
    check(lib.pc_selector_judge(C.byref(m), C.byref(g)))
    return float(m.value), float(g.value)


def num_samples() -> int:
    return int(lib.pc_selector_num_samples())


def samples():
    n = num_samples()
    f = np.empty((n, SELECTOR_FEATURES), np.float32)
    y = np.empty((n, MLP_OUT), np.float32)
    m = np.empty((n, MLP_OUT), np.uint8)
    check(lib.pc_selector_get_samples(ptr(f), ptr(y), ptr(m), n))
    return f, y, m


def add_samples(feats, log_ms, mask):
    f = _lib.as_array(feats, np.float32)
    y = _lib.as_array(log_ms, np.float32)
    m = _lib.as_array(mask, np.uint8)
    check(lib.pc_selector_add_samples(ptr(f), ptr(y), ptr(m), f.shape[0]))


def train(steps: int = 2000, lr: float = 3e-3, seed: int = 7) -> float:
    loss = C.c_float()
    check(lib.pc_selector_train(steps, lr, seed, C.byref(loss)))
    return float(loss.value)


def predict(feats) -> np.ndarray:
    f = _lib.as_array(feats, np.float32)
    out = np.empty((f.shape[0], MLP_OUT), np.float32)
    check(lib.pc_selector_predict(ptr(f), f.shape[0], ptr(out)))
    return out


def autotune(verify=None, k: int = 8, repeats: int = 3):
    """Heuristic thresholds from the collected samples.  With `verify` (graph
    views other than the measured ones), the k best sets by the samples and
    the thresholds in force are timed there and the fastest is kept; returns
    (thresholds, summed ms).  Without, returns the samples' best thresholds."""
    out = np.empty(4, np.float64)
    if not verify:
        check(lib.pc_selector_autotune(ptr(out)))
        return out
    handles = (C.c_void_p * len(verify))(*[pg.handle for pg in verify])
    ms = C.c_double()
    check(lib.pc_selector_autotune_measured(handles, len(verify), k, repeats, ptr(out), C.byref(ms)))
    return out, float(ms.value)


def get_heuristic() -> np.ndarray:
    out = np.empty(4, np.float64)
    check(lib.pc_selector_get_heuristic(ptr(out)))
    return out


def set_heuristic(params):
    p = _lib.as_array(params, np.float64)
    if p.size != 4:
        raise ValueError("four thresholds: in-edges per pivot, 32-lane, 8-lane and matrix prefix lengths")
    check(lib.pc_selector_set_heuristic(ptr(p)))


def clear():
    check(lib.pc_selector_clear())


def trained() -> bool:
    return bool(lib.pc_selector_trained())


def enable(on: bool):
    check(lib.pc_selector_enable(int(on)))


def save(path: str):
    check(lib.pc_selector_save(path.encode()))


def load(path: str):
    check(lib.pc_selector_load(path.encode()))


# -- the MLP's GPU kernels, for gradient checks --

def mlp_num_params() -> int:
    return int(lib.pc_mlp_num_params())


def mlp_forward(params, x) -> np.ndarray:
    p = _lib.as_array(params, np.float32)
    xx = _lib.as_array(x, np.float32).reshape(-1, MLP_IN)
    out = np.empty((xx.shape[0], MLP_OUT), np.float32)
    check(lib.pc_mlp_forward(ptr(p), ptr(xx), xx.shape[0], ptr(out)))
    return out


def mlp_loss_grad(params, x, y, mask):
    p = _lib.as_array(params, np.float32)
    xx = _lib.as_array(x, np.float32).reshape(-1, MLP_IN)
    yy = _lib.as_array(y, np.float32).reshape(-1, MLP_OUT)
    mm = _lib.as_array(mask, np.uint8).reshape(-1, MLP_OUT)
    loss = C.c_float()
    grad = np.empty(p.size, np.float32)
    check(lib.pc_mlp_loss_grad(ptr(p), ptr(xx), ptr(yy), ptr(mm), xx.shape[0], C.byref(loss), ptr(grad)))
    return float(loss.value), grad


def mlp_loss_grad_weighted(params, x, y, mask, weights):
    p = _lib.as_array(params, np.float32)
    xx = _lib.as_array(x, np.float32).reshape(-1, MLP_IN)
    yy = _lib.as_array(y, np.float32).reshape(-1, MLP_OUT)
    mm = _lib.as_array(mask, np.uint8).reshape(-1, MLP_OUT)
    ww = _lib.as_array(weights, np.float32)
    if ww.size != xx.shape[0]:
        raise ValueError("one weight per sample")
    loss = C.c_float()
    grad = np.empty(p.size, np.float32)
    check(lib.pc_mlp_loss_grad_weighted(ptr(p), ptr(xx), ptr(yy), ptr(mm), ptr(ww), xx.shape[0], C.byref(loss),
                                        ptr(grad)))
    return float(loss.value), grad


def mlp_train_steps(params, x, y, mask, steps: int, lr: float):
    p = _lib.as_array(params, np.float32).copy()
    xx = _lib.as_array(x, np.float32).reshape(-1, MLP_IN)
    yy = _lib.as_array(y, np.float32).reshape(-1, MLP_OUT)
    mm = _lib.as_array(mask, np.uint8).reshape(-1, MLP_OUT)
    loss = C.c_float()
    check(lib.pc_mlp_train_steps(ptr(p), ptr(xx), ptr(yy), ptr(mm), xx.shape[0], steps, lr, C.byref(loss)))
    return p, float(loss.value)


__all__ = [n for n in dir() if not n.startswith("_") and n not in ("C", "np", "annotations")] + ["NUM_VARIANTS"]
