"""Host side of the per-partition selector, without a GPU: the sample store
and the proxy autotuner of the plain heuristic (pc_selector_add_samples,
pc_selector_get_samples, pc_selector_autotune, pc_selector_get/set_heuristic).

The samples are synthetic units with planted costs, so the thresholds that
minimise their summed cost are known: the autotuner must find them, respect
the per-sample feasibility masks, and never give the matrix form a unit whose
resident rows exceed 100 MB, however cheap its recorded cost."""
from __future__ import annotations

import numpy as np
import pytest

V = {"bitmap_warp": 0, "bitmap_group8": 1, "bitmap_lane": 2, "hash_warp": 3, "merge_lane": 4, "gallop_lane": 5,
     "matrix": 6}


def unit(npiv, ein, mean_scan, max_id, mdp=100):
    """Raw unit features: pivots, in-edges, sum |N+(b)|, max |N+(b)|, max id + 1,
    sum of prefix bounds, mean and variance of log degree, long-prefix share,
    in-edges per pivot."""
    return np.array([npiv, ein, npiv * mdp / 2, mdp, max_id, ein * mean_scan, 5.0, 1.0, 0.5, ein / npiv],
                    np.float32)


def add(sel, rows):
    """rows: (features, {variant: cost ms}); missing variants are infeasible."""
    f = np.stack([r[0] for r in rows])
    y = np.zeros((len(rows), 7), np.float32)
    m = np.zeros((len(rows), 7), np.uint8)
    for i, (_, costs) in enumerate(rows):
        for name, ms in costs.items():
            y[i, V[name]] = np.log(ms)
            m[i, V[name]] = 1
    sel.add_samples(f, y, m)
    return f, y, m


@pytest.fixture
def sel(pc):
    s = pc.selector
    hp0 = s.get_heuristic()
    s.clear()
    yield s
    s.clear()
    s.set_heuristic(hp0)


def test_samples_round_trip(sel):
    f, y, m = add(sel, [(unit(100, 8000, 50, 1 << 18), {"bitmap_group8": 1.0, "hash_warp": 2.0}),
                        (unit(100, 4000, 50, 1 << 18), {"hash_warp": 0.5})])
    assert sel.num_samples() == 2
    f2, y2, m2 = sel.samples()
    np.testing.assert_array_equal(f2, f)
    np.testing.assert_array_equal(m2, m)
    np.testing.assert_allclose(y2[m2.astype(bool)], y[m.astype(bool)])
    sel.clear()
    assert sel.num_samples() == 0


def test_heuristic_params_round_trip(sel):
    sel.set_heuristic([32.0, 1e30, 16.0, 96.0])
    np.testing.assert_array_equal(sel.get_heuristic(), [32.0, 1e30, 16.0, 96.0])


def test_autotune_finds_planted_thresholds(sel):
    """Heavy units (80 in-edges per pivot) are cheapest under the 8-lane bitmap
    kernel, light ones (40) under the hash kernel, and the 32-lane and one-lane
    bitmap kernels cost more everywhere: only a bitmap bound between 40 and 80
    (64 on the grid), a 32-lane bound above every prefix mean and an 8-lane
    bound at or below them give the minimum."""
    heavy = {"bitmap_warp": 10.0, "bitmap_group8": 1.0, "bitmap_lane": 10.0, "hash_warp": 5.0,
             "merge_lane": 10.0, "gallop_lane": 10.0}
    light = {"bitmap_warp": 10.0, "bitmap_group8": 5.0, "bitmap_lane": 10.0, "hash_warp": 1.0,
             "merge_lane": 10.0, "gallop_lane": 10.0}
    rows = [(unit(1000, 80000, 40 + i, 1 << 18), heavy) for i in range(20)]
    rows += [(unit(1000, 40000, 40 + i, 1 << 18), light) for i in range(20)]
    add(sel, rows)
    a, w, g, mx = sel.autotune()
    assert a == 64.0
    assert w > 59 and g <= 40


def test_autotune_respects_masks(sel):
    """A unit where the variant the best rule would pick is infeasible makes
    that rule unusable: the autotuner must choose thresholds that avoid it."""
    cheap_lane = {"bitmap_lane": 1.0, "hash_warp": 3.0, "merge_lane": 9.0, "gallop_lane": 9.0}
    no_lane = {"bitmap_group8": 2.0, "hash_warp": 3.0, "merge_lane": 9.0, "gallop_lane": 9.0}
    add(sel, [(unit(1000, 80000, 20, 1 << 18), cheap_lane), (unit(1000, 80000, 20, 1 << 18), no_lane)])
    a, w, g, mx = sel.autotune()
    # bitmap_lane (g > 20) is infeasible for the second unit and bitmap_warp /
    # group8 for the first, so the only plan that runs both is the hash kernel
    assert a > 80


def test_matrix_form_needs_rows_that_fit_l2(sel):
    """Hub units whose rows fit 100 MB (16 K pivots below id 2^14: 32 MB) may
    take the matrix form; a unit of 16 K pivots below id 2^16 (128 MB of rows)
    may not, even when its recorded matrix cost is the lowest."""
    fits = {"bitmap_warp": 4.0, "bitmap_group8": 3.0, "bitmap_lane": 9.0, "hash_warp": 9.0,
            "merge_lane": 9.0, "gallop_lane": 9.0, "matrix": 1.0}
    add(sel, [(unit(16384, 16384 * 300, 300, 1 << 14), fits)])
    a, w, g, mx = sel.autotune()
    assert mx <= 300 and a <= 300  # the matrix form is used
    sel.clear()
    too_big = dict(fits)
    add(sel, [(unit(16384, 16384 * 300, 300, 1 << 16), too_big)])
    a, w, g, mx = sel.autotune()
    # the rule cannot give this unit the matrix form, so group8 (3 ms) is the
    # best it can do: a bitmap bound the unit passes and an 8-lane bound at or
    # below its prefix mean, with the 32-lane bound above it
    assert a <= 300 and g <= 300 < w


def test_measured_autotune_rejects_bad_arguments(pc, sel):
    """The measured stage checks its arguments before touching a device."""
    import ctypes as C

    from partitionandconquer_b200 import _lib
    out = np.empty(4, np.float64)
    ms = C.c_double()
    for npg, k, reps in ((0, 4, 2), (1, 0, 2), (1, 4, 0)):
        views = (C.c_void_p * 1)(None)
        rc = _lib.lib.pc_selector_autotune_measured(views, npg, k, reps, _lib.ptr(out), C.byref(ms))
        assert rc == 1  # PC_ERR_INVALID_INPUT
    rc = _lib.lib.pc_selector_autotune_measured((C.c_void_p * 1)(None), 1, 4, 2, _lib.ptr(out), C.byref(ms))
    assert rc == 1  # a null view
