"""The learned per-partition selector: the MLP's hand-written GPU forward and
backward kernels against an FP64 CPU restatement (gradient check), training,
and the selector end to end (collect timings, train, plan) -- with exact
triangle counts whatever the plan."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from partitionandconquer_b200._lib import MLP_HIDDEN as H, MLP_IN as IN, MLP_OUT as OUT  # noqa: E402


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + H * IN].reshape(H, IN); o += H * IN
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + OUT * H].reshape(OUT, H); o += OUT * H
    b3 = p[o:o + OUT]; o += OUT
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def cpu_loss_grad(p, x, y, m, w=None):
    """FP64 forward/backward of the same network and masked MSE loss, each
    sample's squared errors weighted by w (1 when None)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = x.astype(np.float64); y = y.astype(np.float64); m = m.astype(np.float64)
    w = np.ones(x.shape[0]) if w is None else np.asarray(w, np.float64)
    z1 = x @ W1.T + b1; h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2; h2 = np.maximum(z2, 0)
    out = h2 @ W3.T + b3
    cnt = m.sum()
    d = (out - y) * m
    loss = (w[:, None] * d * d).sum() / cnt
    dy = 2 * w[:, None] * d / cnt
    gW3 = dy.T @ h2; gb3 = dy.sum(0)
    dh2 = (dy @ W3) * (z2 > 0)
    gW2 = dh2.T @ h1; gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (z1 > 0)
    gW1 = dh1.T @ x; gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g, out


def random_problem(seed, batch=53):
    rng = np.random.default_rng(seed)
    p = (rng.standard_normal(IN * H + H + H * H + H + OUT * H + OUT) * 0.2).astype(np.float32)
    x = rng.standard_normal((batch, IN)).astype(np.float32)
    y = rng.standard_normal((batch, OUT)).astype(np.float32)
    m = (rng.random((batch, OUT)) < 0.7).astype(np.uint8)
    return p, x, y, m


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_mlp_gradient_matches_fp64_cpu(gpu, seed):
    sel = gpu.selector
    p, x, y, m = random_problem(seed)
    assert sel.mlp_num_params() == p.size
    loss, grad = sel.mlp_loss_grad(p, x, y, m)
    ref_loss, ref_grad, ref_out = cpu_loss_grad(p, x, y, m)
    np.testing.assert_allclose(sel.mlp_forward(p, x), ref_out, rtol=1e-4, atol=1e-5)
    assert loss == pytest.approx(ref_loss, rel=1e-4)
    scale = np.abs(ref_grad).max()
    np.testing.assert_allclose(grad, ref_grad, rtol=1e-3, atol=1e-5 * scale)


@pytest.mark.parametrize("seed", [3, 4])
def test_weighted_mlp_gradient_matches_fp64_cpu(gpu, seed):
    """The weighted loss the selector trains on (each unit weighted by the
    time of its fastest variant): GPU gradient against the FP64 restatement."""
    sel = gpu.selector
    p, x, y, m = random_problem(seed)
    wt = np.random.default_rng(seed + 100).lognormal(0.0, 1.5, x.shape[0]).astype(np.float32)
    wt *= wt.size / wt.sum()
    loss, grad = sel.mlp_loss_grad_weighted(p, x, y, m, wt)
    ref_loss, ref_grad, _ = cpu_loss_grad(p, x, y, m, wt)
    assert loss == pytest.approx(ref_loss, rel=1e-4)
    scale = np.abs(ref_grad).max()
    np.testing.assert_allclose(grad, ref_grad, rtol=1e-3, atol=1e-5 * scale)
    # all-ones weights give the unweighted loss
    l1, g1 = sel.mlp_loss_grad_weighted(p, x, y, m, np.ones(x.shape[0], np.float32))
    l0, g0 = sel.mlp_loss_grad(p, x, y, m)
    assert l1 == pytest.approx(l0, rel=1e-6)
    np.testing.assert_allclose(g1, g0, rtol=1e-6, atol=1e-7 * scale)


def test_mlp_gradient_finite_differences(gpu):
    sel = gpu.selector
    p, x, y, m = random_problem(7, batch=16)
    _, grad = sel.mlp_loss_grad(p, x, y, m)
    rng = np.random.default_rng(3)
    p64 = p.astype(np.float64)
    for i in rng.choice(p.size, 12, replace=False):
        e = np.zeros_like(p64); e[i] = 1e-5
        lp, _, _ = cpu_loss_grad(p64 + e, x, y, m)
        lm, _, _ = cpu_loss_grad(p64 - e, x, y, m)
        fd = (lp - lm) / 2e-5
        assert grad[i] == pytest.approx(fd, rel=2e-2, abs=2e-5), i


def test_mlp_training_reduces_loss(gpu):
    sel = gpu.selector
    rng = np.random.default_rng(11)
    x = rng.standard_normal((200, IN)).astype(np.float32)
    w = rng.standard_normal((IN, OUT))
    y = np.tanh(x @ w).astype(np.float32)
    m = np.ones((200, OUT), np.uint8)
    p = (rng.standard_normal(sel.mlp_num_params()) * 0.1).astype(np.float32)
    l0, _ = sel.mlp_loss_grad(p, x, y, m)
    p2, l1 = sel.mlp_train_steps(p, x, y, m, 300, 3e-3)
    assert l1 < 0.25 * l0
    l2, _ = sel.mlp_loss_grad(p2, x, y, m)
    assert l2 == pytest.approx(l1, rel=0.2)


def test_selector_end_to_end_exact(gpu, O, tmp_path):
    pc = gpu
    sel = pc.selector
    sel.clear()
    graphs = [pc.HostCSR.rmat(14, 16, 3), pc.HostCSR.er(14, 1 << 18, 4), pc.HostCSR.chung_lu(14, 1 << 18, 2.1, 2048, 5)]
    pgs = []
    for h in graphs:
        vl, el, _ = h.arrays()
        n = vl.size - 1
        pg = pc.Partitioned_Graph(pc.Graph(vlist=vl, elist=el), pc.equal_vertex_partition(n, 16))
        pgs.append((pg, O.tc_merge(vl, el)))
        assert sel.collect(pg, max_units=16, repeats=1) > 0
    f, y, m = sel.samples()
    assert f.shape[1] == 10 and y.shape[1] == pc.NUM_VARIANTS and m.any(axis=1).all()
    loss = sel.train(steps=400, lr=3e-3, seed=5)
    assert np.isfinite(loss)
    assert sel.trained()
    pred = sel.predict(f)
    assert pred.shape == y.shape and np.isfinite(pred).all()
    tuned = sel.autotune()
    assert tuned.shape == (4,)
    for pg, t in pgs:
        assert pg.triangle_count(variant=pc.VARIANT_AUTO) == t
        c, st = pg.triangle_count(variant=pc.VARIANT_AUTO, stats=True)
        assert c == t and st.selector == 2
        c, st = pg.triangle_count(variant=pc.VARIANT_HEURISTIC, stats=True)
        assert c == t and st.selector == 1
        plan = sel.plan(pg, pc.VARIANT_AUTO)
        assert plan.dtype == np.int8 and plan.max() < pc.NUM_VARIANTS
    path = str(tmp_path / "sel.bin")
    sel.save(path)
    before = sel.predict(f)
    sel.clear()
    assert not sel.trained()
    sel.load(path)
    np.testing.assert_allclose(sel.predict(f), before, rtol=1e-6)
    sel.enable(False)
    c, st = pgs[0][0].triangle_count(variant=pc.VARIANT_AUTO, stats=True)
    assert st.selector == 1 and c == pgs[0][1]
    sel.enable(True)
    sel.clear()


def test_insitu_collection_charges_every_unit(gpu, O):
    """pc_selector_collect_insitu: one profiled full run per variant; every
    unit with work gets a cost for each variant that can run it, the costs of
    one run add up to that run's kernel time, and counts stay exact."""
    pc = gpu
    sel = pc.selector
    sel.clear()
    vl, el, _ = pc.HostCSR.rmat(16, 16, 2).arrays()
    n = vl.size - 1
    g = pc.Graph(vlist=vl, elist=el)
    pg = pc.Partitioned_Graph(g, pc.equal_vertex_partition(n, 8))
    feats = sel.unit_features(pg)
    work = (feats[:, 1] > 0) & (feats[:, 2] > 0)
    added = sel.collect_insitu(pg, repeats=1)
    assert added == int(work.sum())
    f, y, m = sel.samples()
    assert f.shape[0] == added and m.any(axis=1).all()
    # the warp variants (hash, merge, gallop) run on every unit with work
    assert m[:, 3:6].all()
    assert np.isfinite(y[m.astype(bool)]).all()
    # per-unit shares of the hash run add up to about one full hash-variant run
    total = float(np.exp(y[:, 3]).sum())
    c, st = pg.triangle_count(variant=pc.VARIANTS["hash_warp"], stats=True)
    assert c == O.tc_merge(vl, el)
    assert 0.2 * st.kernel_ms < total < 5.0 * st.kernel_ms
    sel.clear()
    pg.close()
    g.close()


def test_learned_selector_on_config5(gpu):
    """What the trained network gains over the method without it, on config 5
    (RMAT-25 ef16 seed 1, 2048 partitions).  The training data are in-situ
    unit costs the library measures on other graphs (RMAT-22 and RMAT-24, and
    two RMAT-25 graphs with other seeds); the plain heuristic is autotuned on
    the same samples.  Before the bitmap kernels held high-id pivot sets as
    split sets, the plain rule's bitmaps spanned hundreds of thousands of ids
    on this graph and the network gained 1.33x by moving those units to the
    hash kernel; with split sets the plain plan is within a few per cent of
    the per-unit optimum, so the network has little left to gain.  Asserted:
    both counts equal the pinned T, the learned plan is not slower than the
    plain one beyond timing noise (the leave-one-graph-out judge keeps the
    heuristic wherever the model does not beat it), and the plain plan is
    within 10 % of the sum of the per-unit best in-situ costs on this graph."""
    import json

    from conftest import GOLDEN
    pc = gpu
    sel = pc.selector
    hp0 = sel.get_heuristic()
    sel.clear()
    try:
        for scale, seed in ((22, 2), (24, 6), (25, 2), (25, 3)):
            g = pc.Graph.rmat_device(scale, 16, seed)
            n = g.get_vertex_num()
            pg = pc.Partitioned_Graph(g, pc.equal_vertex_partition(n, n // 16384))
            assert sel.collect_insitu(pg, repeats=1) > 0
            pg.close()
            g.close()
        sel.autotune()
        sel.train(steps=1500, lr=3e-3, seed=7)
        margin, gain = sel.judge()
        assert gain >= 1.0, (margin, gain)
        want = json.loads((GOLDEN / "pinned_counts.json").read_text())["rmat25_ef16_s1"]["T"]
        g = pc.Graph.rmat_device(25, 16, 1)
        pg = pc.Partitioned_Graph(g, pc.equal_vertex_partition(g.get_vertex_num(), 2048))
        ms = {}
        for name, v in (("learned", pc.VARIANT_AUTO), ("plain", pc.VARIANT_HEURISTIC)):
            assert pg.triangle_count(variant=v) == want
            times = []
            for _ in range(3):
                c, st = pg.triangle_count(variant=v, stats=True)
                assert c == want
                times.append(st.kernel_ms)
            ms[name] = float(np.median(times))
        assert ms["learned"] <= 1.05 * ms["plain"], ms
        # in-situ cost of every variant on every unit of this graph: the plain
        # plan's units against the best variant of each unit
        n0 = sel.num_samples()
        sel.collect_insitu(pg, repeats=1)
        _, y, m = sel.samples()
        cost = np.where(m[n0:].astype(bool), np.exp(y[n0:].astype(np.float64)), np.inf)
        plan = sel.plan(pg, pc.VARIANT_HEURISTIC)
        plan = plan[plan >= 0].astype(np.int64)
        assert plan.size == cost.shape[0]
        best = float(cost.min(axis=1).sum())
        plain = float(cost[np.arange(plan.size), plan].sum())
        assert plain <= 1.10 * best, (plain, best)
        pg.close()
        g.close()
    finally:
        sel.clear()
        sel.set_heuristic(hp0)


def test_measured_autotune_keeps_a_timed_threshold_set(gpu, O):
    """pc_selector_autotune_measured: the best threshold sets by the collected
    in-situ costs, and the thresholds in force, are timed as whole plans on
    the given views; the kept set is the one in force afterwards, its summed
    time is positive, and counts under it stay exact."""
    pc = gpu
    sel = pc.selector
    hp0 = sel.get_heuristic()
    sel.clear()
    try:
        views = []
        for scale, seed in ((16, 3), (17, 4)):
            vl, el, _ = pc.HostCSR.rmat(scale, 16, seed).arrays()
            g = pc.Graph(vlist=vl, elist=el)
            pg = pc.Partitioned_Graph(g, pc.equal_vertex_partition(vl.size - 1, 16))
            assert sel.collect_insitu(pg, repeats=1) > 0
            views.append((g, pg, O.tc_merge(vl, el)))
        tuned, ms = sel.autotune(verify=[pg for _, pg, _ in views], k=4, repeats=2)
        assert ms > 0 and tuned.shape == (4,)
        assert np.array_equal(sel.get_heuristic(), tuned)
        for g, pg, t in views:
            assert pg.triangle_count(variant=pc.VARIANT_HEURISTIC) == t
            pg.close()
            g.close()
    finally:
        sel.clear()
        sel.set_heuristic(hp0)
