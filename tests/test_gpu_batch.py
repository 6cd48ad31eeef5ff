"""Batched systems (qv_batch_*) against the same systems run one by one.

A batch of independent open systems -- rings and leap-frogging pairs, direct
sums below 2000 points and Barnes-Hut (theta 0.4) above, each with its own
dt -- must reproduce, bit for bit, what a single-system context computes for
each system: velocities, and positions after several Adams-Bashforth steps.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mods():
    from qvort_b200 import lib as L
    from qvort_b200 import workloads as W

    return L, W


def _systems(W, n=12, seed=3, nmax=4000):
    return W.batch_systems(n_systems=n, seed=seed, nmin=100, nmax=nmax)


def _batch(L, ws):
    p = L.default_params(**dict(ws[0].params, boundary="open", velocity="Tree", tree_theta=0.4,
                                precision="mixed"))
    method = [w.params["velocity"] for w in ws]
    return L.Batch(p, [(w.x, w.infront, w.behind) for w in ws], method,
                   [w.params["dt"] for w in ws])


def _single(L, w):
    c = L.Context(L.default_params(**dict(w.params, precision="mixed")))
    c.set_points(w.x, w.infront, w.behind)
    return c


def test_batch_has_both_methods():
    L, W = _mods()
    ws = _systems(W)
    m = {w.params["velocity"] for w in ws}
    assert m == {"BS", "Tree"}


def test_batch_velocity_matches_single_systems_bitwise():
    L, W = _mods()
    ws = _systems(W)
    b = _batch(L, ws)
    ub = b.split(b.velocity())
    for w, u in zip(ws, ub):
        c = _single(L, w)
        ref = c.velocity(False)[0]
        c.close()
        assert np.array_equal(u, ref), (w.name, w.n, w.params["velocity"],
                                        np.abs(u - ref).max())
    b.close()


def test_batch_steps_match_single_systems_bitwise():
    L, W = _mods()
    ws = _systems(W, n=8, seed=4)
    b = _batch(L, ws)
    K = 6
    b.step(K)
    xb, _ = b.get_points()
    st = b.stats()
    b.close()
    for w, x in zip(ws, b.split(xb)):
        c = _single(L, w)
        for _ in range(K):
            if w.params["velocity"] == "Tree":
                c.build_tree()
            c.velocity(False)
            c.step_ab()
        ref, _ = c.get_points()
        c.close()
        assert np.array_equal(x, ref), (w.name, np.abs(x - ref).max())
    assert st["tree_systems"] > 0 and st["items"] > 0


def test_batch_results_do_not_depend_on_launch_shape():
    L, W = _mods()
    ws = _systems(W, n=10, seed=7)
    b = _batch(L, ws)
    u0 = b.velocity()
    for cfg in ((2, 1, 0), (8, 2, 1), (4, 3, 0)):
        b.set_config(*cfg)
        assert np.array_equal(b.velocity(), u0), cfg
    t = b.tune(reps=1)
    assert t["warps_per_block"] in (2, 4, 8)
    assert np.array_equal(b.velocity(), u0)
    b.close()


def test_batch_step_uses_a_graph_and_repeats():
    L, W = _mods()
    ws = _systems(W, n=6, seed=11)
    b1, b2 = _batch(L, ws), _batch(L, ws)
    b1.step(4)
    for _ in range(4):
        b2.step(1)
    x1, _ = b1.get_points()
    x2, _ = b2.get_points()
    assert b1.stats()["graph"]
    assert np.array_equal(x1, x2)
    b1.close()
    b2.close()


def test_batch_rejects_bad_input():
    L, W = _mods()
    ws = _systems(W, n=3, seed=1, nmax=500)
    p = L.default_params(**dict(ws[0].params, boundary="periodic", precision="mixed"))
    with pytest.raises(L.QvError):
        L.Batch(p, [(w.x, w.infront, w.behind) for w in ws], ["BS"] * 3, [1e-7] * 3)
    p = L.default_params(**dict(ws[0].params, boundary="open", precision="mixed"))
    bad = [(w.x, np.zeros_like(w.infront), w.behind) for w in ws]
    with pytest.raises(L.QvError):
        L.Batch(p, bad, ["BS"] * 3, [1e-7] * 3)
