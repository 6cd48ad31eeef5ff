"""CPU tests of the oracle (the C restatement in oracle/qv_oracle.c).

The reference ships no tests or golden data for this path, and it cannot be run
here (no Fortran compiler), so the oracle is pinned by known answers that do
not depend on it: the 50-digit finite-segment field (tests/golden), the ring
speed/energy the reference prints at set-up, the reference's own dt bound, and
structural identities of the tree and the skip rules.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from qvort_b200 import workloads as W

GOLD = Path(__file__).resolve().parent / "golden"


def _kat_system(row):
    P, P2, A, B, Cc = row
    x = np.array([P, P2, A, B, Cc])
    inf = np.array([2, 1, 4, 5, 3], np.int32)
    beh = np.array([2, 1, 5, 3, 4], np.int32)
    return x, inf, beh


@pytest.mark.parametrize("velocity,theta", [("BS", 0.0), ("Tree", 1e-9)])
def test_segment_known_answers(velocity, theta):
    g = np.load(GOLD / "segment_kat.npz")
    p = O.params(velocity=velocity, tree_theta=theta, boundary="open", box_size=0.2,
                 quant_circ=float(g["gamma"]))
    worst = 0.0
    for k in range(g["P"].shape[0]):
        x, inf, beh = _kat_system([g[n][k] for n in ("P", "P2", "A", "B", "C")])
        gh = O.ghosts(p, x, inf, beh)
        tree = O.Tree(p, x, gh[0], inf) if velocity == "Tree" else None
        u, uli, ubs, ev, st = O.velocity(p, x, inf, beh, gh, tree)
        assert st == 0
        np.testing.assert_array_equal(uli[0], 0.0)
        ref = g["U"][k]
        worst = max(worst, np.abs(u[0] - ref).max() / np.abs(ref).max())
    assert worst < 1e-9, worst


def test_ring_speed_energy_known_answer():
    kat = np.load(GOLD / "ring_kat.npz")
    w = W.ring(200, float(kat["R"]), 0.0)
    p = O.params(**w.params)
    gh = O.ghosts(p, w.x, w.infront, w.behind)
    u, *_ = O.velocity(p, w.x, w.infront, w.behind, gh)
    speed = np.abs(u[:, 2].mean())
    assert abs(speed / float(kat["speed"]) - 1) < 0.01
    # all points translate together (axisymmetric ring)
    assert np.std(u[:, 2]) / speed < 1e-6
    assert np.abs(u[:, :2]).max() / speed < 1e-6
    # energy_info's line integral G * sum u.(s x s') dl of a ring of radius R
    # moving at speed v is 2 pi G R^2 v (the Kelvin impulse relation)
    e = O.energy(p, w.x, u, w.infront, gh)
    G, R = float(kat["gamma"]), float(kat["R"])
    assert abs(abs(e) / (2 * np.pi * G * R ** 2 * speed) - 1) < 1e-3



@pytest.mark.parametrize("order", [2, 4])
@pytest.mark.parametrize("fixed", [0, 1])
def test_lia_ring_closed_form(order, fixed):
    """The LIA arm of calc_velocity (src/timestep.f90) on a regular n-gon
    inscribed in a circle of radius R, in closed form.  With chord c =
    2R sin(t/2), t = 2 pi/n, the finite differences of get_deriv_1/2
    (src/derivatives.f90) reduce to the uniform stencils: second order
    |s'| = R sin t / c, |s''| = 2R(1 - cos t)/c^2; fourth order
    |s'| = R(8 sin t - sin 2t)/(6c), |s''| = R(5/2 - 8 cos t/3 + cos 2t/6)/c^2.
    The velocity is beta s' x s'' along the ring's axis with beta = 1.3e-3
    (fixed_LIA_beta) or Gamma/(4 pi) ln(1/(|s''| a))."""
    n, R = 48, 0.01
    w = W.ring(n, R, 0.0)
    p = O.params(**dict(w.params, velocity="LIA", deriv_order=order, fixed_lia_beta=fixed))
    gh = O.ghosts(p, w.x, w.infront, w.behind)
    u, uli, ubs, ev, st = O.velocity(p, w.x, w.infront, w.behind, gh)
    t = 2 * np.pi / n
    c = 2 * R * np.sin(t / 2)
    if order == 2:
        T, K = R * np.sin(t) / c, 2 * R * (1 - np.cos(t)) / c ** 2
    else:
        T = R * (8 * np.sin(t) - np.sin(2 * t)) / (6 * c)
        K = R * (2.5 - 8 * np.cos(t) / 3 + np.cos(2 * t) / 6) / c ** 2
    G, a = w.params["quant_circ"], w.params["corea"]
    beta = 1.3e-3 if fixed else G / (4 * np.pi) * np.log(1 / (K * a))
    speed = beta * T * K
    assert np.abs(np.abs(u[:, 2]) / speed - 1).max() < 1e-9
    assert np.abs(u[:, :2]).max() / speed < 1e-9
    assert np.all(np.sign(u[:, 2]) == np.sign(u[0, 2]))
    # the second-order stencil is exact for the curvature of a circle
    if order == 2:
        assert abs(K * R - 1) < 1e-12

def test_dt_bound():
    # timestep_check, src/initial.f90:606-622
    p = O.params(delta=5e-4, corea=1.3e-8)
    dm = 2.5e-4
    expect = abs(dm ** 2 / (9.97e-4 * np.log(dm / (np.pi * 1.3e-8))))
    assert O.dt_max(p) == pytest.approx(expect, rel=1e-15)
    assert 1e-7 < O.dt_max(p)


def _tree_invariants(ex, x, inf, L):
    m = len(ex["parent"])
    kids = {}
    for k in range(1, m):
        kids.setdefault(ex["parent"][k], []).append(k)
    for k in range(m):
        ch = kids.get(k, [])
        dig = [ex["digit"][c] for c in ch]
        assert dig == sorted(dig) and len(set(dig)) == len(dig)
        if k > 0:
            assert sum(ex["pcount"][c] for c in ch) <= ex["pcount"][k]
            if ex["pcount"][k] == 1:
                assert not ch
        for c in ch:
            assert ex["width"][c] == ex["width"][k] / 2
            assert ex["depth"][c] == ex["depth"][k] + 1
    assert ex["pcount"][0] == len(x)
    leaves = np.where(ex["pcount"] == 1)[0]
    firsts = ex["first"][leaves]
    assert len(set(firsts)) == len(firsts)


def test_tree_structure_tangle():
    w = W.tangle()
    p = O.params(**w.params)
    gh = O.ghosts(p, w.x, w.infront, w.behind)
    t = O.Tree(p, w.x, gh[0], w.infront)
    assert t.status == 0
    ex = t.export()
    _tree_invariants(ex, w.x, w.infront, 0.1)
    # every in-box active point ends in exactly one leaf
    assert (ex["pcount"] == 1).sum() == w.n


def test_tree_drops_out_of_box_and_empty():
    rng = np.random.default_rng(3)
    n = 400
    x = rng.uniform(-0.06, 0.06, (n, 3))   # some points outside [-0.05, 0.05)
    inf = np.roll(np.arange(1, n + 1), -1).astype(np.int32)
    beh = np.roll(np.arange(1, n + 1), 1).astype(np.int32)
    inf[::7] = 0                            # empty slots
    p = O.params(velocity="Tree", tree_theta=0.5, boundary="open", box_size=0.1)
    gh = O.ghosts(p, x, np.where(inf == 0, 1, inf), beh)
    t = O.Tree(p, x, gh[0], inf)
    ex = t.export()
    inside = np.all((x >= -0.05) & (x < 0.05), axis=1) & (inf != 0)
    assert (ex["pcount"] == 1).sum() == inside.sum()
    assert ex["pcount"][0] == n


def test_tree_minus_direct_is_infront_segment():
    """With theta -> 0 every node opens to its leaves, so the tree sum is the
    direct sum minus the segment infront(i) -> infront(infront(i)), which the
    leaf rule skips (src/tree.f90:371) and the direct sum keeps
    (src/timestep.f90:471)."""
    w = W.random_rings(6, 0.005, 0.01, 5e-4, 0.1, seed=5)
    base = dict(w.params, boundary="open")
    pd = O.params(**dict(base, velocity="BS", tree_theta=0.0))
    pt = O.params(**dict(base, velocity="Tree", tree_theta=1e-12))
    gh = O.ghosts(pd, w.x, w.infront, w.behind)
    ud, *_ = O.velocity(pd, w.x, w.infront, w.behind, gh)
    t = O.Tree(pt, w.x, gh[0], w.infront)
    ut, *_ = O.velocity(pt, w.x, w.infront, w.behind, gh, t)
    a = w.infront - 1
    R1 = w.x[a] - w.x
    R2 = gh[0][a] - w.x
    r1 = np.linalg.norm(R1, axis=1)
    r2 = np.linalg.norm(R2, axis=1)
    f = (r1 + r2) / (r1 * r2 * (r1 * r2 + (R1 * R2).sum(1)))
    seg = 9.97e-4 / (4 * np.pi) * f[:, None] * np.cross(R1, R2)
    err = np.abs(ud - ut - seg).max() / np.abs(ud).max()
    assert err < 1e-9, err


def test_ab_ladder_rungs():
    """Euler -> AB2 -> AB3 -> AB4 selected by exact-zero history
    (src/timestep.f90:51-61)."""
    n = 4
    x = np.zeros((n, 3))
    u = np.ones((n, 3))
    h = [np.zeros((n, 3)) for _ in range(3)]
    inf = np.arange(1, n + 1, dtype=np.int32)
    for k in range(1, n):
        for j in range(k):
            h[j][k] = 2.0
    dt = 0.5
    xn, u1, u2, u3 = O.pmotion_ab(dt, x, u, *h, inf)
    assert xn[0, 0] == dt * 1.0
    assert xn[1, 0] == 1.5 * dt * 1.0 - 0.5 * dt * 2.0
    assert xn[2, 0] == pytest.approx(23 / 12 * dt - 4 / 3 * dt * 2 + 5 / 12 * dt * 2, rel=1e-15)
    assert xn[3, 0] == pytest.approx(dt * (55 - 59 * 2 + 37 * 2 - 9 * 2) / 24, rel=1e-15)
    np.testing.assert_array_equal(u1, u)
    np.testing.assert_array_equal(u2, h[0])
    np.testing.assert_array_equal(u3, h[1])


def test_ghost_unwrap_periodic():
    L = 0.1
    x = np.array([[0.049, 0.0, 0.0], [-0.049, 0.0, 0.0], [-0.045, 0.0, 0.0]])
    inf = np.array([2, 3, 1], np.int32)
    beh = np.array([3, 1, 2], np.int32)
    p = O.params(boundary="periodic", box_size=L)
    gi, gb, gii, gbb = O.ghosts(p, x, inf, beh)
    assert gi[0, 0] == pytest.approx(-0.049 + L)
    assert gb[1, 0] == pytest.approx(0.049 - L)
    po = O.params(boundary="open", box_size=L)
    gi2, *_ = O.ghosts(po, x, inf, beh)
    assert gi2[0, 0] == -0.049


def test_pclose_matches_bruteforce_numpy():
    w = W.random_rings(5, 0.004, 0.008, 5e-4, 0.1, seed=11)
    cl, cd = O.pclose(w.x, w.infront, w.behind, np.zeros(w.n, np.int32))
    d = np.linalg.norm(w.x[:, None, :] - w.x[None, :, :], axis=2)
    idx = np.arange(w.n)
    d[idx, idx] = np.inf
    d[idx, w.infront - 1] = np.inf
    d[idx, w.behind - 1] = np.inf
    j = d.argmin(axis=1)
    np.testing.assert_array_equal(cl, j + 1)
    np.testing.assert_allclose(cd, d[idx, j], rtol=1e-15)


def _line_ring(n, radius, delta):
    w = W.ring(n, radius, 0.0, seed=0)
    p = O.params(**dict(w.params, delta=delta))
    g = O.ghosts(p, w.x, w.infront, w.behind)
    st = O.line_state(n, 3 * n, x=w.x, infront=w.infront, behind=w.behind, gi=g[0], gb=g[1],
                      gii=g[2], gbb=g[3])
    return p, st


def test_pinsert_ring_splits_every_segment_onto_the_circle():
    """Every segment of a coarse circle exceeds delta: one new point per segment,
    appended after the last slot (no empty slot), each on the circle (the
    insertion follows the local curvature radius, src/line.f90:68-85) and
    linked between its neighbours."""
    n, R = 40, 0.01
    p, st = _line_ring(n, R, 5e-4)          # spacing 1.57e-3
    n2, k = O.pinsert(p, n, st)
    assert (n2, k) == (2 * n, n)
    r = np.linalg.norm(st["x"][:n2], axis=1)
    assert np.abs(r - R).max() < 1e-3 * R   # the discrete curvature radius of a 40-gon
    inf = st["infront"][:n2]
    assert sorted(inf) == list(range(1, n2 + 1))
    for i in range(n):                       # i -> new point -> old infront
        j = inf[i] - 1
        assert j >= n and inf[j] == (i + 1) % n + 1


def test_pinsert_resolution_kept_and_premove_undoes_crowding():
    """After pinsert no segment is longer than delta on a circle whose spacing
    was between delta and 2 delta; premove on a circle spaced at 0.3 delta
    removes points until consecutive pairs are at least 0.998 delta apart (or
    the scan has passed them)."""
    p, st = _line_ring(60, 0.004, 3.5e-4)   # spacing 4.19e-4 in (delta, 2 delta)
    n2, k = O.pinsert(p, 60, st)
    assert k == 60
    x, inf = st["x"][:n2], st["infront"][:n2]
    seg = np.linalg.norm(x[inf - 1] - x, axis=1)
    assert seg.max() <= 3.5e-4
    p, st = _line_ring(200, 0.004, 4e-4)    # spacing 1.26e-4 = 0.31 delta
    removed = O.premove(p, 200, st)
    assert 0 < removed < 200
    inf = st["infront"][:200]
    act = np.nonzero(inf)[0]
    assert len(act) == 200 - removed
    # the loop is still closed: following infront from any point visits all
    k, seen = act[0], 0
    while True:
        k = inf[k] - 1
        seen += 1
        if k == act[0]:
            break
    assert seen == len(act)


def test_loop_killer_clears_loops_below_five_points():
    """premove leaving a loop of 4 points clears it (src/reconnection.f90:441-458);
    a loop left with 5 survives."""
    for npts, survives in ((5, False), (6, True)):
        b = np.array([0.0, 0.03, 0.06] + list(np.linspace(1.5, 5.0, npts - 3)))
        x = np.stack([0.003 * np.cos(b), 0.003 * np.sin(b), np.zeros(npts)], 1)
        inf = ((np.arange(npts) + 1) % npts + 1).astype(np.int32)
        beh = ((np.arange(npts) - 1) % npts + 1).astype(np.int32)
        p = O.params(**dict(W.ring(8).params, delta=3e-4))
        st = O.line_state(npts, npts, x=x, infront=inf, behind=beh)
        removed = O.premove(p, npts, st)
        alive = int((st["infront"][:npts] != 0).sum())
        if survives:
            assert removed == 1 and alive == npts - 1
        else:
            assert removed == npts and alive == 0


def _touching_rings(n=40, R=0.004, gap=1e-4):
    """Two coplanar rings, both counter-clockwise, a gap apart at x = 0: their
    tangents there are anti-parallel."""
    a = 2 * np.pi * (np.arange(n) + 0.5) / n
    r1 = np.stack([-R - gap / 2 + R * np.cos(a), R * np.sin(a), np.zeros(n)], 1)
    r2 = np.stack([R + gap / 2 + R * np.cos(a + np.pi), R * np.sin(a + np.pi), np.zeros(n)], 1)
    x = np.concatenate([r1, r2])
    k = np.arange(n)
    inf = np.concatenate([(k + 1) % n + 1, n + (k + 1) % n + 1]).astype(np.int32)
    beh = np.concatenate([(k - 1) % n + 1, n + (k - 1) % n + 1]).astype(np.int32)
    return x, inf, beh


def test_precon_merges_two_touching_rings():
    """Anti-parallel filaments closer than delta/2 reconnect (the line gets
    shorter): two loops become one loop through all points."""
    x, inf, beh = _touching_rings()
    n = len(x)
    p = O.params(**dict(W.ring(8).params, delta=5e-4))
    g = O.ghosts(p, x, inf, beh)
    cl, cd = O.pclose(x, inf, beh, np.zeros(n, np.int32))
    st = O.line_state(n, n, x=x, infront=inf, behind=beh, gi=g[0], gb=g[1], gii=g[2], gbb=g[3],
                      closest=cl, closestd=cd)
    assert (cd < 2.5e-4).sum() >= 2
    k = O.precon(p, n, st)
    assert k >= 1
    inf2 = st["infront"]
    alive = np.nonzero(inf2)[0]
    start = i = alive[0]
    seen = 0
    for _ in range(n):
        i = inf2[i] - 1
        seen += 1
        if i == start or i < 0:
            break
    # one loop through every surviving point (the two-point loop the second
    # reconnection cuts off goes to loop_killer)
    assert i == start and seen == len(alive) >= n - 8


def test_tree_walk_general_at_tiny_theta_is_the_segment_sum():
    """With theta -> 0 every leaf is visited: tree_walk_general is the sum over
    all segments (x_j -> ghosti_j) of the straight-segment term divided by
    4 pi (src/tree.f90:444-459), here summed independently with numpy."""
    w = W.random_rings(3, 0.006, 0.01, 5e-4, 0.1, seed=2, centre_box=0.05)
    p = O.params(**dict(w.params, boundary="open", velocity="Tree", tree_theta=1e-9))
    g = O.ghosts(p, w.x, w.infront, w.behind)
    tree = O.Tree(p, w.x, g[0], w.infront)
    pts = np.random.default_rng(5).uniform(-0.03, 0.03, (20, 3))
    u, ev = O.field_velocity_tree(p, tree, pts)
    assert ev == 20 * w.n
    for q, x in enumerate(pts):
        r1 = w.x - x
        r2 = g[0] - x
        a = np.linalg.norm(r1, axis=1)
        b = np.linalg.norm(r2, axis=1)
        c = a * b * (a * b + (r1 * r2).sum(1))
        ref = (((a + b) / c)[:, None] * np.cross(r1, r2)).sum(0) / (4 * np.pi)
        assert np.abs(u[q] - ref).max() <= 1e-9 * np.abs(ref).max()


def test_loop_without_line_ops_is_the_plain_step():
    """oracle.Loop with line_ops 0 runs the same body as State.step (ghosts,
    tree, velocity, AB, search, ghosts, wrap): identical states, bit for bit."""
    w = W.random_rings(6, 0.006, 0.01, 5e-4, 0.1, seed=5, theta=0.4)
    p = O.params(**w.params)
    lp = O.Loop(p, w.x, w.infront, w.behind, line_ops=0)
    st = O.State(p, w.x, w.infront, w.behind)
    for it in range(1, 4):
        assert lp.step(it) == 0 and st.step() == 0
        s = lp.state()
        for k in ("x", "u", "u1", "u2", "u3", "closest", "closestd"):
            np.testing.assert_array_equal(s[k], getattr(st, k), err_msg=k)


def test_loop_with_line_ops_keeps_links_consistent():
    """The default loop (pinsert, pclose_tree, precon, premove) on a tangle whose
    rings touch: every step reconnects or removes somewhere, and afterwards every
    active slot's neighbours point back at it and empty slots carry no links."""
    w = W.random_rings(40, 0.004, 0.012, 5e-4, 0.1, seed=3, theta=0.4, centre_box=0.03)
    p = O.params(**w.params)
    lp = O.Loop(p, w.x, w.infront, w.behind, line_ops=2)
    done = 0
    for it in range(1, 4):
        assert lp.step(it) == 0
        done += lp.counts["reconnected"] + lp.counts["removed"] + lp.counts["inserted"]
        s = lp.state()
        inf, beh = s["infront"], s["behind"]
        act = np.flatnonzero(inf)
        np.testing.assert_array_equal(beh[inf[act] - 1], act + 1)
        np.testing.assert_array_equal(inf[beh[act] - 1], act + 1)
        assert (beh[inf == 0] == 0).all()
    assert done > 0


def test_field_velocity_on_the_ring_axis_known_answer():
    """biot_savart_general on the axis of a ring of N = 200 straight segments
    against the circular ring's field G R^2 / (2 (R^2 + z^2)^(3/2)); the
    polygon differs from the circle at ~(pi/N)^2."""
    w = W.ring(200, 0.01, 0.0)
    p = O.params(**w.params)
    g = O.ghosts(p, w.x, w.infront, w.behind)
    G, R = w.params["quant_circ"], 0.01
    for z in (0.0, 0.003, -0.02):
        u = O.field_velocity(p, w.x, w.infront, g[0], np.array([[0.0, 0.0, z]]))[0]
        ref = G * R * R / (2 * (R * R + z * z) ** 1.5)
        assert abs(abs(u[2]) / ref - 1) < 1e-3, (z, u, ref)
        assert abs(u[0]) < 1e-12 * ref and abs(u[1]) < 1e-12 * ref
