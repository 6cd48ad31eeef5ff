"""pinsert / premove on the GPU against the oracle's restatement, bit for bit.

Each case hands both sides the same state -- positions, velocities, AB
history, links and the stored ghosts (computed before the move, as after
pmotion) -- and compares the whole state afterwards: slot count, links,
positions, velocities, history and the ghosts of every active slot.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mods():
    from qvort_b200 import lib as L
    from qvort_b200 import workloads as W

    return L, W


def _ctx_state(c, n_cap=None):
    x, u = c.get_points()
    u1, u2, u3 = c.get_history()
    g = c.get_ghosts()
    inf, beh = c.get_links()
    return dict(x=x, u=u, u1=u1, u2=u2, u3=u3, gi=g[0], gb=g[1], gii=g[2], gbb=g[3],
                infront=inf, behind=beh)


def _oracle_state(st, cap):
    n = st["x"].shape[0]
    return n, O.line_state(n, cap, **st)


def _compare(c, n_ref, ref):
    assert c.n == n_ref
    got = _ctx_state(c)
    act = ref["infront"][:n_ref] != 0
    for k in ("infront", "behind"):
        assert np.array_equal(got[k], ref[k][:n_ref]), k
    for k in ("x", "u", "u1", "u2", "gi", "gb", "gii", "gbb"):
        a, b = got[k][act], ref[k][:n_ref][act]
        assert np.array_equal(a, b), (k, np.abs(a - b).max())


def _moved_ring(L, W, n=60, radius=0.004, delta=5e-4, boundary="open", shift=None, steps=2):
    """A ring advanced a couple of AB steps through the C ABI: positions moved,
    stored ghosts from before the last move."""
    w = W.ring(n, radius, 2e-5, seed=3)
    x = w.x.copy()
    if shift is not None:
        x = W.wrap(x + shift, 0.1)
    prm = dict(w.params, delta=delta, boundary=boundary, box_size=0.1, dt=2e-6)
    c = L.Context(L.default_params(**prm))
    c.set_points(x, w.infront, w.behind)
    for _ in range(steps):
        c.ghosts()
        c.velocity(False)
        c.step_ab()
    return c, O.params(**prm)


@pytest.mark.parametrize("boundary,shift", [("open", None), ("periodic", (0.048, 0.0, -0.049))])
def test_pinsert_matches_oracle(boundary, shift):
    L, W = _mods()
    # spacing 2 pi 0.004 / 60 = 4.2e-4: 0.4e-3 < delta so that some, not all, split
    c, p = _moved_ring(L, W, delta=4.1e-4, boundary=boundary,
                       shift=None if shift is None else np.array(shift))
    st = _ctx_state(c)
    n0, ref = _oracle_state(st, st["x"].shape[0] + 200)
    n_ref, k_ref = O.pinsert(p, n0, ref)
    k = c.pinsert()
    assert k == k_ref and k > 0
    _compare(c, n_ref, ref)
    c.close()


def test_pinsert_fills_empty_slots_first_and_chains():
    """Empty slots (infront = 0) are taken in ascending order before any slot
    is appended; a point placed in an empty slot beyond the scan position is
    tested again by the scan (a segment longer than 2 delta splits twice)."""
    L, W = _mods()
    w = W.ring(24, 0.004, 0.0, seed=0)            # spacing 1.05e-3
    n_extra = 8
    x = np.concatenate([w.x[:12], np.zeros((n_extra, 3)), w.x[12:]])
    idx = np.concatenate([np.arange(12), np.arange(12 + n_extra, 24 + n_extra)])
    inf = np.zeros(24 + n_extra, np.int32)
    beh = np.zeros(24 + n_extra, np.int32)
    for k, s in enumerate(idx):
        inf[s] = idx[(k + 1) % 24] + 1
        beh[s] = idx[(k - 1) % 24] + 1
    prm = dict(w.params, delta=4e-4, box_size=0.1)
    c = L.Context(L.default_params(**prm))
    c.set_points(x, inf, beh)
    c.ghosts()
    st = _ctx_state(c)
    n0, ref = _oracle_state(st, st["x"].shape[0] + 200)
    p = O.params(**prm)
    n_ref, k_ref = O.pinsert(p, n0, ref)
    k = c.pinsert()
    assert k == k_ref
    assert k > 24 and n_ref > n0          # chains, then appended slots
    _compare(c, n_ref, ref)
    c.close()


def test_pinsert_grows_past_the_allocated_slots():
    L, W = _mods()
    n = 40000
    w = W.ring(n, 0.05, 0.0, seed=1)              # spacing 7.9e-6, delta 5e-6: every segment splits
    prm = dict(w.params, delta=5e-6, box_size=0.3)
    c = L.Context(L.default_params(**prm))
    c.set_points(w.x, w.infront, w.behind)
    c.ghosts()
    st = _ctx_state(c)
    n0, ref = _oracle_state(st, 2 * n + 10)
    n_ref, k_ref = O.pinsert(O.params(**prm), n0, ref)
    assert c.pinsert() == k_ref == n
    _compare(c, n_ref, ref)
    c.close()


def test_premove_matches_oracle_and_kills_small_loops():
    L, W = _mods()
    # ring 1: points bunched so that several points go; ring 2: 5 points whose
    # removal leaves 4 (loop_killer clears it)
    rng = np.random.default_rng(4)
    a = np.sort(rng.uniform(0, 2 * np.pi, 80))
    r1 = np.stack([0.004 * np.cos(a), 0.004 * np.sin(a), np.zeros(80)], 1)
    b = np.array([0.0, 0.03, 0.06, 2.0, 4.0])
    r2 = np.stack([0.01 + 0.003 * np.cos(b), 0.003 * np.sin(b), np.zeros(5)], 1)
    x = np.concatenate([r1, r2])
    inf = np.concatenate([(np.arange(80) + 1) % 80 + 1, 80 + (np.arange(5) + 1) % 5 + 1]).astype(np.int32)
    beh = np.concatenate([(np.arange(80) - 1) % 80 + 1, 80 + (np.arange(5) - 1) % 5 + 1]).astype(np.int32)
    prm = dict(W.ring(8).params, delta=3e-4, box_size=0.1)
    c = L.Context(L.default_params(**prm))
    c.set_points(x, inf, beh)
    c.ghosts()
    st = _ctx_state(c)
    n0, ref = _oracle_state(st, 85)
    k_ref = O.premove(O.params(**prm), n0, ref)
    k = c.premove()
    assert k == k_ref and k > 5
    got_inf, _ = c.get_links()
    assert not got_inf[80:].any()          # the small loop is gone
    _compare(c, n0, ref)
    c.close()


def test_step_with_line_ops_equals_the_call_sequence():
    """qv_step with line_ops = 1 is ghosts, tree, velocity, AB, pinsert,
    candidate search, premove, ghosts, wrap (src/run.f90:41-93 with
    switch_off_recon)."""
    L, W = _mods()
    w = W.random_rings(6, 0.004, 0.006, 3e-4, 0.1, seed=2, centre_box=0.06)
    # spacing 0.75 x 3e-4 = 2.25e-4 > delta: the first step splits every segment
    prm = dict(w.params, delta=2.2e-4, tree_theta=0.4, velocity="Tree", precision="mixed",
               dt=5e-6)
    a = L.Context(L.default_params(**prm, line_ops=1))
    a.set_points(w.x, w.infront, w.behind)
    b = L.Context(L.default_params(**prm))
    b.set_points(w.x, w.infront, w.behind)
    for it in range(1, 4):
        a.step(it)
        b.ghosts()
        b.build_tree()
        b.velocity(False)
        b.step_ab()
        b.pinsert()
        b.closest()
        b.premove()
        b.ghosts()
        b.enforce_periodic()
    assert a.n == b.n > w.n
    xa, _ = a.get_points()
    xb, _ = b.get_points()
    ia, _ = a.get_links()
    ib, _ = b.get_links()
    assert np.array_equal(ia, ib)
    act = ia != 0
    assert np.array_equal(xa[act], xb[act])
    a.close()
    b.close()


def test_precon_matches_oracle():
    L, W = _mods()
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).parent))
    from test_oracle import _touching_rings

    x, inf, beh = _touching_rings()
    prm = dict(W.ring(8).params, delta=5e-4, box_size=0.1)
    c = L.Context(L.default_params(**prm))
    c.set_points(x, inf, beh)
    c.ghosts()
    cl, cd = c.closest()
    st = _ctx_state(c)
    n0, ref = _oracle_state(st, len(x))
    ref["closest"][:] = cl
    ref["closestd"][:] = cd
    k_ref = O.precon(O.params(**prm), n0, ref)
    k = c.precon()
    assert k == k_ref == 2
    _compare(c, n0, ref)
    c.close()


def test_precon_many_pairs_and_tangle_match_oracle():
    """The ordered pass visits only the candidates whose test can reconnect on
    the starting links or whose slots an earlier reconnection relinked: on
    six touching ring pairs (gaps from 2e-5 to 2.4e-4 cm, some of whose
    reconnections leave loops that loop_killer clears, and candidates that do
    not reconnect) next to the config-2 tangle, its links and count are the
    oracle's precon_original bit for bit."""
    L, W = _mods()
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).parent))
    from test_oracle import _touching_rings

    xs, infs, behs, off = [], [], [], 0
    for k, (n, gap) in enumerate([(40, 2e-5), (12, 4e-5), (40, 1.2e-4), (8, 6e-5), (40, 2.4e-4),
                                  (24, 1e-4)]):
        x, inf, beh = _touching_rings(n=n, R=0.002 + 0.0004 * k, gap=gap)
        x = x + np.array([-0.04 + 0.015 * k, 0.03, -0.02])
        xs.append(x); infs.append(inf + off); behs.append(beh + off)
        off += len(x)
    w = W.tangle(0)
    xs.append(w.x); infs.append(w.infront + off); behs.append(w.behind + off)
    x = np.concatenate(xs); inf = np.concatenate(infs).astype(np.int32)
    beh = np.concatenate(behs).astype(np.int32)
    prm = dict(w.params, delta=5e-4)
    c = L.Context(L.default_params(**prm))
    c.set_points(x, inf, beh)
    c.ghosts()
    c.build_tree()
    cl, cd = c.closest()  # pclose_tree
    st = _ctx_state(c)
    n0, ref = _oracle_state(st, len(x))
    ref["closest"][:] = cl
    ref["closestd"][:] = cd
    cand = int(((cd < 2.5e-4) & (cd > 0) & (inf != 0)).sum())
    k_ref = O.precon(O.params(**prm), n0, ref)
    k = c.precon()
    assert k == k_ref and k >= 3, (k, k_ref)
    assert cand > 20, cand
    _compare(c, n0, ref)
    c.close()


def test_step_with_reconnection_equals_the_call_sequence():
    """line_ops = 2: pinsert, candidate search, precon, premove in qv_step."""
    L, W = _mods()
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).parent))
    from test_oracle import _touching_rings

    x, inf, beh = _touching_rings(n=60, R=0.004, gap=4e-5)
    prm = dict(W.ring(8).params, delta=4.5e-4, box_size=0.1, tree_theta=0.4, velocity="Tree",
               precision="mixed", dt=1e-6)
    a = L.Context(L.default_params(**prm, line_ops=2))
    a.set_points(x, inf, beh)
    b = L.Context(L.default_params(**prm))
    b.set_points(x, inf, beh)
    nrec = 0
    for it in range(1, 4):
        a.step(it)
        b.ghosts()
        b.build_tree()
        b.velocity(False)
        b.step_ab()
        b.pinsert()
        b.closest()
        nrec += b.precon()
        b.premove()
        b.ghosts()
        b.enforce_periodic()
    assert nrec > 0 and a.n == b.n
    ia, _ = a.get_links()
    ib, _ = b.get_links()
    assert np.array_equal(ia, ib)
    xa, _ = a.get_points()
    xb, _ = b.get_points()
    act = ia != 0
    assert np.array_equal(xa[act], xb[act])
    a.close()
    b.close()


def test_step_whose_pinsert_outgrows_the_slots_equals_the_call_sequence():
    """qv_step queues the candidate search behind pinsert before it reads the
    new slot count; when pinsert stops to have the arrays grown, that search
    does nothing and runs again after the growth.  Every segment of this ring
    splits (spacing 1.6e-5 > delta 5e-6), far more insertions than the spare
    slots, and the step must equal the separate calls."""
    L, W = _mods()
    n = 20000
    w = W.ring(n, 0.05, 0.0, seed=2)
    prm = dict(w.params, delta=5e-6, box_size=0.3, velocity="Tree", tree_theta=0.4,
               precision="mixed", dt=1e-9)
    a = L.Context(L.default_params(**prm, line_ops=2))
    a.set_points(w.x, w.infront, w.behind)
    b = L.Context(L.default_params(**prm))
    b.set_points(w.x, w.infront, w.behind)
    a.step(1)
    b.ghosts()
    b.build_tree()
    b.velocity(False)
    b.step_ab()
    assert b.pinsert() == n
    cb, _ = b.closest()
    b.precon()
    b.premove()
    b.ghosts()
    b.enforce_periodic()
    assert a.n == b.n == 2 * n
    ia, _ = a.get_links()
    ib, _ = b.get_links()
    assert np.array_equal(ia, ib)
    xa, _ = a.get_points()
    xb, _ = b.get_points()
    act = ia != 0
    assert np.array_equal(xa[act], xb[act])
    ca, da = a.get_closest()
    cb2, db = b.get_closest()
    assert np.array_equal(ca, cb2) and np.array_equal(da, db)
    a.close()
    b.close()
