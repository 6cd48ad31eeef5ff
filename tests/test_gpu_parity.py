"""GPU parity of the CUDA path against the oracle, through the C ABI.

Bars (written per test): integer/index results and the tree are bit-exact;
FP64 velocities agree with the oracle to 1e-10 relative (different but
equivalent FP64 evaluation orders); the mixed-precision path agrees with the
FP64 path to 1e-6 RMS relative velocity error.
"""
import numpy as np
import pytest

from oracle import oracle as O
from qvort_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    from qvort_b200 import lib

    return lib


def ctx_for(L, w, **over):
    prm = dict(w.params)
    prm.update(over)
    c = L.Context(L.default_params(**prm))
    c.set_points(w.x, w.infront, w.behind)
    return c


def opar(w, **over):
    prm = dict(w.params)
    prm.update(over)
    prm.pop("precision", None)
    return O.params(**prm)


def rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def rel_max(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def small_tangle(seed=1, n_rings=20):
    return W.random_rings(n_rings, 0.006, 0.012, 5e-4, 0.1, seed=seed, theta=0.4)


# ------------------------------------------------------------------ ghosts
@pytest.mark.parametrize("bc", ["open", "periodic", "openx", "openxy"])
def test_ghosts_bit_exact(L, bc):
    w = small_tangle()
    c = ctx_for(L, w, boundary=bc)
    c.ghosts()
    g = c.get_ghosts()
    og = O.ghosts(opar(w, boundary=bc), w.x, w.infront, w.behind)
    for a, b in zip(g, og):
        np.testing.assert_array_equal(a, b)


# ------------------------------------------------------------------ direct
def test_direct_fp64_ring_matches_oracle(L):
    w = W.ring()
    c = ctx_for(L, w, precision="fp64")
    u, uli, ubs, ev = c.velocity()
    p = opar(w)
    og = O.ghosts(p, w.x, w.infront, w.behind)
    ou, ouli, oubs, *_ = O.velocity(p, w.x, w.infront, w.behind, og)
    assert rel_max(uli, ouli) < 1e-12
    assert rel_max(u, ou) < 1e-10
    assert ev == w.n * w.n


@pytest.mark.parametrize("bc", ["periodic", "openx", "openxy", "open"])
def test_direct_fp64_images_match_oracle(L, bc, nthreads):
    w = small_tangle(2, 8)
    c = ctx_for(L, w, velocity="BS", tree_theta=0.0, boundary=bc, precision="fp64")
    u, uli, ubs, ev = c.velocity()
    p = opar(w, velocity="BS", tree_theta=0.0, boundary=bc)
    og = O.ghosts(p, w.x, w.infront, w.behind)
    ou, ouli, oubs, *_ = O.velocity(p, w.x, w.infront, w.behind, og, nthreads=nthreads)
    assert rel_max(u, ou) < 1e-10
    assert rel_max(ubs, oubs) < 1e-10


def _seg_terms(P, pts):
    """|field| of each straight segment of the loop pts at P (numpy FP64)."""
    out = []
    for a, b in zip(pts, pts[1:] + pts[:1]):
        R1, R2 = a - P, b - P
        r1, r2 = np.linalg.norm(R1), np.linalg.norm(R2)
        f = (r1 + r2) / (r1 * r2 * (r1 * r2 + R1 @ R2))
        out.append(np.linalg.norm(9.97e-4 / (4 * np.pi) * f * np.cross(R1, R2)))
    return out


def test_direct_segment_known_answers(L):
    """The 50-digit triangle-loop fixtures.  FP64: 1e-9 of the net field.  Mixed:
    1e-6 of the summed segment magnitudes (far loops are dipoles whose net field
    is ~d/size times smaller than each segment's, a cancellation no FP32 term
    survives; the bar is on the per-term accuracy)."""
    from pathlib import Path

    g = np.load(Path(__file__).resolve().parent / "golden" / "segment_kat.npz")
    worst = {"fp64": 0.0, "mixed": 0.0}
    for prec in worst:
        for k in range(g["P"].shape[0]):
            x = np.array([g["P"][k], g["P2"][k], g["A"][k], g["B"][k], g["C"][k]])
            inf = np.array([2, 1, 4, 5, 3], np.int32)
            beh = np.array([2, 1, 5, 3, 4], np.int32)
            c = L.Context(L.default_params(velocity="BS", boundary="open", box_size=0.2,
                                           quant_circ=float(g["gamma"]), precision=prec))
            c.set_points(x, inf, beh)
            u, uli, *_ = c.velocity()
            np.testing.assert_array_equal(uli[0], 0.0)
            if prec == "fp64":
                scale = np.abs(g["U"][k]).max()
            else:
                scale = sum(_seg_terms(g["P"][k], [g["A"][k], g["B"][k], g["C"][k]]))
            worst[prec] = max(worst[prec], np.abs(u[0] - g["U"][k]).max() / scale)
            c.close()
    assert worst["fp64"] < 1e-9, worst
    assert worst["mixed"] < 1e-6, worst


def test_direct_mixed_vs_fp64(L):
    w = small_tangle(3, 12)
    c64 = ctx_for(L, w, velocity="BS", tree_theta=0.0, precision="fp64")
    c32 = ctx_for(L, w, velocity="BS", tree_theta=0.0, precision="mixed")
    u64 = c64.velocity()[0]
    u32 = c32.velocity()[0]
    assert rel_rms(u32, u64) < 1e-6


# ------------------------------------------------------------------ tree
def _compare_trees(g, o):
    assert len(g["parent"]) == len(o["parent"])
    for k in ("parent", "digit", "depth", "pcount", "first"):
        np.testing.assert_array_equal(g[k], o[k], err_msg=k)
    for k in ("pos", "width", "cent", "circ", "Cij"):
        np.testing.assert_array_equal(g[k], o[k], err_msg=k)


@pytest.mark.parametrize("seed", [0, 1])
def test_tree_bit_exact_tangle(L, seed):
    w = W.tangle(seed)
    c = ctx_for(L, w)
    c.ghosts()
    c.build_tree()
    gt = c.tree_export()
    p = opar(w)
    og = O.ghosts(p, w.x, w.infront, w.behind)
    ot = O.Tree(p, w.x, og[0], w.infront).export()
    _compare_trees(gt, ot)


def test_tree_bit_exact_many_ranges(L):
    """~420k points: more block-local ranges of the build than co-resident
    blocks, so blocks take several ranges each."""
    w = W.large_tangle(2, n_rings=1600)
    assert w.n > 400_000  # > 2 ranges per co-resident block (296)
    c = ctx_for(L, w)
    c.ghosts()
    c.build_tree()
    gt = c.tree_export()
    p = opar(w)
    og = O.ghosts(p, w.x, w.infront, w.behind)
    ot = O.Tree(p, w.x, og[0], w.infront).export()
    _compare_trees(gt, ot)
    c.close()


def test_tree_bit_exact_edge_cases(L):
    rng = np.random.default_rng(7)
    n = 3000
    x = rng.uniform(-0.055, 0.055, (n, 3))        # some outside the box
    x[:50] = np.round(x[:50] * 40) / 40            # points on cell boundaries
    x[50:60] = x[60:70] + 1e-13                    # near-coincident pairs
    # one loop through the active slots; every 11th slot empty
    inf = np.zeros(n, np.int32)
    beh = np.zeros(n, np.int32)
    act_slots = np.setdiff1d(np.arange(n), np.arange(0, n, 11))
    inf[act_slots] = np.roll(act_slots, -1) + 1
    beh[act_slots] = np.roll(act_slots, 1) + 1
    prm = dict(velocity="Tree", tree_theta=0.5, boundary="open", box_size=0.1)
    c = L.Context(L.default_params(**prm))
    c.set_points(x, inf, beh)
    c.ghosts()
    c.build_tree()
    gt = c.tree_export()
    p = O.params(**prm)
    og = O.ghosts(p, x, inf, beh)
    gg = c.get_ghosts()
    act = inf != 0
    np.testing.assert_array_equal(gg[0][act], og[0][act])
    ot = O.Tree(p, x, gg[0], inf).export()
    _compare_trees(gt, ot)


def test_tree_depth_error_not_hang(L):
    """Coincident points exactly at the origin never separate: the corner
    stays 0 and every cell [0, w) keeps them down to widths that underflow
    (~1075 levels in the reference).  The build stops at QV_MAX_DEPTH with an
    error instead.  Coincident points elsewhere terminate (the corner sums stop
    changing and the points fall out), as in the reference."""
    n = 8
    x = np.zeros((n, 3))
    inf = np.roll(np.arange(1, n + 1), -1).astype(np.int32)
    beh = np.roll(np.arange(1, n + 1), 1).astype(np.int32)
    c = L.Context(L.default_params(velocity="Tree", tree_theta=0.5, box_size=0.1))
    c.set_points(x, inf, beh)
    with pytest.raises(L.QvError) as e:
        c.build_tree()
    assert e.value.code == L.QV_ERR_TREE_DEPTH


# ------------------------------------------------------------------ walk
@pytest.mark.parametrize("bc", ["periodic", "open"])
def test_walk_fp64_matches_oracle(L, bc, nthreads):
    w = W.tangle(0)
    c = ctx_for(L, w, boundary=bc, precision="fp64")
    c.ghosts()
    c.build_tree()
    u, uli, ubs, ev = c.velocity()
    p = opar(w, boundary=bc)
    og = O.ghosts(p, w.x, w.infront, w.behind)
    tr = O.Tree(p, w.x, og[0], w.infront)
    ou, ouli, oubs, oev, st = O.velocity(p, w.x, w.infront, w.behind, og, tr, nthreads=nthreads)
    assert st == 0
    assert ev == oev           # identical traversals: identical evaluation counts
    assert rel_max(u, ou) < 1e-10
    assert rel_max(ubs, oubs) < 1e-9


def test_walk_mixed_vs_fp64(L):
    w = W.tangle(0)
    c64 = ctx_for(L, w, precision="fp64")
    c32 = ctx_for(L, w, precision="mixed")
    r = []
    for c in (c64, c32):
        c.ghosts()
        c.build_tree()
        r.append(c.velocity())
    assert r[0][3] == r[1][3]  # same nodes visited
    assert rel_rms(r[1][0], r[0][0]) < 1e-6
    assert rel_rms(r[1][2], r[0][2]) < 1e-5


@pytest.mark.parametrize("velocity,bc,opts", [
    ("Tree", "openx", {}),
    ("Tree", "openxy", {}),
    ("Tree", "periodic", {"deriv_order": 4}),
    ("Tree", "periodic", {"tree_extra_correction": 0}),
    ("BS", "openx", {"deriv_order": 4}),
    ("LIA", "periodic", {}),
    ("LIA", "periodic", {"fixed_lia_beta": 1}),
    ("LIA", "open", {"deriv_order": 4}),
])
def test_velocity_options_match_oracle(L, velocity, bc, opts, nthreads):
    """Every velocity arm, boundary and option of calc_velocity
    (src/timestep.f90) in FP64 against the oracle: the same tree traversal
    (identical evaluation counts) and velocities within 1e-10 relative."""
    w = small_tangle(5, 24)
    theta = 0.4 if velocity == "Tree" else 0.0
    c = ctx_for(L, w, boundary=bc, velocity=velocity, tree_theta=theta, precision="fp64", **opts)
    c.ghosts()
    if velocity == "Tree":
        c.build_tree()
    u, uli, ubs, ev = c.velocity()
    p = opar(w, boundary=bc, velocity=velocity, tree_theta=theta, **opts)
    og = O.ghosts(p, w.x, w.infront, w.behind)
    tr = O.Tree(p, w.x, og[0], w.infront) if velocity == "Tree" else None
    ou, ouli, oubs, oev, st = O.velocity(p, w.x, w.infront, w.behind, og, tr, nthreads=nthreads)
    assert st == 0
    if velocity == "Tree":         # the oracle counts tree evaluations only
        assert ev == oev
    # the direct sum adds ~3e4 terms per target in blocked order (the oracle:
    # one running sum), so its FP64 bar is 1e-9 of the largest velocity
    assert rel_max(u, ou) < (1e-9 if velocity == "BS" else 1e-10)
    if velocity != "LIA":          # the LIA arm reports neither part separately
        assert rel_max(uli, ouli) < 1e-12
        assert rel_max(ubs, oubs) < 1e-9


@pytest.mark.parametrize("velocity,bc,opts", [
    ("Tree", "openx", {}),
    ("Tree", "openxy", {"deriv_order": 4}),
    ("Tree", "periodic", {"tree_extra_correction": 0}),
    ("BS", "openxy", {}),
])
def test_velocity_options_mixed_vs_fp64(L, velocity, bc, opts):
    """The mixed-precision kernels under the same options: same traversal as
    FP64, velocities within 1e-6 RMS relative."""
    w = small_tangle(6, 24)
    theta = 0.4 if velocity == "Tree" else 0.0
    r = []
    for prec in ("fp64", "mixed"):
        c = ctx_for(L, w, boundary=bc, velocity=velocity, tree_theta=theta, precision=prec,
                    **opts)
        c.ghosts()
        if velocity == "Tree":
            c.build_tree()
        r.append(c.velocity())
        c.close()
    assert r[0][3] == r[1][3]
    assert rel_rms(r[1][0], r[0][0]) < 1e-6


# ------------------------------------------------------------------ steps
def test_ab_step_bit_exact_given_velocity(L):
    w = small_tangle(4, 10)
    c = ctx_for(L, w, precision="fp64")
    rng = np.random.default_rng(0)
    h = [rng.normal(size=(w.n, 3)) * 0.1 for _ in range(3)]
    h[2][::3] = 0.0
    h[1][::5] = 0.0
    h[0][::7] = 0.0
    c.set_history(*h)
    c.ghosts()
    c.build_tree()
    u, *_ = c.velocity()
    c.step_ab()
    x, _ = c.get_points()
    hist = c.get_history()
    ox, ou1, ou2, ou3 = O.pmotion_ab(w.params["dt"], w.x, u, *h, w.infront)
    np.testing.assert_array_equal(x, ox)
    np.testing.assert_array_equal(hist[0], ou1)
    np.testing.assert_array_equal(hist[1], ou2)
    np.testing.assert_array_equal(hist[2], ou3)


def test_closest_tree_bit_exact(L, nthreads):
    w = W.tangle(1)
    c = ctx_for(L, w, precision="fp64")
    c.ghosts()
    c.build_tree()
    c.velocity()
    c.step_ab()                     # move; the tree is now stale
    rng = np.random.default_rng(5)
    seedcl = rng.integers(0, w.n, w.n).astype(np.int32)
    c.set_closest(seedcl)
    cl, cd = c.closest()
    xn, _ = c.get_points()
    p = opar(w)
    og = O.ghosts(p, w.x, w.infront, w.behind)
    tr = O.Tree(p, w.x, og[0], w.infront)
    ocl, ocd = O.pclose_tree(tr, xn, w.infront, w.behind, seedcl, nthreads)
    np.testing.assert_array_equal(cl, ocl)
    np.testing.assert_array_equal(cd, ocd)



def test_closest_tree_after_pinsert_bit_exact(L):
    """The candidate search after pinsert, as in a step: the tree and its
    parray(1)%infront links are from before the move, the positions and links
    are current, and new points (not in the tree) search too."""
    w = W.random_rings(12, 0.004, 0.008, 3e-4, 0.1, seed=3, theta=0.4)
    c = ctx_for(L, w, precision="fp64", delta=2.2e-4, dt=5e-6)
    c.ghosts()
    c.build_tree()
    x0, _ = c.get_points()
    inf0, beh0 = c.get_links()
    g0 = c.get_ghosts()
    c.velocity(False)
    c.step_ab()
    assert c.pinsert() > 0
    n = c.n
    rng = np.random.default_rng(2)
    seedcl = rng.integers(0, n, n).astype(np.int32)
    c.set_closest(seedcl)
    cl, cd = c.closest()
    xn, _ = c.get_points()
    infn, behn = c.get_links()
    p = opar(w, delta=2.2e-4)
    tr = O.Tree(p, x0, g0[0], inf0)
    ocl, ocd = O.pclose_tree(tr, xn, infn, behn, seedcl)
    np.testing.assert_array_equal(cl, ocl)
    np.testing.assert_array_equal(cd, ocd)
    c.close()


@pytest.mark.parametrize("n,theta", [(64, 0.4), (200, 0.5), (7, 0.4)])
def test_closest_tree_regular_ring_ties(L, n, theta):
    """A regular polygon: every point has two partners at the same distance
    (two links ahead and behind), so the walk order decides which one is
    kept; tiny rings leave no valid partner at all."""
    w = W.ring(n, 0.01, 0.0)
    prm = dict(w.params, velocity="Tree", tree_theta=theta)
    c = L.Context(L.default_params(**prm))
    c.set_points(w.x, w.infront, w.behind)
    c.ghosts()
    c.build_tree()
    seedcl = np.arange(n, dtype=np.int32)[::-1].copy()
    c.set_closest(seedcl)
    cl, cd = c.closest()
    p = O.params(**prm)
    og = O.ghosts(p, w.x, w.infront, w.behind)
    tr = O.Tree(p, w.x, og[0], w.infront)
    ocl, ocd = O.pclose_tree(tr, w.x, w.infront, w.behind, seedcl)
    np.testing.assert_array_equal(cl, ocl)
    np.testing.assert_array_equal(cd, ocd)
    c.close()

def test_pclose_bit_exact(L):
    w = small_tangle(6, 10)
    c = ctx_for(L, w, velocity="BS", tree_theta=0.0)
    cl, cd = c.closest()
    ocl, ocd = O.pclose(w.x, w.infront, w.behind, np.zeros(w.n, np.int32))
    np.testing.assert_array_equal(cl, ocl)
    np.testing.assert_array_equal(cd, ocd)


def test_energy_matches_oracle(L):
    w = W.ring()
    c = ctx_for(L, w)
    u, *_ = c.velocity()
    e = c.energy()
    p = opar(w)
    og = O.ghosts(p, w.x, w.infront, w.behind)
    assert e == pytest.approx(O.energy(p, w.x, u, w.infront, og), rel=1e-12)


def test_ring_trajectory_1000_steps(L):
    """Configuration 1: ring, FP64 direct BS + LIA, AB ladder, 1000 steps,
    against the oracle's own 1000 steps and the analytic speed."""
    w = W.ring()
    c = ctx_for(L, w, precision="fp64")
    st = O.State(opar(w), w.x, w.infront, w.behind)
    nsteps = 1000
    for it in range(1, nsteps + 1):
        c.step(it)
        st.step()
    x, _ = c.get_points()
    assert rel_max(x - w.x, st.x - w.x) < 1e-8
    dz = (x[:, 2] - w.x[:, 2]).mean()
    speed = abs(dz) / (nsteps * w.params["dt"])
    ana = 9.97e-4 / (4 * np.pi * 0.01) * (np.log(8 * 0.01 / 1.3e-8) - 0.5)
    assert abs(speed / ana - 1) < 0.01


def test_rk3_step_matches_oracle(L):
    w = small_tangle(8, 6)
    prm = dict(runge_kutta=1, precision="fp64")
    c = ctx_for(L, w, **prm)
    st = O.State(opar(w), w.x, w.infront, w.behind)
    for it in range(1, 4):
        c.step(it)
        st.step(runge_kutta=True)
    x, _ = c.get_points()
    assert rel_max(x - w.x, st.x - w.x) < 1e-8


def test_tangle_steps_match_oracle(L, nthreads):
    w = small_tangle(9, 30)
    c = ctx_for(L, w, precision="fp64")
    st = O.State(opar(w), w.x, w.infront, w.behind)
    for it in range(1, 6):
        c.step(it)
        st.step(nthreads=nthreads)
    x, _ = c.get_points()
    d = x - st.x
    d -= np.round(d / 0.1) * 0.1   # a wrap decision may differ at the box face
    assert np.abs(d).max() / np.abs(st.x - w.x).max() < 1e-6


def test_unsupported_boundary_is_an_error(L):
    with pytest.raises(L.QvError) as e:
        L.Context(L.default_params(boundary=5))
    assert e.value.code == L.QV_ERR_UNSUPPORTED


def test_coincident_points_off_origin_match_oracle(L):
    n = 8
    x = np.zeros((n, 3)) + 0.0123
    x[4:] += np.array([1e-3, -2e-3, 5e-4])
    inf = np.roll(np.arange(1, n + 1), -1).astype(np.int32)
    beh = np.roll(np.arange(1, n + 1), 1).astype(np.int32)
    prm = dict(velocity="Tree", tree_theta=0.5, box_size=0.1)
    c = L.Context(L.default_params(**prm))
    c.set_points(x, inf, beh)
    c.ghosts()
    c.build_tree()
    gt = c.tree_export()
    p = O.params(**prm)
    og = O.ghosts(p, x, inf, beh)
    t = O.Tree(p, x, og[0], inf)
    assert t.status == 0
    _compare_trees(gt, t.export())


@pytest.mark.parametrize("velocity,boundary,recon_shots", [("BS", "open", 1), ("BS", "periodic", 3),
                                                            ("LIA", "open", 1)])
def test_steps_replay_equals_step_loop(velocity, boundary, recon_shots):
    """qv_steps (a CUDA graph of one step, replayed) leaves the same state as
    calling qv_step for each step: positions, history and candidate pairs."""
    import torch

    from qvort_b200 import lib as L
    from qvort_b200 import workloads as W

    w = W.random_rings(4, 0.006, 0.01, 5e-4, 0.1, seed=6, centre_box=0.05)
    prm = dict(w.params, velocity=velocity, boundary=boundary, tree_theta=0.0,
               recon_shots=recon_shots, precision="fp64")
    s = torch.cuda.Stream()
    a = L.Context(L.default_params(**prm), stream=s.cuda_stream)
    b = L.Context(L.default_params(**prm), stream=s.cuda_stream)
    for c in (a, b):
        c.set_points(w.x, w.infront, w.behind)
    a.steps(1, 12)
    for it in range(1, 13):
        b.step(it)
    xa, ua = a.get_points()
    xb, ub = b.get_points()
    assert np.array_equal(xa, xb) and np.array_equal(ua, ub)
    for ha, hb in zip(a.get_history(), b.get_history()):
        assert np.array_equal(ha, hb)
    ca, da = a.get_closest()
    cb, db = b.get_closest()
    assert np.array_equal(ca, cb) and np.array_equal(da, db)
    a.close()
    b.close()


def test_state_exchange_equals_separate_calls():
    """qv_set_state / qv_get_state move the same data as the separate set/get
    calls, in one call each way."""
    from qvort_b200 import lib as L
    from qvort_b200 import workloads as W

    w = W.random_rings(4, 0.006, 0.01, 5e-4, 0.1, seed=8, centre_box=0.05)
    prm = dict(w.params, precision="mixed", tree_theta=0.4, velocity="Tree")
    a = L.Context(L.default_params(**prm))
    a.set_points(w.x, w.infront, w.behind)
    for it in range(1, 4):
        a.step(it)
    n = a.n
    cap = n + 5
    got = dict(x=np.zeros((cap, 3)), u=np.zeros((cap, 3)), u1=np.zeros((cap, 3)),
               u2=np.zeros((cap, 3)), u3=np.zeros((cap, 3)), infront=np.zeros(cap, np.int32),
               behind=np.zeros(cap, np.int32), closest=np.zeros(cap, np.int32),
               closestd=np.zeros(cap))
    assert a.get_state(cap, **got) == n
    x, u = a.get_points()
    hist = a.get_history()
    inf, beh = a.get_links()
    cl, cd = a.get_closest()
    ref = dict(x=x, u=u, u1=hist[0], u2=hist[1], u3=hist[2], infront=inf, behind=beh,
               closest=cl, closestd=cd)
    for k, v in ref.items():
        assert np.array_equal(got[k][:n], v), k
    with pytest.raises(L.QvError):
        a.get_state(n - 1, **got)
    # one upload == the three separate ones: the next step agrees bit for bit
    b = L.Context(L.default_params(**prm))
    b.set_state(n, **{k: got[k] for k in ("x", "infront", "behind", "u1", "u2", "u3", "closest")})
    c = L.Context(L.default_params(**prm))
    c.set_points(x, inf, beh)
    c.set_history(*hist)
    c.set_closest(cl)
    b.step(4)
    c.step(4)
    assert np.array_equal(b.get_points()[0], c.get_points()[0])
    assert np.array_equal(b.get_closest()[0], c.get_closest()[0])
    for ctx in (a, b, c):
        ctx.close()


@pytest.mark.parametrize("bc,theta", [("periodic", 0.4), ("open", 0.5), ("openx", 0.3)])
def test_field_velocity_tree_matches_oracle(L, bc, theta):
    """tree_walk_general at points of a mesh, at random points and at filament
    points themselves, against the oracle: the same evaluations and the same
    FP64 sums.  At a filament point the reference's own arithmetic can give
    NaN (its leaf is skipped by the epsilon test, but the segment ending there
    may have |R2| = 0); both sides must agree on where."""
    w = small_tangle()
    c = ctx_for(L, w, boundary=bc, velocity="Tree", tree_theta=theta, precision="fp64")
    rng = np.random.default_rng(3)
    g = np.linspace(-0.045, 0.045, 8)
    mesh = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pts = np.concatenate([mesh, rng.uniform(-0.05, 0.05, (200, 3)), w.x[::37]])
    u, ev = c.field_velocity_tree(pts)
    p = opar(w, boundary=bc, velocity="Tree", tree_theta=theta)
    og = O.ghosts(p, w.x, w.infront, w.behind)
    tree = O.Tree(p, w.x, og[0], w.infront)
    uo, evo = O.field_velocity_tree(p, tree, pts)
    c.close()
    assert ev == evo
    nan = np.isnan(uo)
    assert np.array_equal(np.isnan(u), nan)
    ok = ~nan.any(axis=1)
    assert rel_max(u[ok], uo[ok]) < 1e-12, rel_max(u[ok], uo[ok])


@pytest.mark.parametrize("delta", [4.5e-4, 4.1e-4, 9e-4])
def test_step_exchange_equals_set_step_get(delta):
    """qv_step_exchange (one call, copies overlapping the step) leaves the host
    copy of f(:) exactly as qv_set_state, qv_step, qv_get_state do, through
    steps with reconnections (delta 4.5e-4), insertions (4.1e-4, below the
    point spacing 4.2e-4) or removals (9e-4, above half the distance to the
    second neighbour: the cleared slots are zeroed in the copies taken before
    premove ran); a host copy too small for the slot count is an error that
    leaves it untouched."""
    from qvort_b200 import lib as L
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).parent))
    from test_oracle import _touching_rings

    x, inf, beh = _touching_rings(n=60, R=0.004, gap=4e-5)
    prm = dict(W.ring(8).params, delta=delta, box_size=0.1, tree_theta=0.4, velocity="Tree",
               precision="mixed", dt=1e-6, line_ops=2)
    n0 = len(x)
    cap = 4 * n0

    def host():
        h = dict(x=np.zeros((cap, 3)), u=np.zeros((cap, 3)), u1=np.zeros((cap, 3)),
                 u2=np.zeros((cap, 3)), u3=np.zeros((cap, 3)), infront=np.zeros(cap, np.int32),
                 behind=np.zeros(cap, np.int32), closest=np.zeros(cap, np.int32),
                 closestd=np.zeros(cap))
        h["x"][:n0] = x
        h["infront"][:n0] = inf
        h["behind"][:n0] = beh
        return h

    ha, hb = host(), host()
    a = L.Context(L.default_params(**prm))
    b = L.Context(L.default_params(**prm))
    ins = ("x", "infront", "behind", "u1", "u2", "u3", "closest")
    na = nb = n0
    for it in range(1, 6):
        na = a.step_exchange(it, na, cap, {k: ha[k] for k in ins}, ha)
        b.set_state(nb, **{k: hb[k] for k in ins})
        b.step(it)
        nb = b.get_state(cap, **hb)
        assert na == nb
        for k in ha:
            assert np.array_equal(ha[k][:na], hb[k][:nb]), (it, k)
    if delta < 4.2e-4:
        assert na > n0                                      # points were inserted
    elif delta > 8e-4:
        assert (ha["infront"][:na] != 0).sum() < n0          # points were removed
    else:
        assert not np.array_equal(ha["infront"][:n0], inf)  # links were reconnected
    before = {k: v.copy() for k, v in ha.items()}
    with pytest.raises(L.QvError):
        a.step_exchange(6, na, na - 1, {k: ha[k] for k in ins}, ha)
    for k in ha:
        assert np.array_equal(ha[k], before[k]), k
    a.close()
    b.close()


def test_step_exchange_equals_set_step_get_late_level1(L):
    """The same equality on config 2's tangle with the root children's long
    moment sums taken late (forced: the tangle is below the size that takes them
    late by itself): the exchange step's copies of u and the AB history, taken
    behind pinsert, hold the velocities with the deferred far-field terms in."""
    w = W.tangle(0)
    prm = dict(w.params, precision="mixed", line_ops=2)
    n0 = w.n
    cap = n0 + 8192

    def host():
        h = dict(x=np.zeros((cap, 3)), u=np.zeros((cap, 3)), u1=np.zeros((cap, 3)),
                 u2=np.zeros((cap, 3)), u3=np.zeros((cap, 3)), infront=np.zeros(cap, np.int32),
                 behind=np.zeros(cap, np.int32), closest=np.zeros(cap, np.int32),
                 closestd=np.zeros(cap))
        h["x"][:n0] = w.x
        h["infront"][:n0] = w.infront
        h["behind"][:n0] = w.behind
        return h

    ha, hb = host(), host()
    ins = ("x", "infront", "behind", "u1", "u2", "u3", "closest")
    L.test_late_level1(1)
    try:
        a = L.Context(L.default_params(**prm))
        b = L.Context(L.default_params(**prm))
        na = nb = n0
        for it in range(1, 4):
            na = a.step_exchange(it, na, cap, {k: ha[k] for k in ins}, ha)
            b.set_state(nb, **{k: hb[k] for k in ins})
            b.step(it)
            nb = b.get_state(cap, **hb)
            assert na == nb
            for k in ha:
                assert np.array_equal(ha[k][:na], hb[k][:nb]), (it, k)
        a.close()
        b.close()
    finally:
        L.test_late_level1(-1)


@pytest.mark.parametrize("bc", ["open", "periodic", "openx", "openxy"])
def test_field_velocity_direct_matches_oracle(L, bc):
    """biot_savart_general with the boundary's images (the BS arm of
    mesh_velocity, src/timestep.f90:393-416) at mesh points and random points,
    against the oracle's restatement of src/timestep.f90:516-563: FP64 within
    1e-10 relative.  The GPU sums each source's images before the next source,
    the reference each image over all sources, so the two orders differ."""
    w = small_tangle()
    c = ctx_for(L, w, boundary=bc, velocity="BS", tree_theta=0.0, precision="fp64")
    rng = np.random.default_rng(5)
    g = np.linspace(-0.045, 0.045, 6)
    mesh = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pts = np.concatenate([mesh, rng.uniform(-0.05, 0.05, (100, 3))])
    u, _ = c.field_velocity(pts)
    p = opar(w, boundary=bc, velocity="BS", tree_theta=0.0)
    og = O.ghosts(p, w.x, w.infront, w.behind)
    uo = O.field_velocity(p, w.x, w.infront, og[0], pts)
    c.close()
    assert rel_max(u, uo) < 1e-10, rel_max(u, uo)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_root_estimate_gives_the_exact_walk(L, precision):
    """The walk started from the root centroid's bounded estimate (while the
    exact sequential sum runs alongside) returns the velocities and evaluation
    counts of the walk from the exact centroid, bit for bit: with the true
    bound (every root test decided), with a bound widened until some tests are
    undecided (the fix-up drops the images whose root is in fact far), and
    widened until the fix-up's list overflows (the gated second walk redoes
    every task)."""
    w = small_tangle()
    c = ctx_for(L, w, precision=precision)
    try:
        L.test_root_speculation(0)
        u0, _, _, ev0 = c.velocity()
        seen = []
        for scale in (1.0, 1e12, 1e13):
            L.test_root_speculation(1, scale)
            c.set_points(w.x, w.infront, w.behind)
            u, _, _, ev = c.velocity()
            seen.append(c.root_undecided())
            assert np.array_equal(u, u0), scale
            assert ev == ev0, scale
    finally:
        L.test_root_speculation(-1, 1.0)
        c.close()
    assert seen[0] == 0 and 0 < seen[1] <= 8192 < seen[2], seen


def test_root_estimate_gives_the_exact_walk_on_the_tangle(L):
    """Config 2's tangle (24.7k points, below the size that starts the walk
    from the estimate by itself): the mixed walk started from the root
    centroid's bounded estimate gives the velocities and evaluation counts of
    the walk from the exact centroid, bit for bit, whether the fix-up drops the
    undecided images or its list overflows and the gated walk redoes every
    task; the exact walk makes the FP64 walk's decisions (the same evaluation
    count) within 1e-6 RMS of its velocities."""
    w = W.tangle(0)
    c = ctx_for(L, w, precision="mixed")
    c64 = ctx_for(L, w, precision="fp64")
    try:
        L.test_root_speculation(0)
        u0, _, _, ev0 = c.velocity()
        u64, _, _, ev64 = c64.velocity()
        assert ev0 == ev64
        assert np.sqrt(((u0 - u64) ** 2).sum() / (u64 ** 2).sum()) < 1e-6
        seen = []
        for scale in (1.0, 3e10, 1e11, 3e11, 1e12, 1e13, 1e14):
            L.test_root_speculation(1, scale)
            c.set_points(w.x, w.infront, w.behind)
            u, _, _, ev = c.velocity()
            seen.append(c.root_undecided())
            assert np.array_equal(u, u0), scale
            assert ev == ev0, scale
    finally:
        L.test_root_speculation(-1, 1.0)
        c.close()
        c64.close()
    assert seen[0] == 0, seen
    assert any(0 < s <= 8192 for s in seen) and any(s > 8192 for s in seen), seen


# ----------------------------------------------- late level-1 moments (mixed)
@pytest.mark.parametrize("bc", ["periodic", "open"])
def test_late_level1_matches_the_inline_walk(L, bc):
    """A mixed Tree build that packs the big root children late (their circ
    and Cij sums still running when the walk starts: the unshifted image's
    tasks defer those cells' far-field terms, the images' tasks wait for the
    payloads) gives the walk of the inline build's decisions and evaluation
    counts; the deferred terms are added in FP64 after the compensated FP32
    sum instead of inside it, so the velocities differ by that rounding only
    (1e-7 RMS), and both are within 1e-6 RMS of the FP64 walk.  A second walk
    on the same tree, its payloads all in, takes every term inline and repeats
    the inline build's velocities bit for bit."""
    w = W.tangle(0)
    c = ctx_for(L, w, precision="mixed", boundary=bc)
    c64 = ctx_for(L, w, precision="fp64", boundary=bc)
    try:
        L.test_late_level1(0)
        u0, _, _, ev0 = c.velocity()
        L.test_late_level1(1)
        c.set_points(w.x, w.infront, w.behind)
        u1, _, _, ev1 = c.velocity()
        u2, _, _, ev2 = c.velocity()
        u64, _, _, ev64 = c64.velocity()
    finally:
        L.test_late_level1(-1)
        c.close()
        c64.close()
    assert ev1 == ev0 == ev2 == ev64
    assert np.array_equal(u2, u0)
    assert rel_rms(u1, u0) < 1e-7
    assert rel_rms(u1, u64) < 1e-6 and rel_rms(u0, u64) < 1e-6


def test_late_level1_with_the_root_estimate(L):
    """Late level-1 payloads together with the root centroid's bounded
    estimate: whether every root test is decided, the fix-up drops undecided
    images (and their deferred cells), or its list overflows and the gated
    walk redoes every task, the velocities and evaluation counts are those of
    the late build from the exact centroid, bit for bit."""
    w = W.tangle(0)
    c = ctx_for(L, w, precision="mixed")
    try:
        L.test_late_level1(1)
        L.test_root_speculation(0)
        c.set_points(w.x, w.infront, w.behind)
        u0, _, _, ev0 = c.velocity()
        seen = []
        for scale in (1.0, 3e10, 1e11, 3e11, 1e12, 1e13, 1e14):
            L.test_root_speculation(1, scale)
            c.set_points(w.x, w.infront, w.behind)
            u, _, _, ev = c.velocity()
            seen.append(c.root_undecided())
            assert np.array_equal(u, u0), scale
            assert ev == ev0, scale
    finally:
        L.test_root_speculation(-1, 1.0)
        L.test_late_level1(-1)
        c.close()
    assert seen[0] == 0, seen
    assert any(0 < s <= 8192 for s in seen) and any(s > 8192 for s in seen), seen


def test_late_level1_by_size(L):
    """80,843 points (above the size from which a mixed Tree build packs the
    big root children late by default): the default build against the inline
    one, same evaluation counts, 1e-7 RMS apart, both within 1e-6 RMS of the
    FP64 walk; and a few steps of the default loop keep the links and the
    candidate pairs of the inline build's steps."""
    w = W.large_tangle(0, n_rings=300)
    assert w.n >= 65536
    res = {}
    for mode in (-1, 0):
        L.test_late_level1(mode)
        try:
            c = ctx_for(L, w, precision="mixed", line_ops=2)
            u, _, _, ev = c.velocity()
            for it in range(1, 4):
                c.step(it)
            n = c.n
            inf, beh = c.get_links()
            cl, _ = c.get_closest()
            res[mode] = (u, ev, n, inf[:n].copy(), beh[:n].copy(), cl[:n].copy())
            c.close()
        finally:
            L.test_late_level1(-1)
    c64 = ctx_for(L, w, precision="fp64")
    u64, _, _, ev64 = c64.velocity()
    c64.close()
    (ua, eva, *sa), (ub, evb, *sb) = res[-1], res[0]
    assert eva == evb == ev64
    assert rel_rms(ua, ub) < 1e-7
    assert rel_rms(ua, u64) < 1e-6 and rel_rms(ub, u64) < 1e-6
    assert sa[0] == sb[0]
    for x, y in zip(sa[1:], sb[1:]):
        np.testing.assert_array_equal(x, y)
