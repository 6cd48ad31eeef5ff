"""The benchmarked step, as a whole loop, against the oracle.

qv_step with line_ops = 2 runs the reference's default time-loop body
(src/run.f90:41-93): ghostp, construct_tree, pmotion, pinsert, pclose_tree on
the tree built before the move, precon_original, premove, ghostp and
enforce_periodic.  oracle.Loop restates the same body on the CPU.  Both start
from the random-ring tangle (100 rings, N = 24,707, periodic L = 0.1, Barnes-Hut
theta 0.4), whose first steps reconnect, remove and insert points, and both run
20 steps; after every step the slot count, the links and the candidate pair
list must be identical and the positions and velocities close:

* FP64: positions within 1e-10 relative (max over active slots), velocities
  within 1e-10 relative, closestd within 1e-12 relative;
* mixed precision: the same links and pairs, and velocities within 1e-6 RMS
  relative of the oracle's FP64 velocities.

The large tangle (3000 rings, N = 802,906, theta 0.5) is checked on a seeded
1 % sample of its targets: the FP64 walk within 1e-10 of the oracle's
velocities, the mixed walk within 1e-6 RMS.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEPS = 20


def _mods():
    from qvort_b200 import lib as L
    from qvort_b200 import workloads as W

    return L, W


@pytest.fixture(scope="module")
def tangle_loop(nthreads):
    """The oracle's trajectory of the tangle under the default loop: per step
    the state after it (links, closest, closestd, x, u)."""
    _, W = _mods()
    w = W.tangle(0)
    lp = O.Loop(O.params(**w.params), w.x, w.infront, w.behind, line_ops=2, recon_shots=1,
                nthreads=nthreads)
    traj, totals = [], {"inserted": 0, "reconnected": 0, "removed": 0}
    for it in range(1, STEPS + 1):
        assert lp.step(it) == 0
        for k in totals:
            totals[k] += lp.counts[k]
        traj.append(lp.state())
    return w, traj, totals


def _rel_max(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def _run_gpu(w, precision, check):
    L, _ = _mods()
    c = L.Context(L.default_params(**dict(w.params, precision=precision, line_ops=2,
                                          recon_shots=1)))
    c.set_points(w.x, w.infront, w.behind)
    try:
        for it in range(1, STEPS + 1):
            c.step(it)
            x, u = c.get_points()
            inf, beh = c.get_links()
            cl, cd = c.get_closest()
            check(it, dict(x=x, u=u, infront=inf, behind=beh, closest=cl, closestd=cd))
    finally:
        c.close()


def test_default_loop_fp64_matches_oracle(tangle_loop):
    w, traj, totals = tangle_loop
    # the run exercises every line operation
    assert totals["inserted"] > 0 and totals["reconnected"] > 0 and totals["removed"] > 0

    def check(it, got):
        ref = traj[it - 1]
        n = ref["x"].shape[0]
        assert got["x"].shape[0] == n, (it, got["x"].shape[0], n)
        for k in ("infront", "behind", "closest"):
            assert np.array_equal(got[k], ref[k]), (it, k)
        act = ref["infront"] != 0
        assert _rel_max(got["x"][act], ref["x"][act]) < 1e-10, it
        assert _rel_max(got["u"][act], ref["u"][act]) < 1e-10, it
        assert _rel_max(got["closestd"][act], ref["closestd"][act]) < 1e-12, it

    _run_gpu(w, "fp64", check)


def test_default_loop_mixed_matches_oracle(tangle_loop):
    w, traj, _ = tangle_loop
    worst = [0.0]

    def check(it, got):
        ref = traj[it - 1]
        n = ref["x"].shape[0]
        assert got["x"].shape[0] == n, (it, got["x"].shape[0], n)
        # no decision of the line operations lies within the mixed error
        # here, so the links and the pair list are the oracle's exactly
        for k in ("infront", "behind", "closest"):
            assert np.array_equal(got[k], ref[k]), (it, k)
        act = ref["infront"] != 0
        e = _rms_rel(got["u"][act], ref["u"][act])
        worst[0] = max(worst[0], e)
        assert e < 1e-6, (it, e)

    _run_gpu(w, "mixed", check)
    assert worst[0] > 0.0  # the mixed path really differs from FP64


@pytest.fixture(scope="module")
def large_sample(nthreads):
    _, W = _mods()
    w = W.large_tangle()
    p = O.params(**w.params)
    g = O.ghosts(p, w.x, w.infront, w.behind)
    tree = O.Tree(p, w.x, g[0], w.infront)
    assert tree.status == 0
    rng = np.random.default_rng(2024)
    tg = np.sort(rng.choice(w.n, w.n // 100, replace=False)).astype(np.int32)
    u, _, _, ev, st = O.velocity(p, w.x, w.infront, w.behind, g, tree, targets=tg,
                                 nthreads=nthreads)
    assert st == 0
    tree.close()
    return w, tg, u, ev


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_large_tangle_sample_matches_oracle(large_sample, precision):
    L, _ = _mods()
    w, tg, u_ref, ev_ref = large_sample
    c = L.Context(L.default_params(**dict(w.params, precision=precision)))
    c.set_points(w.x, w.infront, w.behind)
    u, *_ = c.velocity(False)
    c.close()
    if precision == "fp64":
        assert _rel_max(u[tg], u_ref) < 1e-10
    else:
        assert _rms_rel(u[tg], u_ref) < 1e-6
