"""GPU tests of the hand-written derivatives against central finite differences.

Tolerance: 1e-5 relative on directional derivatives (the bar the adjoint is
built to).  The FP64 forward maps are smooth between tree opening decisions;
steps of 1e-7 (1e-8 with the tree, so that no decision flips) balance the
truncation error against the rounding noise of the forward sums.  The rings
are placed so that none crosses the box: with open boundaries a wrapped ring
would contain a box-long segment, whose near-singular Biot-Savart terms make
any difference quotient rounding-dominated.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mods():
    import torch

    from qvort_b200 import adjoint as A
    from qvort_b200 import lib as L
    from qvort_b200 import workloads as W

    return torch, A, L, W


def _system(W, L, A, velocity="BS", boundary="open", theta=0.0, order=2, precision="fp64",
            seed=4, n_rings=6):
    w = W.random_rings(n_rings, 0.006, 0.01, 5e-4, 0.1, seed=seed, centre_box=0.05)
    prm = dict(w.params, velocity=velocity, boundary=boundary, tree_theta=theta,
               deriv_order=order, precision=precision)
    return w, A.FilamentSystem(L.default_params(**prm), w.infront, w.behind)


def _dirderiv_fd(f, x, d, h):
    return (f(x + h * d) - f(x - h * d)) / (2 * h)


@pytest.mark.parametrize("velocity,boundary,theta,order", [
    ("BS", "open", 0.0, 2), ("BS", "periodic", 0.0, 2), ("BS", "open", 0.0, 4),
    ("Tree", "periodic", 0.5, 2), ("LIA", "open", 0.0, 2)])
def test_velocity_vjp_matches_fd(velocity, boundary, theta, order):
    torch, A, L, W = _mods()
    w, sysm = _system(W, L, A, velocity, boundary, theta, order)
    rng = np.random.default_rng(1)
    x = torch.tensor(w.x, device="cuda")
    ub = torch.tensor(rng.normal(size=w.x.shape), device="cuda")
    xr = x.clone().requires_grad_(True)
    u = A.velocity(xr, sysm)
    (xb,) = torch.autograd.grad((u * ub).sum(), xr)
    worst = 0.0
    for k in range(3):
        d = torch.tensor(rng.normal(size=w.x.shape), device="cuda")
        d /= d.norm()
        f = lambda y: float((A.velocity(y, sysm) * ub).sum())
        fd = _dirderiv_fd(f, x, d, 1e-7 if velocity != "Tree" else 1e-8)
        an = float((xb * d).sum())
        worst = max(worst, abs(fd - an) / abs(an))
    sysm.close()
    assert worst < 1e-5, worst


@pytest.mark.parametrize("order", [2, 4])
def test_energy_grad_matches_fd(order):
    torch, A, L, W = _mods()
    w, sysm = _system(W, L, A, order=order)
    rng = np.random.default_rng(2)
    x = torch.tensor(w.x, device="cuda")
    u = torch.tensor(rng.normal(size=w.x.shape) * 0.1, device="cuda")
    xr, ur = x.clone().requires_grad_(True), u.clone().requires_grad_(True)
    e = A.energy(xr, ur, sysm)
    xb, ubar = torch.autograd.grad(e, (xr, ur))
    for k in range(2):
        d = torch.tensor(rng.normal(size=w.x.shape), device="cuda")
        d /= d.norm()
        fx = _dirderiv_fd(lambda y: float(A.energy(y, u, sysm)), x, d, 1e-7)
        fu = _dirderiv_fd(lambda v: float(A.energy(x, v, sysm)), u, d, 1e-6)
        assert abs(fx - float((xb * d).sum())) <= 1e-5 * abs(fx)
        assert abs(fu - float((ubar * d).sum())) <= 1e-5 * abs(fu)
    sysm.close()


def test_energy_matches_the_path_energy():
    torch, A, L, W = _mods()
    w, sysm = _system(W, L, A)
    c = L.Context(sysm.params)
    c.set_points(w.x, w.infront, w.behind)
    u, *_ = c.velocity()
    e_ref = c.energy()
    x = torch.tensor(w.x, device="cuda")
    e = float(A.energy(x, torch.tensor(u, device="cuda"), sysm))
    assert e == pytest.approx(e_ref, rel=1e-12)
    sysm.close()


def test_trajectory_loss_gradient_matches_fd():
    """Gradient of E(x_K) + sum|x_K - x_0|^2 after K AB steps (checkpointed
    every 4 steps) w.r.t. x_0, against central differences of the same loss."""
    torch, A, L, W = _mods()
    w, sysm = _system(W, L, A, boundary="periodic", n_rings=4)
    K = 10
    val, g = A.gradient(w.x, sysm, K, checkpoint_every=4)
    rng = np.random.default_rng(3)
    x = torch.tensor(w.x, device="cuda")
    worst = 0.0
    for k in range(4):
        d = rng.normal(size=w.x.shape)
        d /= np.linalg.norm(d)
        dd = torch.tensor(d, device="cuda")
        with torch.no_grad():
            f = lambda y: float(A.loss(y, sysm, K, checkpoint_every=4))
            fd = _dirderiv_fd(f, x, dd, 1e-7)
        an = float((g * d).sum())
        worst = max(worst, abs(fd - an) / abs(an))
    sysm.close()
    assert worst < 1e-5, worst


def test_mixed_tree_gradient_matches_fp64_tree_gradient():
    """The fast path's gradient (mixed-precision Barnes-Hut forward) against the
    reference gradient from the FP64 velocity (same tree decisions)."""
    torch, A, L, W = _mods()
    grads = []
    for prec in ("mixed", "fp64"):
        w, sysm = _system(W, L, A, "Tree", "periodic", 0.5, precision=prec, n_rings=8)
        grads.append(A.gradient(w.x, sysm, 8, checkpoint_every=4)[1])
        sysm.close()
    rel = np.linalg.norm(grads[0] - grads[1]) / np.linalg.norm(grads[1])
    assert rel < 1e-5, rel


@pytest.mark.parametrize("grad_images", [False, True])
def test_field_velocity_and_exact_gradient(grad_images):
    torch, A, L, W = _mods()
    w, sysm = _system(W, L, A, boundary="periodic")
    c = L.Context(sysm.params)
    c.set_points(w.x, w.infront, w.behind)
    rng = np.random.default_rng(5)
    pts = rng.uniform(-0.04, 0.04, (5, 3))
    u, du = c.field_velocity(pts, grad_images)
    h = 1e-7
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        up, _ = c.field_velocity(pts + e, grad_images)
        um, _ = c.field_velocity(pts - e, grad_images)
        if not grad_images:
            # velocity_quasip differentiates the unshifted sum only
            q = L.default_params(**dict(w.params, boundary="open"))
            c2 = L.Context(q)
            c2.set_points(w.x, w.infront, w.behind)
            up, _ = c2.field_velocity(pts + e)
            um, _ = c2.field_velocity(pts - e)
            c2.close()
        fd = (up - um) / (2 * h)
        np.testing.assert_allclose(du[:, :, k], fd, rtol=1e-5, atol=1e-9 * np.abs(du).max())
    c.close()
    sysm.close()


def test_trefoil_trajectory_gradient_fd_check():
    """The differentiation configuration's check at reduced size: trefoil rings
    (mode-3 perturbation, seeded 1e-5 cm displacement), periodic, FP64 direct
    velocity, K=32 steps checkpointed every 16, central differences along
    seeded unit directions.  The step is 1e-7 cm: at 1e-9 cm the rounding
    noise of the loss (an energy summed over all points) divided by h reaches
    1e-6..6e-5 of the directional derivative on this system."""
    torch, A, L, W = _mods()
    from qvort_b200 import gradcheck as G

    w = W.trefoil_rings(seed=0, n_rings=4, pts_per_ring=64)
    r = G.fd_check(w, steps=32, dirs=8, hs=(1e-7,), velocity="BS", tree_theta=0.0)
    assert r["by_h"]["1e-07"]["rel_max"] < 1e-5, r["by_h"]
    m = G.mixed_vs_fp64(w, steps=32, velocity="Tree", tree_theta=0.4)
    assert m["rel"] < 1e-5, m


def test_ab_step_is_the_step_update_bitwise_and_its_vjp_is_the_transpose():
    """qv_ab_step_device takes the update kernel's operations: from the same
    positions, velocities and history it gives the positions qv_step_ab +
    qv_enforce_periodic store, bit for bit, on every rung of the ladder.  Its
    adjoint is the transpose of the (piecewise linear) map: <xo_bar, J d> =
    <J^T xo_bar, d> for random directions d in (x, u, u1, u2, u3)."""
    torch, A, L, W = _mods()
    w, sysm = _system(W, L, A, "BS", "periodic", 0.0)
    n = w.n
    rng = np.random.default_rng(8)
    hist = [rng.normal(size=(n, 3)) for _ in range(3)]
    rung = rng.integers(1, 5, n)         # 1: Euler ... 4: AB4
    for k in range(3):
        hist[k][rung <= k + 1] = 0.0     # u1 = 0 for Euler, u2 = 0 for AB2, u3 = 0 for AB3
    # the context's own update and wrap, from its own velocities
    c = L.Context(sysm.params)
    c.set_points(w.x, w.infront, w.behind)
    c.set_history(*hist)
    u = c.velocity(False)[0]
    c.step_ab()
    c.enforce_periodic()
    x_ref, _ = c.get_points()
    c.close()
    # the differentiable step from the same inputs
    xt = torch.tensor(w.x, device="cuda")
    ut = torch.tensor(u, device="cuda")
    ht = [torch.tensor(h, device="cuda") for h in hist]
    sysm.load(xt)
    xo = A.ab_step(xt, ut, *ht, sysm)
    assert np.array_equal(xo.cpu().numpy(), x_ref)
    # adjoint = transpose (steps small enough that no point crosses the box)
    ins = [xt.clone().requires_grad_(True), ut.clone().requires_grad_(True)] + \
          [h.clone().requires_grad_(True) for h in ht]
    xob = torch.tensor(rng.normal(size=(n, 3)), device="cuda")
    out = A.ab_step(*ins, sysm)
    grads = torch.autograd.grad((out * xob).sum(), ins)
    # a zero history entry selects the rung: perturb only the nonzero ones
    masks = [torch.ones(n, 3, device="cuda")] * 2 + [(h != 0).double() for h in ht]
    for _ in range(3):
        ds = [torch.tensor(rng.normal(size=(n, 3)), device="cuda") * 1e-9 * m for m in masks]
        with torch.no_grad():
            jd = (A.ab_step(*[a + d for a, d in zip(ins, ds)], sysm) -
                  A.ab_step(*[a - d for a, d in zip(ins, ds)], sysm)) / 2
        lhs = float((xob * jd).sum())
        rhs = float(sum((g * d).sum() for g, d in zip(grads, ds)))
        assert abs(lhs - rhs) <= 1e-6 * abs(rhs), (lhs, rhs)
    sysm.close()
