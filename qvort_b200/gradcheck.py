"""Central-difference check of the trajectory-loss gradient on trefoil rings.

The loss is the filament kinetic energy plus the squared displacement of the
points after K Adams-Bashforth steps (qvort_b200.adjoint.loss), its gradient
with respect to the initial positions comes from the hand-written adjoint, and
this module compares that gradient with central differences
(L(x0 + h d) - L(x0 - h d)) / 2h along seeded unit directions d, and with the
gradient obtained from the FP64 velocity when the forward runs in mixed
precision.

  python -m qvort_b200.gradcheck [--rings 16] [--pts 200] [--steps 256]
      [--dirs 64] [--h 1e-9 1e-8 1e-7] [--velocity BS] [--theta 0.0] [--dt 1e-7]

prints one JSON object.  Central differences need a forward map that is
smooth along d: FP64 velocities (the mixed forward's FP32 rounding is far
above h), no Barnes-Hut opening decision that flips within +-h (direct sums,
or tree runs whose decisions are far from their thresholds), and a time step
inside the Adams-Bashforth stability limit of the geometry (otherwise the
gradient is that of an exponentially unstable map, which no difference
quotient resolves).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import adjoint as A
from . import lib as L
from . import workloads as W


def system(w: W.Workload, **over) -> A.FilamentSystem:
    prm = dict(w.params)
    prm.update(over)
    return A.FilamentSystem(L.default_params(**prm), w.infront, w.behind)


def fd_check(w: W.Workload, steps: int, dirs: int, hs=(1e-9,), seed: int = 0,
             checkpoint_every: int = 16, **over) -> dict:
    """Gradient of the FP64 forward against central differences along `dirs`
    seeded unit directions, for each step h in `hs`; relative error
    |fd - g.d| / |g.d| per direction."""
    s = system(w, precision="fp64", **over)
    t0 = time.perf_counter()
    val, g = A.gradient(w.x, s, steps, checkpoint_every)
    t_grad = time.perf_counter() - t0
    rng = np.random.default_rng(seed)
    x = torch.tensor(w.x, device=s.device)
    rel = {h: [] for h in hs}
    with torch.no_grad():
        for _ in range(dirs):
            d = rng.normal(size=w.x.shape)
            d /= np.linalg.norm(d)
            dd = torch.tensor(d, device=s.device)
            an = float((g * d).sum())
            for h in hs:
                fp = float(A.loss(x + h * dd, s, steps, checkpoint_every))
                fm = float(A.loss(x - h * dd, s, steps, checkpoint_every))
                fd = (fp - fm) / (2.0 * h)
                rel[h].append(abs(fd - an) / max(abs(an), 1e-300))
    s.close()
    by_h = {}
    for h, r in rel.items():
        r = np.asarray(r)
        by_h[repr(h)] = {"rel_max": float(r.max()), "rel_median": float(np.median(r)),
                         "rel_all": [float(v) for v in r]}
    return {"loss": val, "grad_norm": float(np.linalg.norm(g)), "directions": dirs,
            "by_h": by_h, "grad_seconds": t_grad, "gradient": g}


def mixed_vs_fp64(w: W.Workload, steps: int, checkpoint_every: int = 16, **over) -> dict:
    """Relative 2-norm difference between the gradient of the mixed-precision
    forward and the gradient of the FP64 forward (both through the FP64 adjoint)."""
    gs = {}
    for prec in ("mixed", "fp64"):
        s = system(w, precision=prec, **over)
        gs[prec] = A.gradient(w.x, s, steps, checkpoint_every)[1]
        s.close()
    num = np.linalg.norm(gs["mixed"] - gs["fp64"])
    return {"rel": float(num / np.linalg.norm(gs["fp64"]))}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--rings", type=int, default=16)
    ap.add_argument("--pts", type=int, default=200)
    ap.add_argument("--steps", type=int, default=256)
    ap.add_argument("--dirs", type=int, default=64)
    ap.add_argument("--h", type=float, nargs="+", default=[1e-9, 1e-8, 1e-7])
    ap.add_argument("--velocity", default="BS", choices=["BS", "Tree", "LIA"])
    ap.add_argument("--theta", type=float, default=0.0)
    ap.add_argument("--dt", type=float, default=1e-7)
    ap.add_argument("--checkpoint-every", type=int, default=16)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--smooth", action="store_true",
                    help="smooth seeded displacement (the spacing stays near its mean)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-vs-FP64 gradient")
    a = ap.parse_args(argv)
    w = W.trefoil_rings(seed=a.seed, n_rings=a.rings, pts_per_ring=a.pts, smooth=a.smooth)
    over = dict(velocity=a.velocity, tree_theta=a.theta, dt=a.dt)
    dtm = W.dt_max(w)
    out = {"system": f"{a.rings} trefoil rings x {a.pts} points (N={w.n}), "
                     f"{'smooth' if a.smooth else 'per-point'} seeded displacement",
           "steps": a.steps, "checkpoint_every": a.checkpoint_every, **over,
           "dt_max_at_actual_spacing": dtm, "dt_passes_timestep_check": a.dt < dtm}
    r = fd_check(w, a.steps, a.dirs, tuple(a.h), a.seed, a.checkpoint_every, **over)
    r.pop("gradient")
    out["fd"] = r
    if not a.no_mixed:
        out["mixed_vs_fp64"] = mixed_vs_fp64(w, a.steps, a.checkpoint_every, **over)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
