"""Seeded synthetic filament systems for the benchmark and test configurations.

No external dataset is involved: every configuration is generated from a
numpy Generator seed.  Geometry follows the reference's own set-up routines
where one exists -- the single ring of setup_single_loop
(src/initial_loop.f90:11-38: points at angles pi(2i-1)/N, x = R sin, y = R cos),
the leap-frogging pair of setup_leap_frog (src/initial_loop.f90:206-245, the
second ring 2*delta above the first) and the random rings of
setup_random_loops (src/initial_loop.f90:850-960, spacing 0.75*delta).  The box
is centred at the origin, [-L/2, L/2) (src/tree.f90:49).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

GAMMA_HE4 = 9.97e-4   # quant_circ default, cm^2/s
CORE_A = 1.3e-8       # core radius used by the benchmark configurations, cm


@dataclass
class Workload:
    name: str
    x: np.ndarray          # (n, 3) float64
    infront: np.ndarray    # (n,) int32, 1-based, 0 = empty
    behind: np.ndarray     # (n,) int32
    params: dict = field(default_factory=dict)
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.x.shape[0]


def _ring_links(start: int, m: int):
    """1-based infront/behind for a closed loop of m points starting at slot start+1."""
    idx = np.arange(m)
    inf = start + (idx + 1) % m + 1
    beh = start + (idx - 1) % m + 1
    return inf.astype(np.int32), beh.astype(np.int32)


def _basis(normal: np.ndarray):
    n = normal / np.linalg.norm(normal)
    a = np.array([1.0, 0.0, 0.0]) if abs(n[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    e1 = np.cross(n, a)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(n, e1)
    return e1, e2


def wrap(x: np.ndarray, L: float) -> np.ndarray:
    """enforce_periodic (src/periodic.f90:188-214) applied once."""
    x = x.copy()
    h = L / 2.0
    x[x > h] -= L
    x[x < -h] += L
    return x


def ring(n: int = 200, radius: float = 0.01, perturb: float = 1e-5, seed: int = 0,
         box: float = 0.1, dt: float = 1e-7, delta: float = 5e-4) -> Workload:
    """Configuration 1: one ring in the xy-plane, radial noise perturb*U(-1,1)."""
    rng = np.random.default_rng(seed)
    i = np.arange(1, n + 1)
    ang = np.pi * (2 * i - 1) / n
    r = radius + perturb * rng.uniform(-1.0, 1.0, n)
    x = np.stack([r * np.sin(ang), r * np.cos(ang), np.zeros(n)], axis=1)
    inf, beh = _ring_links(0, n)
    params = dict(boundary="open", velocity="BS", tree_theta=0.0, box_size=box, dt=dt,
                  delta=delta, quant_circ=GAMMA_HE4, corea=CORE_A)
    return Workload("ring", x, inf, beh, params, dict(radius=radius))


def random_rings(n_rings: int, rmin: float, rmax: float, delta: float, box: float = 0.1,
                 seed: int = 0, spacing: float = 0.75, theta: float = 0.4,
                 dt: float = 1e-7, name: str = "tangle", centre_box: float | None = None) -> Workload:
    """Rings with radius U(rmin, rmax), centres uniform in the box (or in a cube
    of side centre_box about the origin), normals uniform on the sphere, point
    spacing spacing*delta, wrapped into the periodic box."""
    rng = np.random.default_rng(seed)
    xs, infs, behs = [], [], []
    start = 0
    for _ in range(n_rings):
        R = rng.uniform(rmin, rmax)
        m = max(5, int(round(2 * np.pi * R / (spacing * delta))))
        cb = box if centre_box is None else centre_box
        c = rng.uniform(0.0, cb, 3) - cb / 2.0
        nrm = rng.normal(size=3)
        e1, e2 = _basis(nrm)
        k = np.arange(1, m + 1)
        ang = np.pi * (2 * k - 1) / m
        pts = c + R * (np.sin(ang)[:, None] * e1 + np.cos(ang)[:, None] * e2)
        xs.append(pts)
        inf, beh = _ring_links(start, m)
        infs.append(inf)
        behs.append(beh)
        start += m
    x = wrap(np.concatenate(xs), box)
    params = dict(boundary="periodic", velocity="Tree", tree_theta=theta, box_size=box, dt=dt,
                  delta=delta, quant_circ=GAMMA_HE4, corea=CORE_A)
    return Workload(name, x, np.concatenate(infs), np.concatenate(behs), params,
                    dict(n_rings=n_rings))


def tangle(seed: int = 0) -> Workload:
    """Configuration 2: 100 random rings, R ~ U(0.008, 0.02), delta 5e-4, L 0.1,
    periodic, Barnes-Hut theta 0.4 (N ~ 22k)."""
    return random_rings(100, 0.008, 0.02, 5e-4, 0.1, seed, theta=0.4, name="tangle")


def large_tangle(seed: int = 0, n_rings: int = 3000) -> Workload:
    """Configuration 3: 3000 random rings, R ~ U(0.004, 0.015), delta 3e-4,
    periodic, theta 0.5 (N ~ 0.8M)."""
    return random_rings(n_rings, 0.004, 0.015, 3e-4, 0.1, seed, theta=0.5, name="large")


def trefoil_rings(seed: int = 0, n_rings: int = 16, pts_per_ring: int = 3125,
                  radius: float = 0.01, amp: float = 5e-4, noise: float = 1e-5,
                  box: float = 0.1, smooth: bool = False) -> Workload:
    """Configuration 4: rings of radius 0.01 with an azimuthal mode-3 radial
    perturbation of amplitude amp and a seeded displacement of noise, random
    centres and orientations in a periodic box (N = n_rings * pts_per_ring).

    smooth=False: every point is displaced independently by noise*U(-1,1) per
    coordinate.  At 3125 points per ring (spacing 2e-5 cm) that leaves segments
    down to ~1e-6 cm, and dt = 1e-7 s is then far beyond the reference's
    timestep_check bound (src/initial.f90:606-622) evaluated at that spacing.
    smooth=True: the seeded displacement is a sum of random Fourier modes 4..16
    along each ring, scaled to a largest displacement of noise, so the spacing
    stays within a few percent of its mean and the bound evaluated at the
    smallest actual spacing (dt_max of this module) is ~1.8e-8 s."""
    rng = np.random.default_rng(seed)
    xs, infs, behs = [], [], []
    start = 0
    for _ in range(n_rings):
        c = rng.uniform(-box / 4, box / 4, 3)
        e1, e2 = _basis(rng.normal(size=3))
        k = np.arange(1, pts_per_ring + 1)
        ang = np.pi * (2 * k - 1) / pts_per_ring
        r = radius + amp * np.cos(3 * ang)
        pts = c + r[:, None] * (np.sin(ang)[:, None] * e1 + np.cos(ang)[:, None] * e2)
        if smooth:
            disp = np.zeros_like(pts)
            for m in range(4, 17):
                coef = rng.normal(size=(2, 3))
                disp += np.cos(m * ang)[:, None] * coef[0] + np.sin(m * ang)[:, None] * coef[1]
            pts = pts + noise * disp / np.abs(disp).max()
        else:
            pts = pts + noise * rng.uniform(-1.0, 1.0, pts.shape)
        xs.append(pts)
        inf, beh = _ring_links(start, pts_per_ring)
        infs.append(inf)
        behs.append(beh)
        start += pts_per_ring
    x = wrap(np.concatenate(xs), box)
    params = dict(boundary="periodic", velocity="BS", tree_theta=0.0, box_size=box, dt=1e-7,
                  delta=5e-4, quant_circ=GAMMA_HE4, corea=CORE_A)
    return Workload("trefoil", x, np.concatenate(infs), np.concatenate(behs), params,
                    dict(n_rings=n_rings))


def leap_frog(n: int, radius: float, delta: float, seed: int = 0, box: float = 0.1) -> Workload:
    """Two coaxial rings (setup_leap_frog): n/2 points each, the second 2*delta above."""
    m = n // 2
    k = np.arange(1, m + 1)
    ang = np.pi * (2 * k - 1) / m
    a = np.stack([radius * np.sin(ang), radius * np.cos(ang), np.zeros(m)], axis=1)
    b = a.copy()
    b[:, 2] = 2.0 * delta
    inf1, beh1 = _ring_links(0, m)
    inf2, beh2 = _ring_links(m, m)
    x = np.concatenate([a, b])
    params = dict(boundary="open", velocity="BS", tree_theta=0.0, box_size=box, dt=1e-7,
                  delta=delta, quant_circ=GAMMA_HE4, corea=CORE_A)
    return Workload("leap_frog", x, np.concatenate([inf1, inf2]), np.concatenate([beh1, beh2]),
                    params)


def batch_systems(n_systems: int = 512, seed: int = 0, nmin: int = 100, nmax: int = 8000,
                  direct_below: int = 2000) -> list[Workload]:
    """Configuration 5: independent open systems, each a single ring
    (R ~ U(0.005, 0.02)) or a leap-frogging pair, N log-uniform in [nmin, nmax],
    dt from {5e-8, 1e-7, 2e-7}; direct sum below direct_below points, else
    Barnes-Hut theta 0.4, each in its own box of side 0.1 centred on it."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n_systems):
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        n += n % 2
        R = rng.uniform(0.005, 0.02)
        dt = float(rng.choice([5e-8, 1e-7, 2e-7]))
        if rng.uniform() < 0.5:
            w = ring(n, R, 1e-5, seed=int(rng.integers(1 << 30)))
        else:
            w = leap_frog(n, R, 2 * np.pi * R / (n // 2))
            w.x[:, 2] -= w.x[:, 2].mean()
        w.params.update(dt=dt)
        if n >= direct_below:
            w.params.update(velocity="Tree", tree_theta=0.4)
        w.name = f"sys{s}"
        out.append(w)
    return out


def dt_max(w: Workload) -> float:
    """timestep_check (src/initial.f90:606-622) with delta taken as the smallest
    actual segment length of the system: dt_max = d^2 / |G ln(d / (pi a))|,
    d = min segment / 2."""
    act = np.flatnonzero(w.infront)
    seg = np.linalg.norm(w.x[w.infront[act] - 1] - w.x[act], axis=1)
    box = w.params.get("box_size", 0.1)
    seg = seg[seg < box / 2]  # a segment that crosses a periodic face is short once unwrapped
    d = seg.min() / 2.0
    return float(d * d / abs(w.params["quant_circ"] * np.log(d / (np.pi * w.params["corea"]))))
