"""Generate the committed golden fixtures in this folder.

segment_kat.npz -- known-answer vectors for the velocity induced at a point
    P by a closed triangular loop A -> B -> C -> A, computed independently of
    the code under test in 50-digit decimal arithmetic from the classical
    finite-segment Biot-Savart law u = G/(4 pi h) (cos a1 - cos a2) e (h the
    distance of P from the segment's line, a1/a2 the angles at its two ends),
    summed over the three segments.  Both pair forms of the reference
    (src/timestep.f90:472-479 and src/tree.f90:380-390) must reproduce these to
    rounding.
ring_kat.npz -- the analytic self-induced speed, energy and momentum of a thin
    ring that the reference prints at set-up (src/initial_loop.f90:17-19).

Run: python tests/golden/make_golden.py
"""
from decimal import Decimal, getcontext
from pathlib import Path

import numpy as np

getcontext().prec = 50
HERE = Path(__file__).resolve().parent
G = Decimal("9.97e-4")
PI = Decimal("3.14159265358979323846264338327950288419716939937510")


def dsqrt(x):
    return x.sqrt()


def seg_velocity(P, A, B):
    P = [Decimal(repr(float(v))) for v in P]
    A = [Decimal(repr(float(v))) for v in A]
    B = [Decimal(repr(float(v))) for v in B]
    s = [B[k] - A[k] for k in range(3)]
    L = dsqrt(sum(c * c for c in s))
    t = [c / L for c in s]
    ap = [P[k] - A[k] for k in range(3)]
    proj = sum(ap[k] * t[k] for k in range(3))
    foot = [A[k] + proj * t[k] for k in range(3)]
    hv = [P[k] - foot[k] for k in range(3)]
    h = dsqrt(sum(c * c for c in hv))
    # cos of the angles between the segment direction and the rays to P
    r1 = ap
    r2 = [P[k] - B[k] for k in range(3)]
    c1 = sum(r1[k] * t[k] for k in range(3)) / dsqrt(sum(c * c for c in r1))
    c2 = sum(r2[k] * t[k] for k in range(3)) / dsqrt(sum(c * c for c in r2))
    mag = G / (4 * PI * h) * (c1 - c2)
    # direction t x (P - foot) / h
    e = [t[1] * hv[2] - t[2] * hv[1], t[2] * hv[0] - t[0] * hv[2], t[0] * hv[1] - t[1] * hv[0]]
    return [float(mag * e[k] / h) for k in range(3)]


def main():
    rng = np.random.default_rng(20240601)
    m = 48
    rows = []
    for k in range(m):
        # target P on its own two-point loop (P <-> P2): the reference skips both
        # of its segments (j == i, j == behind(i)) and its LIA term is zero, so
        # the velocity at P is the field of the triangle loop A -> B -> C -> A.
        P = rng.uniform(-0.04, 0.04, 3)
        P2 = P + rng.normal(size=3) * 1e-4
        size = 10 ** rng.uniform(-4.5, -2.5)
        cen = P + rng.normal(size=3) / 1.0 * 10 ** rng.uniform(-4, -1.6)
        A, B, Cc = (cen + rng.normal(size=3) * size for _ in range(3))
        U = np.zeros(3)
        for a_, b_ in ((A, B), (B, Cc), (Cc, A)):
            U += np.array(seg_velocity(P, a_, b_))
        rows.append((P, P2, A, B, Cc, U))
    arr = {name: np.array([r[i] for r in rows]) for i, name in enumerate("P P2 A B C U".split())}
    np.savez(HERE / "segment_kat.npz", gamma=float(G), **arr)
    R, a = 0.01, 1.3e-8
    Gf = float(G)
    v = Gf / (4 * np.pi * R) * (np.log(8 * R / a) - 0.5)
    E = 0.5 * Gf ** 2 * R * (np.log(8 * R / a) - 2.0)
    Pm = Gf * np.pi * R ** 2
    np.savez(HERE / "ring_kat.npz", R=R, a=a, gamma=Gf, speed=v, energy=E, momentum=Pm)
    print("wrote", HERE / "segment_kat.npz", HERE / "ring_kat.npz")


if __name__ == "__main__":
    main()
