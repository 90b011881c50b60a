"""Generates tests/golden/bc_kat.json: known-answer vectors of the ghost
states of UCNS3D's physical boundaries (BOUNDARYS,
src/flow_operations.f90:2860-3375) for codes 1 (inflow), 2 (outflow),
3 (symmetry), 4 (inviscid wall, ITESTCASE 3) and 6 (far field) under
BOUNDTYPE 0 and 1, from an independent numpy restatement written from the
Fortran text: the 5x5 rotation matrices of ROTATEF/ROTATEB
(src/grid_t.f90:4217-4305) built entry by entry and applied with a matrix
product, the face normal NX = cos a1 sin a2, NY = sin a1 sin a2,
NZ = cos a2, and the SUBSON1/2/3 formulas with SKINS/IKINS.  INFLOW and
OUTFLOW (flow_operations.f90:1161, 1526) return the free stream
(RRES, uvel, vvel, wvel, PRES).

    python tests/golden/make_bc_golden.py
"""
import json
import os

import numpy as np

TOLSMALL = 1.0e-13


def rotation(a1, a2):
    t = np.zeros((5, 5))
    t[0, 0] = 1.0
    t[1, 1], t[1, 2], t[1, 3] = np.cos(a1) * np.sin(a2), np.sin(a1) * np.sin(a2), np.cos(a2)
    t[2, 1], t[2, 2], t[2, 3] = np.cos(a1) * np.cos(a2), np.sin(a1) * np.cos(a2), -np.sin(a2)
    t[3, 1], t[3, 2] = -np.sin(a1), np.cos(a1)
    t[4, 4] = 1.0
    return t


def inv_rotation(a1, a2):
    t = np.zeros((5, 5))
    t[0, 0] = 1.0
    t[1, 1], t[1, 2], t[1, 3] = np.cos(a1) * np.sin(a2), np.cos(a1) * np.cos(a2), -np.sin(a1)
    t[2, 1], t[2, 2], t[2, 3] = np.sin(a1) * np.sin(a2), np.sin(a1) * np.cos(a2), np.cos(a1)
    t[3, 1], t[3, 2] = np.cos(a2), -np.sin(a2)
    t[4, 4] = 1.0
    return t


def to_prim(g, u):
    r = u[0]
    vel = u[1:4] / r
    return np.array([r, *vel, (g - 1.0) * (u[4] - 0.5 * r * (vel @ vel))])


def to_cons(g, w):
    skins = 0.5 * (w[1] ** 2 + w[2] ** 2 + w[3] ** 2)
    ikins = w[4] / ((g - 1.0) * w[0])
    return np.array([w[0], w[1] * w[0], w[2] * w[0], w[3] * w[0], w[0] * ikins + w[0] * skins])


def sub_in(s1, s2, sps, n):
    s3 = np.zeros(5)
    s3[4] = 0.5 * (s1[4] + s2[4] - s2[0] * sps * (n @ (s1[1:4] - s2[1:4])))
    s3[0] = s1[0] + (s3[4] - s1[4]) / sps ** 2
    s3[1:4] = s1[1:4] - n * (s1[4] - s3[4]) / (sps * s2[0])
    return s3


def sub_out(s1, s2, sps, n):
    s3 = np.zeros(5)
    s3[4] = s1[4]
    s3[0] = s2[0] + (s3[4] - s2[4]) / sps ** 2
    s3[1:4] = s2[1:4] + n * (s2[4] - s3[4]) / (sps * s2[0])
    return s3


def boundarys(code, boundtype, g, free, a1, a2, left, navier_stokes=False):
    """Ghost state RIGHTV of BOUNDARYS for the conserved LEFTV `left`."""
    n = np.array([np.cos(a1) * np.sin(a2), np.sin(a1) * np.sin(a2), np.cos(a2)])
    inflow = to_cons(g, free)
    s2 = to_prim(g, left)
    sps = np.sqrt(g * s2[4] / s2[0])
    vel = np.sqrt(s2[1] ** 2 + s2[2] ** 2 + s2[3] ** 2)
    if code == 1:
        if boundtype == 0 or vel / (sps + TOLSMALL) > 1.0:
            return inflow
        return to_cons(g, sub_in(free, s2, sps, n))
    if code == 2:
        if boundtype == 0 or vel / (sps + TOLSMALL) > 1.0:
            return left.copy()
        return to_cons(g, sub_out(free, s2, sps, n))
    if code == 4 and navier_stokes:  # ITESTCASE 4: no slip
        return np.array([left[0], -left[1], -left[2], -left[3], left[4]])
    if code in (3, 4):
        rot = rotation(a1, a2) @ left
        rot[1] = -rot[1]
        return inv_rotation(a1, a2) @ rot
    if code == 6:
        vnb = (rotation(a1, a2) @ left)[1]
        if vnb <= 0.0:
            if abs(vnb) >= sps:
                return inflow
            return to_cons(g, sub_in(free, s2, sps, n))
        if abs(vnb) >= sps:
            return left.copy()
        return to_cons(g, sub_out(free, s2, sps, n))
    raise ValueError(code)


def main():
    g = 1.4
    rng = np.random.default_rng(20251203)
    free = np.array([1.0, 0.675 * np.sqrt(1.4), 0.05, -0.02, 1.0])
    states = []
    # hand-picked left states (primitive) and face angles: subsonic and
    # supersonic, flow into and out of the domain, and |rho u_n| >= c with
    # |u| < c (far-field branch on the normal momentum)
    picks = [((1.0, 0.3, 0.1, 0.0, 1.0), 0.3, 1.2), ((1.0, -0.3, 0.1, 0.0, 1.0), 0.3, 1.2),
             ((1.0, 2.5, 0.2, 0.1, 1.0), 0.0, np.pi / 2), ((1.0, -2.5, 0.2, 0.1, 1.0), 0.0, np.pi / 2),
             ((3.0, 0.9, 0.0, 0.0, 1.0), 0.0, np.pi / 2), ((3.0, -0.9, 0.0, 0.0, 1.0), 0.0, np.pi / 2),
             ((0.5, 0.1, -0.4, 0.3, 0.7), 2.1, 0.4), ((1.2, 0.0, 0.0, -1.8, 1.1), 1.0, np.pi)]
    for w, a1, a2 in picks:
        states.append((np.array(w, dtype=float), a1, a2))
    for _ in range(16):
        w = np.array([rng.uniform(0.3, 3.0), *rng.uniform(-2.0, 2.0, 3), rng.uniform(0.3, 3.0)])
        states.append((w, rng.uniform(-np.pi, np.pi), rng.uniform(0.0, np.pi)))
    cases = []
    for code in (1, 2, 3, 4, 6):
        for bt in (0, 1):
            for ns in ((False, True) if code == 4 else (False,)):
                for w, a1, a2 in states:
                    left = to_cons(g, w)
                    cases.append({"code": code, "boundtype": bt, "governing": 1 if ns else 2,
                                  "angles": [float(a1), float(a2)], "left": left.tolist(),
                                  "ghost": boundarys(code, bt, g, free, a1, a2, left, ns).tolist()})
    out = {"gamma": g, "free_stream": free.tolist(), "cases": cases}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "bc_kat.json"), "w") as fh:
        json.dump(out, fh, indent=0)


if __name__ == "__main__":
    main()
