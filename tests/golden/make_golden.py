"""Generates tests/golden/hllc_kat.json: known-answer vectors of the HLLC
flux used by UCNS3D (HLLC_RIEMANN_SOLVER, src/riemann.f90:221-426), from an
independent numpy restatement of that formula: Einfeldt-type wave speeds from
Roe averages clipped to SL <= 0 <= SR, contact speed SM, star states, and the
sign(SM) selection of the star flux.

    python tests/golden/make_golden.py
"""
import json
import os

import numpy as np


def hllc(g, UL, UR):
    def prim(U):
        r = U[0]
        u, v, w = U[1] / r, U[2] / r, U[3] / r
        p = (g - 1) * (U[4] - 0.5 * r * (u * u + v * v + w * w))
        return r, u, v, w, p

    rl, ul, vl, wl, pl = prim(UL)
    rr, ur, vr, wr, pr = prim(UR)
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    sl_, sr_ = np.sqrt(rl), np.sqrt(rr)
    ct = np.sqrt((cl ** 2 * sl_ + cr ** 2 * sr_) / (sl_ + sr_) + 0.5 * sl_ * sr_ / (sl_ + sr_) ** 2 * (ur - ul) ** 2)
    ut = (ul * sl_ + ur * sr_) / (sl_ + sr_)
    SL = min(ul - cl, ut - ct, 0.0)
    SR = max(ur + cr, ut + ct, 0.0)
    SM = (pr - pl + rl * ul * (SL - ul) - rr * ur * (SR - ur)) / (rl * (SL - ul) - rr * (SR - ur))

    def side(U, r, u, v, w, p, S):
        F = np.array([r * u, r * u * u + p, r * u * v, r * u * w, u * (U[4] + p)])
        m = r * (S - u) / (S - SM)
        Us = m * np.array([1.0, SM, v, w, U[4] / r + (SM - u) * (SM + p / (r * (S - u)))])
        return F + S * (Us - U)

    return side(UL, rl, ul, vl, wl, pl, SL) if SM >= 0 else side(UR, rr, ur, vr, wr, pr, SR)


def cons(g, r, u, v, w, p):
    return np.array([r, r * u, r * v, r * w, p / (g - 1) + 0.5 * r * (u * u + v * v + w * w)])


def main():
    g = 1.4
    rng = np.random.default_rng(20240601)
    cases = []
    fixed = [((1.0, 0.0, 0.0, 0.0, 1.0), (0.125, 0.0, 0.0, 0.0, 0.1)),   # Sod
             ((1.0, -2.0, 0.0, 0.0, 0.4), (1.0, 2.0, 0.0, 0.0, 0.4)),     # 123 problem
             ((1.0, 0.5, 0.2, -0.1, 1.0), (1.0, 0.5, 0.2, -0.1, 1.0)),    # uniform
             ((5.99924, 19.5975, 0, 0, 460.894), (5.99242, -6.19633, 0, 0, 46.095))]
    for a, b in fixed:
        cases.append((cons(g, *a), cons(g, *b)))
    for _ in range(12):
        a = (rng.uniform(0.1, 3), *rng.uniform(-2, 2, 3), rng.uniform(0.1, 5))
        b = (rng.uniform(0.1, 3), *rng.uniform(-2, 2, 3), rng.uniform(0.1, 5))
        cases.append((cons(g, *a), cons(g, *b)))
    out = {"gamma": g, "cases": [{"left": L.tolist(), "right": R.tolist(), "flux": hllc(g, L, R).tolist()}
                                 for L, R in cases]}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "hllc_kat.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()
