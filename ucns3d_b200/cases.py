"""The benchmark workloads, as seeded synthetic meshes.

No dataset is involved: the reference's own test mesh is not available, so
each workload is generated with the shapes, sizes and value distributions of
its description.

1. ``tgv_hex_muscl``   Taylor-Green vortex, periodic [0,2pi]^3, n^3 hexahedra
   (32^3 = 32,768 cells), Navier-Stokes, Mach 0.1, Re 1600, Pr 0.71, MUSCL +
   Venkatakrishnan + HLLC, SSP-RK3, CFL 0.5.
2. ``tgv_tet_weno3``   the same vortex (Euler) on n^3 hexahedra split into 6
   tetrahedra each (24^3*6 = 82,944), vertices jittered +-0.15h, WENO order 3.
3. ``vortex_hex_weno5`` isentropic vortex (strength 5, gamma 1.4) advected at
   Mach 0.5 along (1,1,0), periodic [0,10]^3 with n^3 hexahedra (64^3 =
   262,144), Euler, WENO order 5.
4. ``bump_muscl``      channel with a 10 % sinusoidal bump, 240x80 quads split
   50/50 into triangles, 4 layers (hexahedra + prisms), Euler, Mach 0.675
   inflow, subsonic outflow, slip walls, MUSCL.
5. ``mixed_cweno4``    Taylor-Green vortex on a periodic n^3 box of hexahedra,
   pyramids, tetrahedra and prisms, Navier-Stokes, CWENO order 4.

The Taylor-Green initial condition is that of UCNS3D's INITCOND 95
(src/profile.f90:253-288) without its shift by -pi (the shift only flips the
sign of the velocity field); p0 = 1/(gamma M^2) sets the Mach number.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .config import EULER, NAVIER_STOKES, make_config
from .mesh import IC_TGV, IC_UNIFORM, IC_VORTEX, SCHEME_MUSCL, SCHEME_WENO, Mesh

GAMMA = 1.4


@dataclass
class Case:
    name: str
    mesh: Mesh
    cfg: N.UcgConfig
    U0: np.ndarray
    cfl: float
    steps: int
    meta: dict = field(default_factory=dict)


def _tgv_params(mach=0.1):
    return [GAMMA, 1.0 / (GAMMA * mach * mach), 1.0]


def tgv_hex_muscl(n=32, precision=N.UCG_FP64, nthreads=0) -> Case:
    m = Mesh.box_hex(n, n, n).prepare(SCHEME_MUSCL, 1, nthreads=nthreads)
    p0 = _tgv_params()[1]
    cfg = make_config(m, governing=NAVIER_STOKES, precision=precision, prandtl=0.71, reynolds=1600.0,
                      rres=1.0, ufreestream=1.0, pres=p0)
    U0 = m.initial_condition(IC_TGV, _tgv_params())
    return Case("tgv_hex_muscl", m, cfg, U0, 0.5, 100, dict(n=n, scheme="MUSCL", order=2, equations="NS"))


def tgv_tet_weno3(n=24, precision=N.UCG_FP64, jitter=0.15, seed=1234, nthreads=0) -> Case:
    m = Mesh.box_tet(n, n, n, jitter=jitter, seed=seed).prepare(SCHEME_WENO, 2, nthreads=nthreads)
    p0 = _tgv_params()[1]
    cfg = make_config(m, governing=EULER, precision=precision, pres=p0, lwci=1000.0)
    U0 = m.initial_condition(IC_TGV, _tgv_params())
    return Case("tgv_tet_weno3", m, cfg, U0, 0.5, 50, dict(n=n, scheme="WENO", order=3, equations="Euler"))


def vortex_params(L=10.0, t=0.0, mach=0.5, strength=5.0):
    c = math.sqrt(GAMMA)
    u = mach * c / math.sqrt(2.0)
    return [GAMMA, strength, u, u, 0.0, 0.5 * L, 0.5 * L, 0.5 * L, t, L, L, L]


def vortex_hex_weno5(n=64, precision=N.UCG_FP64, L=10.0, nthreads=0, wenwrt=1) -> Case:
    m = Mesh.box_hex(n, n, n, L=(L, L, L)).prepare(SCHEME_WENO, 4, nthreads=nthreads)
    cfg = make_config(m, governing=EULER, precision=precision, pres=1.0, lwci=1000.0, wenwrt=wenwrt)
    U0 = m.initial_condition(IC_VORTEX, vortex_params(L))
    return Case("vortex_hex_weno5", m, cfg, U0, 0.5, 200, dict(n=n, L=L, scheme="WENO", order=5, equations="Euler"))


def bump_muscl(nx=240, ny=80, nlayers=4, precision=N.UCG_FP64, seed=1234, nthreads=0) -> Case:
    m = Mesh.bump_channel(nx, ny, nlayers, seed=seed).prepare(SCHEME_MUSCL, 1, nthreads=nthreads)
    mach = 0.675
    u = mach * math.sqrt(GAMMA * 1.0 / 1.0)
    cfg = make_config(m, governing=EULER, precision=precision, pres=1.0, bc_state=(1.0, u, 0.0, 0.0, 1.0))
    U0 = m.initial_condition(IC_UNIFORM, [GAMMA, 1.0, u, 0.0, 0.0, 1.0])
    return Case("bump_muscl", m, cfg, U0, 0.5, 200, dict(nx=nx, ny=ny, scheme="MUSCL", order=2, equations="Euler"))


def mixed_cweno4(n=96, precision=N.UCG_FP64, seed=1234, nthreads=0) -> Case:
    m = Mesh.mixed_box(n, seed=seed).prepare(SCHEME_WENO, 3, ees=5, nthreads=nthreads)
    p0 = _tgv_params()[1]
    cfg = make_config(m, governing=NAVIER_STOKES, precision=precision, prandtl=0.71, reynolds=1600.0,
                      pres=p0, lwci=1000.0)
    U0 = m.initial_condition(IC_TGV, _tgv_params())
    return Case("mixed_cweno4", m, cfg, U0, 0.5, 50, dict(n=n, scheme="CWENO", order=4, equations="NS"))


CASES = {
    "tgv_hex_muscl": tgv_hex_muscl,
    "tgv_tet_weno3": tgv_tet_weno3,
    "vortex_hex_weno5": vortex_hex_weno5,
    "bump_muscl": bump_muscl,
    "mixed_cweno4": mixed_cweno4,
}


def bytes_per_cell_stage(cfg: N.UcgConfig, nfaces: int = 6, table_bytes: int | None = None) -> int:
    """Algorithmic bytes of one cell-stage (state, tables, geometry), the
    per-unit figure of the HBM roofline; neighbour state counted once."""
    s = table_bytes if table_bytes is not None else (4 if cfg.precision == N.UCG_MIXED else 8)
    ideg, imax, A = cfg.ideg, cfg.imax, cfg.admis_max
    nq = max(cfg.nq_quad, cfg.nq_tri)
    b = 3 * 5 * 8                                  # read U, read U^n, write U
    if cfg.ees == 5:
        b += s * (ideg * imax + cfg.ideg2 * cfg.imax2 * (A - 1))
        b += 4 * (imax + cfg.imax2 * (A - 1))
        b += s * (ideg * ideg + cfg.ideg2 * cfg.ideg2)
    else:
        b += s * ideg * imax * A
        b += 4 * imax * A
        if cfg.scheme == 3:
            b += s * ideg * ideg
    b += 8 * nfaces * nq * 3                       # face quadrature points
    b += 8 * nfaces * 4 + 4 * nfaces + 16          # normal+area, neighbour ids, volume+MINEDGE
    if cfg.governing == 1:
        b += 8 * (9 + nfaces)                      # Jacobian, DIH
    return b
