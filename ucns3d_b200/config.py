"""Engine configuration (ucg_config) from UCNS3D.DAT-style parameters.

Derived quantities follow src/parameters.f90: VISC = rho*U*L/Re
(parameters.f90:1241), R_gas = 1 when the free-stream speed is below 10
(parameters.f90:1223-1227), IORDER = spatialorder - 1 (parameters.f90:1276),
the WENO epsilon 10E-12 (reconstruct_p.f90:437) and KAPPA_VEN = 10
(reconstruct_p.f90:3436).
"""
from __future__ import annotations

from . import _native as N

NAVIER_STOKES = 1
EULER = 2


def make_config(mesh, governing: int = EULER, precision: int = N.UCG_FP64, gamma: float = 1.4,
                prandtl: float = 0.72, reynolds: float | None = None, rres: float = 1.0,
                ufreestream: float = 1.0, pres: float = 1.0, char_length: float = 1.0,
                lwci: float = 1000.0, wenoz: int = 0, limiter: int = 7,
                bc_state=(1.0, 0.0, 0.0, 0.0, 1.0), lamx: float = 1.0, wenwrt: int = 1,
                riemann: int = 1, boundtype: int = 1, reorder: int = 1, mood: int = 0, mood_mode: int = 1,
                mood_var=(1e-4, 1e-3, 1e-4, 1e-3)) -> N.UcgConfig:
    """A ucg_config for a prepared mesh.  ``reynolds`` sets VISC for
    Navier-Stokes; ``bc_state`` is the free-stream primitive state used by
    inflow/outflow/far-field boundaries; ``boundtype`` is BOUNDTYPE (0 supersonic
    inflow/outflow ghosts, 1 the characteristic subsonic treatment);
    ``wenwrt`` 1 reconstructs the conserved
    variables, 2 the characteristic variables (WENWRT of UCNS3D.DAT);
    ``riemann`` 1 HLLC, 2 Rusanov, 3 Roe, 4 rotated Roe-HLL, 5 t-Roe, 9 HLL
    (iRiemann); ``mood`` 1 turns on MOOD in the RK3 stages with MOOD_MODE
    ``mood_mode`` (1 relaxed, 0 original) and MOOD_VAR1-4 ``mood_var`` (the
    lines of MOOD.DAT)."""
    if not getattr(mesh, "prepared", False):
        raise ValueError("mesh must be prepared first")
    cfg = N.UcgConfig()
    mesh.fill_config(cfg)
    cfg.governing = governing
    cfg.wenwrt = wenwrt
    cfg.limiter = limiter
    cfg.riemann = riemann
    cfg.precision = precision
    cfg.wenoz = wenoz
    cfg.gamma = gamma
    cfg.prandtl = prandtl
    cfg.rres = rres
    cfg.pres = pres
    cfg.r_gas = 1.0 if ufreestream < 10.0 else 287.052874
    if governing == NAVIER_STOKES:
        if not reynolds:
            raise ValueError("Navier-Stokes needs a Reynolds number")
        cfg.visc = rres * ufreestream * char_length / reynolds
    else:
        cfg.visc = 0.0
    cfg.lwci = lwci
    cfg.weno_eps = 10e-12
    cfg.kappa_ven = 10.0
    cfg.lamx = lamx
    cfg.boundtype = boundtype
    cfg.reorder = reorder
    cfg.mood = mood
    cfg.mood_mode = mood_mode
    for k in range(4):
        cfg.mood_var[k] = mood_var[k]
    for k in range(5):
        cfg.bc_state[k] = bc_state[k]
    return cfg
