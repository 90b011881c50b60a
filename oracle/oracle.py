"""ORACLE - test infrastructure only (tests/, __graft_entry__.smoke and the
cpu_baseline leg of bench.py).  ctypes wrapper of oracle/_build/liboracle.so,
the FP64 CPU restatement of the reference hot path (see
oracle/ucns3d_oracle.cpp).  Nothing in the ucns3d_b200 package imports this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build() -> None:
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        from ucns3d_b200 import _native as N
        L = C.CDLL(LIB)
        cfgp, geop, recp = C.POINTER(N.UcgConfig), C.POINTER(N.UcgGeometry), C.POINTER(N.UcgRecon)
        f64p = C.POINTER(C.c_double)
        L.orc_residual.restype = C.c_int
        L.orc_residual.argtypes = [cfgp, geop, recp, f64p, f64p]
        L.orc_face_values.restype = C.c_int
        L.orc_face_values.argtypes = [cfgp, geop, recp, f64p, f64p]
        L.orc_compute_dt.restype = C.c_int
        L.orc_compute_dt.argtypes = [cfgp, geop, f64p, C.c_double, f64p]
        L.orc_rk3_step.restype = C.c_int
        L.orc_rk3_step.argtypes = [cfgp, geop, recp, C.c_double, f64p]
        L.orc_rk3_stage.restype = C.c_int
        L.orc_rk3_stage.argtypes = [cfgp, geop, recp, C.c_double, C.c_int, f64p, f64p]
        L.orc_implicit_step.restype = C.c_int
        L.orc_implicit_step.argtypes = [cfgp, geop, recp, C.c_double, C.c_int, C.c_int, f64p]
        L.orc_dual_time_step.restype = C.c_int
        L.orc_dual_time_step.argtypes = [cfgp, geop, recp, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int,
                                         f64p, f64p, f64p, C.POINTER(C.c_int)]
        L.orc_dual_time_step_explicit.restype = C.c_int
        L.orc_dual_time_step_explicit.argtypes = [cfgp, geop, recp, C.c_double, C.c_double, C.c_int, C.c_double,
                                                  f64p, f64p, f64p, C.POINTER(C.c_int)]
        L.orc_rk3_step_mood.restype = C.c_int
        L.orc_rk3_step_mood.argtypes = [cfgp, geop, recp, C.c_double, f64p, C.POINTER(C.c_int8),
                                        C.POINTER(C.c_int32)]
        L.orc_hllc.restype = C.c_int
        L.orc_hllc.argtypes = [C.c_double, f64p, f64p, f64p]
        L.orc_boundary.restype = C.c_int
        L.orc_boundary.argtypes = [cfgp, C.c_int, f64p, f64p, f64p]
        L.orc_riemann.restype = C.c_int
        L.orc_riemann.argtypes = [C.c_int, C.c_double, f64p, f64p, f64p, f64p]
        L.orc_reduce.restype = C.c_int
        L.orc_reduce.argtypes = [geop, f64p, C.c_int, f64p]
        L.orc_force.restype = C.c_int
        L.orc_force.argtypes = [cfgp, geop, recp, f64p, f64p]
        L.orc_wall_loads.restype = C.c_int
        L.orc_wall_loads.argtypes = [cfgp, geop, recp, f64p, f64p, f64p]
        L.orc_enstrophy.restype = C.c_int
        L.orc_enstrophy.argtypes = [cfgp, geop, recp, f64p, f64p]
        _lib = L
    return _lib


def hllc(gamma, cl, cr):
    cl = np.ascontiguousarray(cl, dtype=np.float64)
    cr = np.ascontiguousarray(cr, dtype=np.float64)
    out = np.zeros(5)
    lib().orc_hllc(gamma, _p(cl), _p(cr), _p(out))
    return out


def boundary(cfg, code, angles, cl):
    """Ghost state of BOUNDARYS for one face (code, ANGLE1/ANGLE2, left state)."""
    angles = np.ascontiguousarray(angles, dtype=np.float64)
    cl = np.ascontiguousarray(cl, dtype=np.float64)
    out = np.zeros(5)
    if lib().orc_boundary(C.byref(cfg), code, _p(angles), _p(cl), _p(out)):
        raise ValueError(f"no boundary code {code}")
    return out


def riemann(kind, gamma, cl, cr, n):
    """Global-frame flux of Roe (3), rotated Roe-HLL (4) or t-Roe (5)."""
    cl, cr, n = (np.ascontiguousarray(a, dtype=np.float64) for a in (cl, cr, n))
    out = np.zeros(5)
    if lib().orc_riemann(kind, gamma, _p(cl), _p(cr), _p(n), _p(out)):
        raise ValueError(f"no global-frame Riemann solver {kind}")
    return out


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """CPU restatement bound to one prepared mesh and configuration."""

    def __init__(self, mesh, cfg):
        self.mesh = mesh
        self.cfg = cfg
        self.geo = mesh.geometry_struct()
        self.rec = mesh.recon_struct()
        self.n = mesh.ncells

    def residual(self, U: np.ndarray) -> np.ndarray:
        U = np.ascontiguousarray(U, dtype=np.float64)
        out = np.zeros_like(U)
        rc = lib().orc_residual(C.byref(self.cfg), C.byref(self.geo), C.byref(self.rec), _p(U), _p(out))
        if rc:
            raise RuntimeError(f"orc_residual failed: {rc}")
        return out

    def face_values(self, U: np.ndarray) -> np.ndarray:
        U = np.ascontiguousarray(U, dtype=np.float64)
        out = np.zeros((self.n, 6, 16, 5))
        rc = lib().orc_face_values(C.byref(self.cfg), C.byref(self.geo), C.byref(self.rec), _p(U), _p(out))
        if rc:
            raise RuntimeError(f"orc_face_values failed: {rc}")
        return out

    def compute_dt(self, U: np.ndarray, cfl: float) -> float:
        U = np.ascontiguousarray(U, dtype=np.float64)
        dt = C.c_double()
        rc = lib().orc_compute_dt(C.byref(self.cfg), C.byref(self.geo), _p(U), cfl, C.byref(dt))
        if rc:
            raise RuntimeError(f"orc_compute_dt failed: {rc}")
        return dt.value

    def rk3_step(self, U: np.ndarray, dt: float) -> np.ndarray:
        U = np.array(U, dtype=np.float64, copy=True, order="C")
        rc = lib().orc_rk3_step(C.byref(self.cfg), C.byref(self.geo), C.byref(self.rec), dt, _p(U))
        if rc:
            raise RuntimeError(f"orc_rk3_step failed: {rc}")
        return U

    def implicit_step(self, U: np.ndarray, cfl: float, nsteps: int = 1, nsweeps: int = 10) -> np.ndarray:
        """`nsteps` IMPLICIT_TIMEs steps (local time steps at `cfl`, `nsweeps`
        relaxation sweeps)."""
        U = np.array(U, dtype=np.float64, copy=True, order="C")
        rc = lib().orc_implicit_step(C.byref(self.cfg), C.byref(self.geo), C.byref(self.rec), cfl, nsteps, nsweeps,
                                     _p(U))
        if rc:
            raise RuntimeError(f"orc_implicit_step failed: {rc}")
        return U

    def dual_time_step(self, U: np.ndarray, hist: tuple, dt: float, cfl: float, maxit: int = 20,
                       tol: float = 1e-3, nsweeps: int = 10) -> tuple:
        """One DUAL_TIME physical step: (U, (U^n, U^{n-1}), inner iterations);
        hist is None before the first step."""
        U = np.array(U, dtype=np.float64, copy=True, order="C")
        U2, U3 = (U.copy(), U.copy()) if hist is None else (np.array(hist[0], copy=True), np.array(hist[1], copy=True))
        it = C.c_int()
        rc = lib().orc_dual_time_step(C.byref(self.cfg), C.byref(self.geo), C.byref(self.rec), dt, cfl, maxit, tol,
                                      nsweeps, _p(U), _p(U2), _p(U3), C.byref(it))
        if rc:
            raise RuntimeError(f"orc_dual_time_step failed: {rc}")
        return U, (U2, U3), it.value

    def dual_time_step_explicit(self, U: np.ndarray, hist: tuple, dt: float, cfl: float, maxit: int = 50,
                                tol: float = 1e-3) -> tuple:
        """One DUAL_TIME_EX physical step (explicit pseudo-time iterations):
        (U, (U^n, U^{n-1}), inner iterations); hist is None before the first
        step.  The returned U is the next step's first iterate 2 U^n - U^{n-1}."""
        U = np.array(U, dtype=np.float64, copy=True, order="C")
        U2, U3 = (U.copy(), U.copy()) if hist is None else (np.array(hist[0], copy=True), np.array(hist[1], copy=True))
        it = C.c_int()
        rc = lib().orc_dual_time_step_explicit(C.byref(self.cfg), C.byref(self.geo), C.byref(self.rec), dt, cfl,
                                               maxit, tol, _p(U), _p(U2), _p(U3), C.byref(it))
        if rc:
            raise RuntimeError(f"orc_dual_time_step_explicit failed: {rc}")
        return U, (U2, U3), it.value

    def rk3_step_mood(self, U: np.ndarray, dt: float, recalc: np.ndarray) -> tuple:
        """One RUNGE_KUTTA3_MOOD step (cfg.mood 1): the new state and MOOD_O per
        cell; recalc (int8 [n], RECALC, zero before the first step) is
        updated in place."""
        U = np.array(U, dtype=np.float64, copy=True, order="C")
        assert recalc.dtype == np.int8 and recalc.flags.c_contiguous and recalc.size == self.n
        order = np.zeros(self.n, dtype=np.int32)
        rc = lib().orc_rk3_step_mood(C.byref(self.cfg), C.byref(self.geo), C.byref(self.rec), dt, _p(U),
                                     recalc.ctypes.data_as(C.POINTER(C.c_int8)),
                                     order.ctypes.data_as(C.POINTER(C.c_int32)))
        if rc:
            raise RuntimeError(f"orc_rk3_step_mood failed: {rc}")
        return U, order

    def rk3_stage(self, Un: np.ndarray, U: np.ndarray, dt: float, stage: int) -> None:
        """Stage `stage` (1..3) of one RK3 step, in place on U (U = Un before stage 1)."""
        Un = np.ascontiguousarray(Un, dtype=np.float64)
        assert U.flags.c_contiguous and U.dtype == np.float64
        rc = lib().orc_rk3_stage(C.byref(self.cfg), C.byref(self.geo), C.byref(self.rec), dt, stage, _p(Un), _p(U))
        if rc:
            raise RuntimeError(f"orc_rk3_stage failed: {rc}")

    def force(self, U: np.ndarray) -> float:
        """Wall pressure force in x (COMPUTEFORCE, inviscid part)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        out = C.c_double()
        rc = lib().orc_force(C.byref(self.cfg), C.byref(self.geo), C.byref(self.rec), _p(U), C.byref(out))
        if rc:
            raise RuntimeError(f"orc_force failed: {rc}")
        return out.value

    def wall_loads(self, U: np.ndarray, centre=None) -> np.ndarray:
        """COMPUTEFORCE: FX, FY, FZ (pressure and, Navier-Stokes, shear) and
        the pressure moments MX, MY, MZ about the cell centres (zero without
        `centre` [n][3])."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        out = np.zeros(6)
        cen = None if centre is None else np.ascontiguousarray(centre, dtype=np.float64)
        rc = lib().orc_wall_loads(C.byref(self.cfg), C.byref(self.geo), C.byref(self.rec), _p(U),
                                  None if cen is None else _p(cen), _p(out))
        if rc:
            raise RuntimeError(f"orc_wall_loads failed: {rc}")
        return out

    def enstrophy(self, U: np.ndarray) -> float:
        """TOTENS of a periodic TGV run (ENSTROPHY_CALC), Navier-Stokes MUSCL."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        out = C.c_double()
        rc = lib().orc_enstrophy(C.byref(self.cfg), C.byref(self.geo), C.byref(self.rec), _p(U), C.byref(out))
        if rc:
            raise RuntimeError(f"orc_enstrophy failed: {rc}")
        return out.value

    def reduce(self, U: np.ndarray, what: int) -> float:
        U = np.ascontiguousarray(U, dtype=np.float64)
        out = C.c_double()
        lib().orc_reduce(C.byref(self.geo), _p(U), what, C.byref(out))
        return out.value
