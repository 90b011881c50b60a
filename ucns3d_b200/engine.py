"""Host-side mirror of UCNS3D's explicit time-stepping interface over the
CUDA engine's C ABI (include/ucns3d_gpu.h).

Method names follow the Fortran routines they replace:

    calculate_cfl(cfl)            CALCULATE_CFL             src/time_p.f90:27-191
    call_flux_subroutines_3d()    CALL_FLUX_SUBROUTINES_3D  src/time_p.f90:2253-2497
    runge_kutta3(dt)              RUNGE_KUTTA3              src/time_p.f90:885-1027
    time_marching(nsteps, cfl)    the CFL + RK3 part of TIME_MARCHING (src/time_p.f90:4026)

Errors come back as ``EngineError`` carrying the UCG_* code; there is no CPU
fallback: creating an Engine without a B200 raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class EngineError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{N.ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


class Engine:
    def __init__(self, mesh, cfg: N.UcgConfig, device: int = 0, upload: bool = True, tables: str = "host",
                 roles=None):
        """``tables``: "host" uploads the set-up library's reconstruction
        tables (ucg_upload_recon), "device" builds them on the GPU from the
        cell shapes (ucg_build_recon; the mesh may be prepared without
        tables).  ``roles`` (int8 per cell, a partition's: 0 owned, 1 ring 1,
        2 the rest of the halo; ucg_set_cell_roles) limits the work to what
        the owned cells need."""
        self.lib = N.engine()
        self.mesh = mesh
        self.cfg = cfg
        self.n = mesh.ncells
        h = C.c_void_p()
        rc = self.lib.ucg_create(C.byref(cfg), self.n, device, C.byref(h))
        if rc:
            raise EngineError(rc, self.lib.ucg_create_error().decode())
        self._h = h
        if roles is not None:
            self._roles = np.ascontiguousarray(roles, dtype=np.int8)
            if self._roles.shape != (self.n,):
                self.close()
                raise ValueError("one role per cell")
            self._check(self.lib.ucg_set_cell_roles(h, self._roles.ctypes.data_as(C.POINTER(C.c_int8))))
        if upload:
            self.upload_geometry(mesh.geometry_struct())
            if tables == "device":
                self.build_recon(mesh.shapes_struct(), mesh.recon_struct())
            else:
                self.upload_recon(mesh.recon_struct())

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self.lib.ucg_destroy(h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc:
            buf = C.create_string_buffer(1024)
            self.lib.ucg_last_error(self._h, buf, 1024)
            raise EngineError(rc, buf.value.decode())

    # ------------------------------------------------------------ set-up
    def upload_geometry(self, g: N.UcgGeometry):
        self._check(self.lib.ucg_upload_geometry(self._h, C.byref(g)))

    def upload_recon(self, r: N.UcgRecon):
        self._check(self.lib.ucg_upload_recon(self._h, C.byref(r)))

    def build_recon(self, s: N.UcgShapes, r: N.UcgRecon):
        """The reconstruction tables built on the device (ucg_build_recon)."""
        self._check(self.lib.ucg_build_recon(self._h, C.byref(s), C.byref(r)))

    # ------------------------------------------------------------- state
    def set_state(self, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (self.n, 5):
            raise ValueError(f"state must have shape ({self.n}, 5)")
        self._check(self.lib.ucg_set_state(self._h, N.ptr(U, C.c_double), self.n))

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.n, 5))
        self._check(self.lib.ucg_get_state(self._h, N.ptr(out, C.c_double), self.n))
        return out

    # ----------------------------------------------------------- stepping
    def calculate_cfl(self, cfl: float) -> float:
        dt = C.c_double()
        self._check(self.lib.ucg_compute_dt(self._h, cfl, C.byref(dt)))
        return dt.value

    def call_flux_subroutines_3d(self) -> np.ndarray:
        """RHS(I)%VAL of the current state, shape (n, 5)."""
        out = np.empty((self.n, 5))
        self._check(self.lib.ucg_residual(self._h, N.ptr(out, C.c_double)))
        return out

    residual = call_flux_subroutines_3d

    def runge_kutta3(self, dt: float):
        self._check(self.lib.ucg_rk3_step(self._h, dt))

    def rk3_stage(self, stage: int, dt: float):
        """One of the three stages of `runge_kutta3` (1, 2, 3, in order)."""
        self._check(self.lib.ucg_rk3_stage(self._h, stage, dt))

    # ------------------------------------------------------- partitions
    def halo_set(self, send_cells: np.ndarray, recv_cells: np.ndarray):
        """Rows this rank sends (its owned cells, per peer in the peer's
        order) and receives (halo cells), as cell indices of this mesh."""
        s = np.ascontiguousarray(send_cells, dtype=np.int32)
        r = np.ascontiguousarray(recv_cells, dtype=np.int32)
        self._check(self.lib.ucg_halo_set(self._h, N.ptr(s, C.c_int32), len(s), N.ptr(r, C.c_int32), len(r)))

    def halo_pack(self, stage: int, send_ptr: int):
        """Gather the send rows of stage `stage`'s input state into the device
        buffer at `send_ptr` ([nsend][5] FP64), on the engine's stream."""
        self._check(self.lib.ucg_halo_pack(self._h, stage, C.c_void_p(send_ptr)))

    def halo_unpack(self, stage: int, recv_ptr: int):
        """Scatter the device buffer at `recv_ptr` ([nrecv][5] FP64) into the
        receive rows of stage `stage`'s input state, on the engine's stream."""
        self._check(self.lib.ucg_halo_unpack(self._h, stage, C.c_void_p(recv_ptr)))

    def time_marching(self, nsteps: int, cfl: float):
        """nsteps of CALCULATE_CFL + RUNGE_KUTTA3 with dt kept on the device."""
        self._check(self.lib.ucg_step(self._h, cfl, nsteps))

    def last_dt(self) -> float:
        dt = C.c_double()
        self._check(self.lib.ucg_last_dt(self._h, C.byref(dt)))
        return dt.value

    def reduce(self, what: int) -> float:
        out = C.c_double()
        self._check(self.lib.ucg_reduce(self._h, what, C.byref(out)))
        return out.value

    def kinetic_energy(self) -> float:
        return self.reduce(N.UCG_REDUCE_KE)

    def enstrophy(self) -> float:
        """TOTENS of a periodic TGV run (ENSTROPHY_CALC); Navier-Stokes MUSCL."""
        return self.reduce(N.UCG_REDUCE_ENSTROPHY)

    def wall_loads(self, centre=None) -> np.ndarray:
        """COMPUTEFORCE in full (src/io.f90:18752-19000): FX, FY, FZ (pressure
        and, Navier-Stokes, viscous shear) and the pressure moments MX, MY,
        MZ about the cell centres `centre` (n, 3) (zero when None)."""
        out = np.zeros(6)
        cen = None if centre is None else np.ascontiguousarray(centre, dtype=np.float64)
        self._check(self.lib.ucg_wall_loads(self._h, None if cen is None else N.ptr(cen, C.c_double),
                                            N.ptr(out, C.c_double)))
        return out

    # ------------------------------------------- adjoint and tangent (FP64 MUSCL, Euler)
    def force(self) -> float:
        """Wall pressure force in x at the current state (COMPUTEFORCE, src/io.f90:18752)."""
        out = C.c_double()
        self._check(self.lib.ucg_force(self._h, C.byref(out)))
        return out.value

    def force_vjp(self) -> np.ndarray:
        """dJ/dU of the wall force at the current state, shape (n, 5)."""
        out = np.empty((self.n, 5))
        self._check(self.lib.ucg_force_vjp(self._h, N.ptr(out, C.c_double)))
        return out

    def residual_vjp(self, lam: np.ndarray):
        """(dR/dU)^T lam, shape (n, 5), and (dR/dp)^T lam, shape (5,)."""
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        mu, pbar = np.empty((self.n, 5)), np.empty(5)
        self._check(self.lib.ucg_residual_vjp(self._h, N.ptr(lam, C.c_double), N.ptr(mu, C.c_double),
                                              N.ptr(pbar, C.c_double)))
        return mu, pbar

    def residual_jvp(self, du: np.ndarray, dp: np.ndarray | None = None) -> np.ndarray:
        """(dR/dU) du + (dR/dp) dp, shape (n, 5)."""
        du = np.ascontiguousarray(du, dtype=np.float64)
        dp = None if dp is None else np.ascontiguousarray(dp, dtype=np.float64)
        out = np.empty((self.n, 5))
        self._check(self.lib.ucg_residual_jvp(self._h, N.ptr(du, C.c_double), N.ptr(dp, C.c_double),
                                              N.ptr(out, C.c_double)))
        return out

    def adjoint_run(self, nsteps: int, dt: float, every: int = 20, objective: int = N.UCG_OBJ_FORCE_X):
        """J after nsteps RK3 steps of fixed dt, dJ/dU0 (n, 5) and dJ/dp (5,);
        the state becomes the final state.  ``objective``: UCG_OBJ_FORCE_X
        (wall force, MUSCL) or UCG_OBJ_KE (domain kinetic energy, MUSCL or
        WENO/CWENO)."""
        J, g, gp = C.c_double(), np.empty((self.n, 5)), np.empty(5)
        self._check(self.lib.ucg_adjoint_run_obj(self._h, objective, nsteps, dt, every, C.byref(J),
                                                 N.ptr(g, C.c_double), N.ptr(gp, C.c_double)))
        return J.value, g, gp

    def tangent_run(self, nsteps: int, dt: float, dU0: np.ndarray, dp: np.ndarray | None = None,
                    objective: int = N.UCG_OBJ_FORCE_X):
        """J and its directional derivative along (dU0, dp) after nsteps
        RK3 steps of fixed dt; the state becomes the final state."""
        dU0 = np.ascontiguousarray(dU0, dtype=np.float64)
        dp = None if dp is None else np.ascontiguousarray(dp, dtype=np.float64)
        J, dJ = C.c_double(), C.c_double()
        self._check(self.lib.ucg_tangent_run_obj(self._h, objective, nsteps, dt, N.ptr(dU0, C.c_double),
                                                 N.ptr(dp, C.c_double), C.byref(J), C.byref(dJ)))
        return J.value, dJ.value

    def time_adjoint(self, reps: int = 5) -> dict:
        """Average device ms of the residual, its VJP and its JVP."""
        ms = (C.c_double * 3)()
        self._check(self.lib.ucg_time_adjoint(self._h, reps, ms))
        return dict(residual=ms[0], vjp=ms[1], jvp=ms[2])

    def time_kernels(self, reps: int = 5) -> dict:
        """Average device ms of the reconstruction, flux and time-step
        kernels (CUDA events on the engine stream)."""
        ms = (C.c_double * 4)()
        self._check(self.lib.ucg_time_kernels(self._h, reps, ms))
        return dict(recon=ms[0], flux=ms[1], cfl=ms[2], lsq=ms[3])

    def check_health(self):
        self._check(self.lib.ucg_check_health(self._h))

    def synchronize(self):
        self._check(self.lib.ucg_synchronize(self._h))

    def cell_order(self) -> dict:
        """The device numbering chosen at upload: whether the engine
        renumbered the cells, the caller's cell at each device position, and
        the gather costs (cache lines per warp and face slot) of the caller's
        order and of reverse Cuthill-McKee."""
        ren = C.c_int32()
        n2o = np.empty(self.n, dtype=np.int32)
        cost = np.zeros(2)
        self._check(self.lib.ucg_cell_order(self._h, C.byref(ren), N.ptr(n2o, C.c_int32), N.ptr(cost, C.c_double)))
        return dict(renumbered=bool(ren.value), n2o=n2o, cost_caller=float(cost[0]), cost_rcm=float(cost[1]))

    def implicit_step(self, cfl: float, nsteps: int = 1, nsweeps: int = 10):
        """`nsteps` implicit pseudo-time steps toward the steady state
        (IMPLICIT_TIMEs with `nsweeps` relaxation sweeps)."""
        self._check(self.lib.ucg_implicit_step(self._h, cfl, nsteps, nsweeps))

    def dual_time_step(self, dt: float, cfl: float, max_inner: int = 20, inner_tol: float = 1e-3,
                       nsweeps: int = 10) -> int:
        """One DUAL_TIME physical step dt (BDF2, implicit inner iterations
        at pseudo CFL `cfl`); returns the inner iterations taken."""
        it = C.c_int32()
        self._check(self.lib.ucg_dual_time_step(self._h, dt, cfl, max_inner, inner_tol, nsweeps, C.byref(it)))
        return int(it.value)

    def dual_time_step_explicit(self, dt: float, cfl: float, max_inner: int = 50, inner_tol: float = 1e-3) -> int:
        """One DUAL_TIME_EX physical step dt (BDF2, explicit pseudo-time
        iterations at pseudo CFL `cfl`); returns the inner iterations taken.
        The state afterwards is the next step's first iterate 2 U^n - U^{n-1}."""
        it = C.c_int32()
        self._check(self.lib.ucg_dual_time_step_explicit(self._h, dt, cfl, max_inner, inner_tol, C.byref(it)))
        return int(it.value)

    def mood_state(self) -> dict:
        """MOOD after the last RK3 stage (cfg.mood 1): MOOD_O per cell (1
        first order, 2 MUSCL, IORDER + 1 the target scheme) and RECALC (the
        cells whose next reconstruction may fall back to MUSCL), in the
        caller's cell order."""
        order = np.empty(self.n, dtype=np.int32)
        recalc = np.empty(self.n, dtype=np.int32)
        self._check(self.lib.ucg_mood_state(self._h, N.ptr(order, C.c_int32), N.ptr(recalc, C.c_int32)))
        return dict(order=order, recalc=recalc)

    @property
    def stream_ptr(self) -> int:
        return int(self.lib.ucg_get_stream(self._h) or 0)

    @property
    def launch_count(self) -> int:
        return int(self.lib.ucg_launch_count(self._h))

    @property
    def device_bytes(self) -> int:
        return int(self.lib.ucg_device_bytes(self._h))


def lift_drag(loads, aoa_deg: float, rres: float, ufreestream: float, vector=(1.0, 1.0, 1.0)):
    """CL and CD from the wall loads as COMPUTEFORCE forms them in the body
    frame (RFRAME 0, src/io.f90:18933-18941): the forces scaled by VECTORX,
    Y, Z, then lift = FZ cos a + FY cos a - FX sin a, drag = FX cos a +
    FY sin a + FZ sin a, and C = 2 force / (RRES u_inf^2)."""
    fx, fy, fz = (float(loads[k]) * float(vector[k]) for k in range(3))
    a = (aoa_deg / 180.0) * np.pi
    lift = (fz * np.cos(a)) + (fy * np.cos(a)) - (fx * np.sin(a))
    drag = (fx * np.cos(a)) + (fy * np.sin(a)) + (fz * np.sin(a))
    return (2.0 * lift) / (rres * ufreestream ** 2), (2.0 * drag) / (rres * ufreestream ** 2)
