"""The five benchmark workloads at their stated sizes and step counts: the
FP64 engine against the oracle, through the C ABI, on a B200.

1. Taylor-Green vortex, 32^3 hexahedra, MUSCL + HLLC + viscous fluxes,
   100 SSP-RK3 steps at CFL 0.5: the kinetic-energy history (the TGV sum of
   TIME_MARCHING, src/time_p.f90:4145-4198) at every step within 1e-10
   relative, and the final density and energy fields within 1e-10 of their
   largest magnitude.
2. 24^3 x 6 = 82,944 jittered tetrahedra, WENO3: the residual within 1e-12
   (of each cell's flux scale) at step 0 and after 50 steps, the 50-step
   trajectory within 1e-10, and the final state bit for bit equal across two
   runs.
3. 64^3 = 262,144 hexahedra, isentropic vortex, WENO5: one FP64 residual
   within 1e-12.
5. The 2,119,680-cell mixed hexahedron/pyramid/prism/tetrahedron box,
   CWENO4 + viscous fluxes: one FP64 residual within 1e-12; the mixed
   precision form's density against the FP64 form after 50 steps (relative
   L2 within 1e-6).

Every step uses the oracle's dt on both sides (the engine's own CFL dt is
checked against it to 1e-12), so that the two trajectories are comparable
step by step.  The fourth workload (the bump channel) is the adjoint's and
is checked at its stated size in tests/test_adjoint.py.
"""
import numpy as np
import pytest

from oracle import Oracle
from ucns3d_b200 import _native as N
from ucns3d_b200 import cases
from ucns3d_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _flux_scale(mesh, U, gamma=1.4):
    g = mesh.geometry()
    r, u = U[:, 0], U[:, 1:4] / U[:, :1]
    p = (gamma - 1.0) * (U[:, 4] - 0.5 * r * (u * u).sum(1))
    area = (g["face_area"] * (np.arange(6)[None, :] < g["nfaces"][:, None])).sum(1)
    s = np.abs(U).max(1) * (np.abs(u).max(1) + np.sqrt(gamma * p / r)) + p
    return (s * area)[:, None]


def _residual_err(e, o, mesh, U):
    e.set_state(U)
    Rg = e.call_flux_subroutines_3d()
    Ro = o.residual(U)
    return float((np.abs(Rg - Ro) / _flux_scale(mesh, U)).max())


def _rel_l2(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def test_tgv_32_muscl_ns_100_steps_ke_history():
    c = cases.tgv_hex_muscl(n=32)
    assert c.mesh.ncells == 32768
    o = Oracle(c.mesh, c.cfg)
    e = Engine(c.mesh, c.cfg)
    e.set_state(c.U0)
    Uo = c.U0.copy()
    ke_g, ke_o, dts = [], [], []
    for _ in range(100):
        dt = o.compute_dt(Uo, 0.5)
        dt_g = e.calculate_cfl(0.5)
        assert abs(dt_g - dt) <= 1e-12 * dt
        e.runge_kutta3(dt)
        Uo = o.rk3_step(Uo, dt)
        ke_g.append(e.kinetic_energy())
        ke_o.append(o.reduce(Uo, N.UCG_REDUCE_KE))
        dts.append(dt)
    e.check_health()
    ke_g, ke_o = np.array(ke_g), np.array(ke_o)
    ke_err = float((np.abs(ke_g - ke_o) / np.abs(ke_o)).max())
    Ug = e.get_state()
    rho_err = float(np.abs(Ug[:, 0] - Uo[:, 0]).max() / np.abs(Uo[:, 0]).max())
    en_err = float(np.abs(Ug[:, 4] - Uo[:, 4]).max() / np.abs(Uo[:, 4]).max())
    print(f"TGV 32^3, 100 steps (t = {sum(dts):.4f}): KE history max rel err {ke_err:.3e}, "
          f"density {rho_err:.3e}, energy {en_err:.3e}; KE {ke_o[0]:.10e} -> {ke_o[-1]:.10e}")
    assert ke_err < 1e-10
    assert rho_err < 1e-10 and en_err < 1e-10
    # the viscous flow decays: the history is not flat
    assert ke_o[-1] < ke_o[0]


@pytest.fixture(scope="module")
def tets():
    return cases.tgv_tet_weno3(n=24)


def test_tets_82944_weno3_50_steps(tets):
    c = tets
    assert c.mesh.ncells == 82944
    o = Oracle(c.mesh, c.cfg)
    e = Engine(c.mesh, c.cfg)
    err0 = _residual_err(e, o, c.mesh, c.U0)
    e.set_state(c.U0)
    Uo = c.U0.copy()
    for _ in range(50):
        dt = o.compute_dt(Uo, 0.5)
        assert abs(e.calculate_cfl(0.5) - dt) <= 1e-12 * dt
        e.runge_kutta3(dt)
        Uo = o.rk3_step(Uo, dt)
    e.check_health()
    Ug = e.get_state()
    traj = float((np.abs(Ug - Uo) / np.abs(Uo).max(0)).max())
    err50 = _residual_err(e, o, c.mesh, Ug)
    print(f"tets 82,944, WENO3: residual rel err step 0 {err0:.3e}, step 50 {err50:.3e}; "
          f"50-step state rel err {traj:.3e}")
    assert err0 < 1e-12
    assert err50 < 1e-12
    assert traj < 1e-10


def test_tets_82944_weno3_bitwise_deterministic(tets):
    c = tets
    out = []
    for _ in range(2):
        e = Engine(c.mesh, c.cfg)
        e.set_state(c.U0)
        e.time_marching(50, 0.5)
        out.append(e.get_state())
        e.close()
    assert np.array_equal(out[0], out[1])


def test_tets_82944_weno3_mixed_vs_fp64_50_steps(tets):
    c = tets
    cm = N.UcgConfig.from_buffer_copy(c.cfg)
    cm.precision = N.UCG_MIXED
    rho = []
    dt = None
    for cfg in (c.cfg, cm):
        e = Engine(c.mesh, cfg)
        e.set_state(c.U0)
        if dt is None:
            dt = e.calculate_cfl(0.5)
        for _ in range(50):
            e.runge_kutta3(dt)
        e.check_health()
        rho.append(e.get_state()[:, 0])
        e.close()
    l2 = _rel_l2(rho[1], rho[0])
    linf = float(np.abs(rho[1] - rho[0]).max() / np.abs(rho[0]).max())
    print(f"tets 82,944, WENO3, 50 steps: mixed vs FP64 density rel L2 {l2:.3e}, Linf {linf:.3e}")
    assert l2 < 1e-6


def test_vortex_64_weno5_fp64_residual():
    c = cases.vortex_hex_weno5(n=64)
    assert c.mesh.ncells == 262144
    o = Oracle(c.mesh, c.cfg)
    e = Engine(c.mesh, c.cfg)
    err = _residual_err(e, o, c.mesh, c.U0)
    e.close()
    print(f"vortex 64^3, WENO5, FP64: residual rel err {err:.3e}")
    assert err < 1e-12


def test_mixed_box_2m_cweno4_ns_fp64_residual_and_mixed_error():
    c = cases.mixed_cweno4(n=96)
    assert c.mesh.ncells == 2119680
    o = Oracle(c.mesh, c.cfg)
    e = Engine(c.mesh, c.cfg)
    err = _residual_err(e, o, c.mesh, c.U0)
    del o
    dt = e.calculate_cfl(0.5)
    for _ in range(50):
        e.runge_kutta3(dt)
    e.check_health()
    rho64 = e.get_state()[:, 0].copy()
    e.close()
    cm = N.UcgConfig.from_buffer_copy(c.cfg)
    cm.precision = N.UCG_MIXED
    em = Engine(c.mesh, cm)
    em.set_state(c.U0)
    for _ in range(50):
        em.runge_kutta3(dt)
    em.check_health()
    rho32 = em.get_state()[:, 0]
    em.close()
    l2 = _rel_l2(rho32, rho64)
    linf = float(np.abs(rho32 - rho64).max() / np.abs(rho64).max())
    print(f"mixed box 2,119,680 cells, CWENO4 NS: FP64 residual rel err {err:.3e}; 50 steps mixed vs FP64 "
          f"density rel L2 {l2:.3e}, Linf {linf:.3e}")
    assert err < 1e-12
    assert l2 < 1e-6
