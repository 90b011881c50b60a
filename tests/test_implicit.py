"""Implicit pseudo-time steps toward a steady state (RUNGEKUTTA = 10:
IMPLICIT_TIMEs, src/time_p.f90:2783-2905; RELAXATION, CALCULATE_JACOBIAN,
CALCULATE_CFLL): the oracle's convergence on the CPU and (marked gpu) the
engine against the oracle.

Both relax in the same block-Jacobi form (every sweep reads the previous
sweep's corrections), so after several steps the engine's state agrees
with the oracle's to 1e-10 of its magnitude; the differences come from the
residual's evaluation order (each face once on the GPU, each cell's faces
in the oracle)."""
import numpy as np
import pytest

from oracle import Oracle
from ucns3d_b200 import cases
from ucns3d_b200.config import EULER, NAVIER_STOKES, make_config
from ucns3d_b200.mesh import IC_TGV, SCHEME_MUSCL, SCHEME_WENO, Mesh


def _bump(gov=EULER):
    c = cases.bump_muscl(nx=24, ny=8, nlayers=4)
    if gov == NAVIER_STOKES:
        cfg = make_config(c.mesh, governing=NAVIER_STOKES, reynolds=200.0, pres=1.0,
                          bc_state=tuple(c.cfg.bc_state))
        return c.mesh, cfg, c.U0
    return c.mesh, c.cfg, c.U0


def _farfield():
    """Far-field faces on both ends of a box, subsonic flow along x that
    varies in x, y and z (a state uniform along x ties the limiter's bounds,
    and a 1e-15 change of it moves the oracle's own result by 1e-1 after two
    steps)."""
    m = Mesh.box_hex(10, 6, 6, L=(3.0, 1.0, 1.0), periodic=(0, 1, 1), bc=(6, 6, 0, 0, 0, 0)).prepare(SCHEME_MUSCL, 1)
    bc = (1.0, 0.5, 0.0, 0.0, 1.0)
    cfg = make_config(m, governing=EULER, bc_state=bc)
    c = m.centres()
    rho = 1.0 + 0.2 * np.sin(2 * np.pi * c[:, 1]) + 0.1 * np.cos(2 * np.pi * c[:, 0] / 3.0 + 0.4)
    ux = 0.5 + 0.1 * np.sin(2 * np.pi * c[:, 0] / 3.0 + 1.1) * np.cos(2 * np.pi * c[:, 2])
    uy = 0.05 * np.sin(2 * np.pi * c[:, 1] + 0.3)
    U = np.zeros((m.ncells, 5))
    U[:, 0], U[:, 1], U[:, 2], U[:, 4] = rho, rho * ux, rho * uy, 1.0 / 0.4 + 0.5 * rho * (ux * ux + uy * uy)
    return m, cfg, U


def _tgv(scheme, iorder, gov, mk):
    m = mk().prepare(scheme, iorder)
    kw = dict(reynolds=100.0, pres=71.43) if gov == NAVIER_STOKES else {}
    cfg = make_config(m, governing=gov, **kw)
    U = m.initial_condition(IC_TGV, [1.4, 71.43 if gov == NAVIER_STOKES else 5.0, 1.0])
    return m, cfg, U


CASES = {
    "muscl_bump": lambda: _bump(),
    "muscl_ns_bump": lambda: _bump(NAVIER_STOKES),
    "muscl_farfield": _farfield,
    "weno3_tet_tgv": lambda: _tgv(SCHEME_WENO, 2, EULER, lambda: Mesh.box_tet(5, 5, 5, seed=3)),
    "muscl_ns_hex_tgv": lambda: _tgv(SCHEME_MUSCL, 1, NAVIER_STOKES, lambda: Mesh.box_hex(8, 8, 8)),
}


def test_oracle_implicit_steps_converge():
    """The bump channel from the free stream: 40 implicit steps at CFL 50
    take the residual norm below a tenth of its start (the explicit RK3
    stability limit is CFL 1)."""
    m, cfg, U = _bump()
    o = Oracle(m, cfg)
    r0 = np.linalg.norm(o.residual(U))
    U = o.implicit_step(U, 50.0, 40, 10)
    r1 = np.linalg.norm(o.residual(U))
    print(f"residual norm {r0:.3e} -> {r1:.3e}")
    assert np.isfinite(U).all() and r1 < 0.1 * r0


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_engine_implicit_steps_match_oracle(name):
    from ucns3d_b200.engine import Engine
    m, cfg, U = CASES[name]()
    o = Oracle(m, cfg)
    Uo = o.implicit_step(U, 20.0, 5, 10)
    e = Engine(m, cfg)
    e.set_state(U)
    e.implicit_step(20.0, 5, 10)
    e.check_health()
    Ug = e.get_state()
    err = np.abs(Ug - Uo).max() / np.abs(Uo).max()
    moved = np.abs(Uo - U).max() / np.abs(U).max()
    print(f"{name}: state rel err {err:.3e} (state moved {moved:.3e})")
    assert moved > 1e-6
    assert err < 1e-10


@pytest.mark.gpu
def test_engine_implicit_converges_and_agrees_with_explicit_steady_state():
    """200 implicit steps at CFL 50 on the bump channel: the residual falls
    by orders of magnitude, and the state is close to where 4000 explicit
    RK3 steps at CFL 0.9 (ucg_step) lead."""
    from ucns3d_b200.engine import Engine
    m, cfg, U = _bump()
    e = Engine(m, cfg)
    e.set_state(U)
    r0 = np.linalg.norm(e.call_flux_subroutines_3d())
    e.implicit_step(50.0, 200, 10)
    e.check_health()
    r1 = np.linalg.norm(e.call_flux_subroutines_3d())
    Ui = e.get_state()
    x = Engine(m, cfg)
    x.set_state(U)
    x.time_marching(4000, 0.9)
    x.check_health()
    rx = np.linalg.norm(x.call_flux_subroutines_3d())
    Ux = x.get_state()
    d = np.abs(Ui - Ux).max() / np.abs(Ux).max()
    print(f"implicit residual {r0:.3e} -> {r1:.3e}; explicit after 4000 steps {rx:.3e}; states differ {d:.3e}")
    assert r1 < 1e-3 * r0
    assert d < 1e-2


def _vortex():
    from ucns3d_b200 import cases as C
    c = C.vortex_hex_weno5(n=10)
    return c.mesh, c.cfg, c.U0


def test_oracle_dual_time_follows_the_explicit_solution():
    """DUAL_TIME with dt four times the explicit CFL step: the inner
    iterations converge (fewer than the limit) and after three physical
    steps the vortex is within 3 % of twelve explicit RK3 steps of dt/4."""
    m, cfg, U0 = _vortex()
    o = Oracle(m, cfg)
    dt = 4.0 * o.compute_dt(U0, 0.5)
    U, hist = U0.copy(), None
    for _ in range(3):
        U, hist, it = o.dual_time_step(U, hist, dt, 20.0, 20, 1e-3)
        assert it < 20
    Ue = U0.copy()
    for _ in range(12):
        Ue = o.rk3_step(Ue, dt / 4.0)
    assert np.abs(U - Ue).max() / np.abs(Ue).max() < 0.03


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["vortex_weno5", "muscl_ns_bump"])
def test_engine_dual_time_matches_oracle(name):
    """Three DUAL_TIME steps: the engine's state within 1e-10 of the
    oracle's and the same number of inner iterations in each step."""
    from ucns3d_b200.engine import Engine
    m, cfg, U0 = _vortex() if name == "vortex_weno5" else _bump(NAVIER_STOKES)
    o = Oracle(m, cfg)
    dt = 4.0 * o.compute_dt(U0, 0.5)
    e = Engine(m, cfg)
    e.set_state(U0)
    U, hist = U0.copy(), None
    for s in range(3):
        U, hist, it_o = o.dual_time_step(U, hist, dt, 20.0, 20, 1e-3)
        it_g = e.dual_time_step(dt, 20.0, 20, 1e-3)
        assert it_g == it_o, (s, it_g, it_o)
    e.check_health()
    Ug = e.get_state()
    err = np.abs(Ug - U).max() / np.abs(U).max()
    print(f"{name}: dual time state rel err {err:.3e}, inner iterations {it_o}")
    assert err < 1e-10


def test_oracle_explicit_dual_time_follows_the_explicit_solution():
    """DUAL_TIME_EX with dt twice the explicit CFL step: the explicit
    pseudo-time iterations converge (fewer than the limit), the state after
    three physical steps is within 2 % of six explicit RK3 steps of dt/2, and
    the returned state is the extrapolated first iterate 2 U^n - U^{n-1}."""
    m, cfg, U0 = _vortex()
    o = Oracle(m, cfg)
    dt = 2.0 * o.compute_dt(U0, 0.5)
    U, hist = U0.copy(), None
    for _ in range(3):
        U, hist, it = o.dual_time_step_explicit(U, hist, dt, 1.5, 200, 1e-3)
        assert it < 200
    assert np.array_equal(U, 2.0 * hist[0] - hist[1])
    Ue = U0.copy()
    for _ in range(6):
        Ue = o.rk3_step(Ue, dt / 2.0)
    assert np.abs(hist[0] - Ue).max() / np.abs(Ue).max() < 0.02


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["vortex_weno5", "muscl_ns_bump"])
def test_engine_explicit_dual_time_matches_oracle(name):
    """Three DUAL_TIME_EX steps: the engine's state (the extrapolated next
    iterate) within 1e-10 of the oracle's and the same number of inner
    iterations in each step."""
    from ucns3d_b200.engine import Engine
    m, cfg, U0 = _vortex() if name == "vortex_weno5" else _bump(NAVIER_STOKES)
    o = Oracle(m, cfg)
    dt = 2.0 * o.compute_dt(U0, 0.5)
    e = Engine(m, cfg)
    e.set_state(U0)
    U, hist = U0.copy(), None
    for s in range(3):
        U, hist, it_o = o.dual_time_step_explicit(U, hist, dt, 1.5, 200, 1e-3)
        it_g = e.dual_time_step_explicit(dt, 1.5, 200, 1e-3)
        assert it_g == it_o, (s, it_g, it_o)
    e.check_health()
    Ug = e.get_state()
    err = np.abs(Ug - U).max() / np.abs(U).max()
    print(f"{name}: explicit dual time state rel err {err:.3e}, inner iterations {it_o}")
    assert err < 1e-10
