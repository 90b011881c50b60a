"""MOOD a posteriori limiting (RUNGE_KUTTA3_MOOD, src/time_p.f90:582-880;
src/mood.f90): the oracle's restatement on the CPU, the configuration
checks of ucg_create, and (marked gpu) the engine against the oracle.

Per RK stage: the candidate state from the reconstruction under the last
RECALC; PAD_NAD flags cells whose candidate is not admissible (density or
pressure not positive, or density / energy outside the stage-input bounds
of the cell and its face neighbours, widened in the relaxed mode); FIX_LIST
adds the face neighbours; the first cascade recomputes the selected reduced
cells with MUSCL, the second the flagged cells at first order; the
selected cells' stage is redone each time.  The engine agrees with the
oracle to 1e-10 of the state's magnitude after three steps and on MOOD_O
and RECALC exactly (cases whose flags are not decided by rounding: see
CASES)."""
import ctypes as C

import numpy as np
import pytest

from oracle import Oracle
from ucns3d_b200 import _native as N
from ucns3d_b200.config import EULER, NAVIER_STOKES, make_config
from ucns3d_b200.mesh import IC_VORTEX, SCHEME_MUSCL, SCHEME_WENO, Mesh


def _shock_tube(m):
    """A Sod-like jump across the middle of a periodic box (and the seam)."""
    x = m.centres()[:, 0]
    left = x < 0.5 * (x.min() + x.max())
    U = np.zeros((m.ncells, 5))
    U[:, 0] = np.where(left, 1.0, 0.125)
    U[:, 4] = np.where(left, 1.0, 0.1) / 0.4
    return U


def _blast(m):
    """A pressure pulse (10 against 0.1) in the middle of a periodic box at
    uniform density."""
    x = m.centres()[:, 0]
    mid = 0.5 * (x.min() + x.max())
    U = np.zeros((m.ncells, 5))
    U[:, 0] = 1.0
    U[:, 4] = np.where(np.abs(x - mid) < 0.125 * (x.max() - x.min()), 10.0, 0.1) / 0.4
    return U


def _smooth_wave(m):
    """Density waves advected along x at uniform speed and pressure: the
    original (unrelaxed) bounds clip the discrete extrema."""
    c = m.centres()
    rho = 1.0 + 0.2 * np.sin(2 * np.pi * c[:, 0] / 2.0) + 0.1 * np.sin(2 * np.pi * c[:, 1])
    U = np.zeros((m.ncells, 5))
    U[:, 0], U[:, 1], U[:, 4] = rho, rho, 1.0 / 0.4 + 0.5 * rho
    return U


# The original mode (MOOD_MODE 0) flags a candidate that exceeds its bounds
# by any amount, so on a plateau (the cells of a shock tube away from the
# jump) the decision rests on the last bit of the flux sum, which the
# engine (each face once) and the oracle (each cell's faces) round
# differently; the flagged cells there change nothing (first order equals
# the plateau) until a flag lands next to the jump.  Its cases are smooth
# waves, where the flags sit at real overshoots of the extrema.
CASES = {
    # name: (mesh, scheme order, ees, wenwrt, MOOD_MODE, initial state)
    "weno5_hex_relaxed": (lambda: Mesh.box_hex(24, 6, 6, L=(4.0, 1.0, 1.0)), 4, 0, 1, 1, _blast),
    "weno3_tet_relaxed": (lambda: Mesh.box_tet(12, 4, 4, L=(3.0, 1.0, 1.0), seed=3), 2, 0, 1, 1, _shock_tube),
    "cweno4_tet_relaxed": (lambda: Mesh.box_tet(12, 4, 4, L=(3.0, 1.0, 1.0), seed=5), 3, 5, 1, 1, _shock_tube),
    "weno3_tet_characteristic": (lambda: Mesh.box_tet(12, 4, 4, L=(3.0, 1.0, 1.0), seed=3), 2, 0, 2, 1,
                                 _shock_tube),
    "weno5_hex_original": (lambda: Mesh.box_hex(16, 6, 6, L=(2.0, 1.0, 1.0)), 4, 0, 1, 0, _smooth_wave),
    "weno3_tet_original": (lambda: Mesh.box_tet(8, 4, 4, L=(2.0, 1.0, 1.0), seed=3), 2, 0, 1, 0, _smooth_wave),
}


def _case(name, precision=N.UCG_FP64):
    mk, iorder, ees, wenwrt, mode, ic = CASES[name]
    m = mk().prepare(SCHEME_WENO, iorder, ees)
    cfg = make_config(m, governing=EULER, precision=precision, wenwrt=wenwrt, mood=1, mood_mode=mode)
    return m, cfg, ic(m)


def _oracle_run(m, cfg, U, dt, steps):
    o = Oracle(m, cfg)
    rc = np.zeros(m.ncells, np.int8)
    orders = []
    for _ in range(steps):
        U, order = o.rk3_step_mood(U, dt, rc)
        orders.append(order)
    return U, orders, rc


def test_oracle_mood_without_flags_is_the_plain_step():
    """Smooth vortex, relaxed bounds: no cell is flagged, every cell is FULL
    and passes CHECKSOL (16^3: on 10^3 some cells of the vortex core fail it,
    and those keep their WENO values under MOOD but take MUSCL without), so
    the MOOD step is the plain RK3 step bit for bit."""
    m = Mesh.box_hex(16, 16, 16, L=(10.0, 10.0, 10.0)).prepare(SCHEME_WENO, 4)
    from ucns3d_b200.cases import vortex_params
    U = m.initial_condition(IC_VORTEX, vortex_params(10.0))
    cfg = make_config(m, governing=EULER, mood=1, mood_mode=1, mood_var=(1e-2, 1e-2, 1e-2, 1e-2))
    o = Oracle(m, cfg)
    dt = o.compute_dt(U, 0.5)
    rc = np.zeros(m.ncells, np.int8)
    U1, order = o.rk3_step_mood(U, dt, rc)
    assert (order == 5).all() and not rc.any()
    assert np.array_equal(U1, o.rk3_step(U, dt))


@pytest.mark.parametrize("name", ["weno3_tet_relaxed", "weno5_hex_original"])
def test_oracle_mood_flags(name):
    """The jump (or the extrema of the waves) is flagged: MOOD_O takes 1
    there and the target order elsewhere, RECALC is the first-order set,
    the state stays physical."""
    m, cfg, U = _case(name)
    dt = Oracle(m, cfg).compute_dt(U, 0.5)
    U1, orders, rc = _oracle_run(m, cfg, U, dt, 2)
    assert set(np.unique(orders[-1])) <= {1, 2, cfg.iorder + 1}
    assert (orders[-1] == 1).any() and (orders[-1] == cfg.iorder + 1).any()
    assert np.array_equal(rc.astype(bool), orders[-1] == 1)
    p = 0.4 * (U1[:, 4] - 0.5 * (U1[:, 1:4] ** 2).sum(1) / U1[:, 0])
    assert np.isfinite(U1).all() and (U1[:, 0] > 0).all() and (p > 0).all()


def test_create_refuses_mood_outside_its_scope():
    """MOOD is WENO / CWENO with Euler (the reference's MOOD recomputes only
    the convective fluxes), MOOD_MODE 0 or 1, finite non-negative MOOD_VAR."""
    lib = N.engine()
    mw = Mesh.box_hex(4, 4, 4).prepare(SCHEME_WENO, 2)
    mm = Mesh.box_hex(4, 4, 4).prepare(SCHEME_MUSCL, 1)
    h = C.c_void_p()
    bad = [make_config(mw, governing=NAVIER_STOKES, reynolds=100.0, mood=1),
           make_config(mm, mood=1),
           make_config(mw, mood=2),
           make_config(mw, mood=1, mood_mode=2),
           make_config(mw, mood=1, mood_var=(-1e-4, 1e-3, 1e-4, 1e-3)),
           make_config(mw, mood=1, mood_var=(1e-4, float("nan"), 1e-4, 1e-3))]
    for cfg in bad:
        assert lib.ucg_create(C.byref(cfg), mw.ncells, 0, C.byref(h)) == N.UCG_EINVAL
        assert not h.value


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_engine_mood_matches_oracle(name):
    from ucns3d_b200.engine import Engine
    m, cfg, U = _case(name)
    o = Oracle(m, cfg)
    dt = o.compute_dt(U, 0.5)
    Uo, orders, rc = _oracle_run(m, cfg, U, dt, 3)
    e = Engine(m, cfg)
    e.set_state(U)
    for _ in range(3):
        e.runge_kutta3(dt)
    e.check_health()
    Ug = e.get_state()
    st = e.mood_state()
    err = np.abs(Ug - Uo).max() / np.abs(Uo).max()
    flagged = int((orders[-1] < cfg.iorder + 1).sum())
    print(f"{name}: state rel err {err:.3e}, cells below the target order {flagged} of {m.ncells}")
    assert flagged > 0
    assert np.array_equal(st["order"], orders[-1])
    assert np.array_equal(st["recalc"].astype(np.int8), rc)
    assert err < 1e-10


@pytest.mark.gpu
def test_engine_mood_without_flags_is_the_plain_step():
    """No flags and no reduced cells (smooth vortex at 16^3, wide bounds):
    the MOOD stages give the plain RK3 result bit for bit."""
    from ucns3d_b200.cases import vortex_params
    from ucns3d_b200.engine import Engine
    m = Mesh.box_hex(16, 16, 16, L=(10.0, 10.0, 10.0)).prepare(SCHEME_WENO, 4)
    U = m.initial_condition(IC_VORTEX, vortex_params(10.0))
    out = []
    for mood in (1, 0):
        cfg = make_config(m, governing=EULER, mood=mood, mood_var=(1e-2, 1e-2, 1e-2, 1e-2))
        e = Engine(m, cfg)
        e.set_state(U)
        e.runge_kutta3(0.05)
        e.check_health()
        out.append(e.get_state())
        if mood:
            assert (e.mood_state()["order"] == 5).all()
    assert np.array_equal(out[0], out[1])


@pytest.mark.gpu
def test_engine_mood_mixed_precision_runs_physical():
    """The mixed form under MOOD: the flags may differ from the FP64 form's
    near the thresholds, so only closeness in L2 (1e-3 relative) and a
    physical state are required."""
    from ucns3d_b200.engine import Engine
    m, cfg64, U = _case("weno3_tet_relaxed")
    cfg32 = N.UcgConfig.from_buffer_copy(cfg64)
    cfg32.precision = N.UCG_MIXED
    dt = Oracle(m, cfg64).compute_dt(U, 0.5)
    res = []
    for cfg in (cfg64, cfg32):
        e = Engine(m, cfg)
        e.set_state(U)
        for _ in range(3):
            e.runge_kutta3(dt)
        e.check_health()
        res.append(e.get_state())
    l2 = np.sqrt(np.mean((res[0] - res[1]) ** 2)) / np.sqrt(np.mean(res[0] ** 2))
    print(f"MOOD mixed vs FP64 relative L2 {l2:.3e}")
    assert l2 < 1e-3
