"""Cell renumbering inside the engine (ucg_config.reorder = 1, reverse
Cuthill-McKee on the face graph), through the C ABI on a B200.

* On the same caller numbering, reorder 1 gives the residual and the state
  after RK3 steps bit for bit equal to reorder 0: stencil and face orders
  are kept and every face flux is still evaluated on the side of the lower
  caller index.
* A mesh handed over in a shuffled numbering (as cells arrive from a
  partitioner or a grid file) gives, permuted back, the residual of the
  original numbering within 1e-13 of the per-cell flux scale (the owner side
  of some faces changes with the numbering, which changes the last bits of
  those face fluxes), and the oracle's residual on the shuffled mesh within
  1e-12.
The host-side renumbering itself (tests/test_prep.py) is checked without a
GPU."""
import numpy as np
import pytest

from oracle import Oracle
from ucns3d_b200 import _native as N
from ucns3d_b200.config import EULER, NAVIER_STOKES, make_config
from ucns3d_b200.engine import Engine
from ucns3d_b200.mesh import IC_TGV, SCHEME_MUSCL, SCHEME_WENO, Mesh, RenumberedMesh

pytestmark = pytest.mark.gpu

MESHES = {
    "muscl_ns_hex": (lambda: Mesh.box_hex(8, 8, 8), SCHEME_MUSCL, 1, 0, NAVIER_STOKES),
    "weno3_tet": (lambda: Mesh.box_tet(5, 5, 5, seed=3), SCHEME_WENO, 2, 0, EULER),
    "weno5_hex": (lambda: Mesh.box_hex(10, 10, 10), SCHEME_WENO, 4, 0, EULER),
    "cweno4_ns_mixed": (lambda: Mesh.mixed_box(8, seed=4), SCHEME_WENO, 3, 5, NAVIER_STOKES),
    "muscl_bump": (lambda: Mesh.bump_channel(24, 10, 2, seed=2), SCHEME_MUSCL, 1, 0, EULER),
}


def _setup(name, reorder, precision=N.UCG_FP64, wenwrt=1):
    mk, scheme, iorder, ees, gov = MESHES[name]
    m = mk().prepare(scheme, iorder, ees)
    bc = (1.0, 0.675 * np.sqrt(1.4), 0.0, 0.0, 1.0)
    p0 = 71.43 if gov == NAVIER_STOKES else 1.0
    cfg = make_config(m, governing=gov, precision=precision, reynolds=1600.0, pres=p0, prandtl=0.71, bc_state=bc,
                      wenwrt=wenwrt, reorder=reorder)
    if name == "muscl_bump":
        U = m.initial_condition(1, [1.4, *bc])
        c = m.centres()
        U[:, 0] *= 1.0 + 0.05 * np.sin(2 * np.pi * c[:, 0] / 3.0) * np.sin(np.pi * c[:, 1])
    else:
        U = m.initial_condition(IC_TGV, [1.4, 71.43 if gov == NAVIER_STOKES else 5.0, 1.0])
    return m, cfg, U


def _flux_scale(m, U):
    g = m.geometry()
    r, u = U[:, 0], U[:, 1:4] / U[:, :1]
    p = 0.4 * (U[:, 4] - 0.5 * r * (u * u).sum(1))
    area = (g["face_area"] * (np.arange(6)[None, :] < g["nfaces"][:, None])).sum(1)
    return ((np.abs(U).max(1) * (np.abs(u).max(1) + np.sqrt(1.4 * p / r)) + p) * area)[:, None]


def _run(m, cfg, U, steps):
    e = Engine(m, cfg)
    e.set_state(U)
    R = e.residual()
    for _ in range(steps):
        e.runge_kutta3(2e-3)
    e.check_health()
    out = R, e.get_state()
    e.close()
    return out


def _shuffled(name, reorder, **kw):
    m, cfg, U = _setup(name, reorder, **kw)
    order = np.random.default_rng(11).permutation(m.ncells)
    return m, RenumberedMesh(m, order), cfg, U, order


def _order(m, cfg):
    e = Engine(m, cfg)
    out = e.cell_order()
    e.close()
    return out


@pytest.mark.parametrize("name", list(MESHES))
def test_reorder_is_bitwise_transparent(name):
    """On a shuffled numbering the engine renumbers (reverse Cuthill-McKee
    gathers from fewer cache lines); results equal reorder 0 bit for bit."""
    m, ms, cfg0, U, order = _shuffled(name, 0)
    cfg1 = N.UcgConfig.from_buffer_copy(cfg0)
    cfg1.reorder = 1
    o = _order(ms, cfg1)
    print(f"{name}: gather cost shuffled {o['cost_caller']:.2f}, reverse Cuthill-McKee {o['cost_rcm']:.2f}")
    assert o["renumbered"]
    assert sorted(o["n2o"].tolist()) == list(range(m.ncells))
    R0, S0 = _run(ms, cfg0, U[order], 3)
    R1, S1 = _run(ms, cfg1, U[order], 3)
    assert np.array_equal(R0, R1)
    assert np.array_equal(S0, S1)


def test_structured_order_is_kept():
    """A box numbered row by row already gathers from fewer lines than
    reverse Cuthill-McKee would: the engine keeps it."""
    m, cfg, U = _setup("weno5_hex", 1)
    o = _order(m, cfg)
    assert not o["renumbered"] and o["cost_caller"] < o["cost_rcm"]
    assert np.array_equal(o["n2o"], np.arange(m.ncells))


@pytest.mark.parametrize("precision", [N.UCG_FP64, N.UCG_MIXED])
def test_reorder_characteristic_weno_bitwise(precision):
    m, ms, cfg0, U, order = _shuffled("weno3_tet", 0, precision=precision, wenwrt=2)
    cfg1 = N.UcgConfig.from_buffer_copy(cfg0)
    cfg1.reorder = 1
    assert np.array_equal(_run(ms, cfg0, U[order], 1)[1], _run(ms, cfg1, U[order], 1)[1])


@pytest.mark.parametrize("name", ["weno3_tet", "cweno4_ns_mixed", "muscl_bump"])
def test_shuffled_numbering_gives_the_same_residual(name):
    m, cfg, U = _setup(name, 1)
    order = np.random.default_rng(11).permutation(m.ncells)
    ms = RenumberedMesh(m, order)
    Rb, _ = _run(m, cfg, U, 0)
    Rs, _ = _run(ms, cfg, U[order], 0)
    scale = _flux_scale(m, U)
    err = (np.abs(ms.to_base(Rs) - Rb) / scale).max()
    err_o = (np.abs(Rs - Oracle(ms, cfg).residual(U[order])) / scale[order]).max()
    print(f"{name}: shuffled vs original residual {err:.3e}, vs oracle on the shuffled mesh {err_o:.3e}")
    assert err < 1e-13
    assert err_o < 1e-12
    # the renumbering inside the engine is transparent on the shuffled mesh too
    cfg0 = N.UcgConfig.from_buffer_copy(cfg)
    cfg0.reorder = 0
    assert np.array_equal(_run(ms, cfg0, U[order], 0)[0], Rs)


def test_reorder_adjoint_matches_caller_order():
    """VJP and JVP of the MUSCL bump channel (shuffled numbering) with the
    engine renumbered internally, against the same with the caller's order
    kept (1e-13: the reverse map sums a cell's contributions in device
    order)."""
    _, m, cfg1, U, order = _shuffled("muscl_bump", 1)
    U = U[order]
    cfg0 = N.UcgConfig.from_buffer_copy(cfg1)
    cfg0.reorder = 0
    assert _order(m, cfg1)["renumbered"]
    rng = np.random.default_rng(3)
    lam, du = rng.standard_normal(U.shape), 1e-2 * rng.standard_normal(U.shape)
    out = []
    for cfg in (cfg0, cfg1):
        e = Engine(m, cfg)
        e.set_state(U)
        mu, pbar = e.residual_vjp(lam)
        out.append((mu, pbar, e.residual_jvp(du), e.force_vjp()))
        e.close()
    for a, b in zip(out[0], out[1]):
        assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
