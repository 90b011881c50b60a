"""COMPUTEFORCE in full on the GPU (ucg_wall_loads): forces with the viscous
shear and the pressure moments about the cell centres, against the oracle's
restatement (orc_wall_loads), for MUSCL and CWENO, Euler and Navier-Stokes
(no-slip walls), both precision forms, with the engine's cell renumbering,
and summed over partition ranks."""
import numpy as np
import pytest

from ucns3d_b200 import _native as N
from ucns3d_b200.engine import Engine, lift_drag

pytestmark = pytest.mark.gpu


def _bump(scheme_order, ns):
    from ucns3d_b200.config import NAVIER_STOKES, make_config
    from ucns3d_b200.mesh import SCHEME_MUSCL, SCHEME_WENO, Mesh
    scheme, order, ees = scheme_order
    m = Mesh.bump_channel(24, 8, 4, seed=2).prepare(SCHEME_WENO if scheme == "weno" else SCHEME_MUSCL, order, ees)
    gov = dict(governing=NAVIER_STOKES, reynolds=50.0) if ns else dict(governing=2)
    cfg = make_config(m, bc_state=(1.0, 0.8, 0.0, 0.0, 1.0), pres=0.9, **gov)
    c = m.centres()
    U = np.tile([1.0, 0.8, 0.0, 0.0, 1.0 / 0.4 + 0.32], (m.ncells, 1))
    U = U * (1.0 + 0.05 * np.sin(3.0 * c[:, :1] + 2.0 * c[:, 1:2] + 1.7 * c[:, 2:3] + np.arange(5)[None, :]))
    return m, cfg, U


CASES = {"muscl_euler": (("muscl", 1, 0), False), "muscl_ns": (("muscl", 1, 0), True),
         "weno3_ns": (("weno", 2, 0), True), "cweno4_ns": (("weno", 3, 5), True)}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision", [N.UCG_FP64, N.UCG_MIXED])
def test_wall_loads_match_oracle(name, precision):
    from oracle import Oracle
    m, cfg, U = _bump(*CASES[name])
    cfg.precision = precision
    c = m.centres()
    ref = Oracle(m, cfg).wall_loads(U, c)
    e = Engine(m, cfg)
    try:
        e.set_state(U)
        got = e.wall_loads(c)
        assert np.array_equal(e.wall_loads()[3:], np.zeros(3))
        # FP64: the sums' order differs (two-pass device sums against the
        # oracle's running sum); mixed: FP32 face-value differences
        tol = 1e-12 if precision == N.UCG_FP64 else 1e-5
        scale = np.abs(ref).max()
        print(f"{name} {precision}: {got} vs {ref}, max rel {np.abs(got - ref).max() / scale:.2e}")
        assert np.abs(got - ref).max() <= tol * scale, (got, ref)
        if precision == N.UCG_FP64 and not CASES[name][1]:
            assert abs(got[0] - e.force()) <= 1e-12 * abs(got[0])
        cl, cd = lift_drag(got, 2.0, 1.0, 0.8)
        assert np.isfinite(cl) and np.isfinite(cd)
    finally:
        e.close()


def test_wall_loads_with_renumbered_cells():
    """reorder 1: the centres go into the engine's order with the state."""
    from ucns3d_b200.config import make_config
    m, cfg, U = _bump(("muscl", 1, 0), True)
    c = m.centres()
    a = Engine(m, cfg)
    cfg2 = make_config(m, governing=cfg.governing, reynolds=50.0, bc_state=(1.0, 0.8, 0.0, 0.0, 1.0), pres=0.9,
                       reorder=1)
    b = Engine(m, cfg2)
    try:
        a.set_state(U)
        b.set_state(U)
        la, lb = a.wall_loads(c), b.wall_loads(c)
        assert np.abs(la - lb).max() <= 1e-13 * np.abs(la).max(), (la, lb)
    finally:
        a.close()
        b.close()


def test_wall_loads_sum_over_partition_ranks():
    from test_partition import _case
    from ucns3d_b200.partition import LocalCluster, PartitionPlan, rcb
    m, cfg, U = _case("muscl_ns_bump")
    plan = PartitionPlan(m, rcb(m.centres(), 3))
    whole = Engine(m, cfg)
    cluster = LocalCluster(plan, cfg, restrict=True)
    try:
        whole.set_state(U)
        cluster.set_state(U)
        c = m.centres()
        w = whole.wall_loads(c)
        s = cluster.wall_loads(c)
        assert np.abs(s - w).max() <= 1e-12 * np.abs(w).max(), (s, w)
    finally:
        cluster.close()
        whole.close()
