"""Partitions on the GPU through the C ABI: ucg_rk3_stage, ucg_halo_set,
ucg_halo_pack and ucg_halo_unpack.  Several ranks' engines run in this
process on one device (LocalCluster: every transfer is a device copy ordered
by the host between the packs and the unpacks, so no kernel waits for
another); their owned cells must step exactly like one engine on the whole
mesh, and their CFL time step must be the whole mesh's."""
import numpy as np
import pytest

from ucns3d_b200 import _native as N
from ucns3d_b200.engine import Engine, EngineError
from ucns3d_b200.partition import LocalCluster, PartitionPlan, rcb

pytestmark = pytest.mark.gpu


def _case(name, precision=N.UCG_FP64):
    from test_partition import _case as case
    m, cfg, U = case(name)
    cfg.precision = precision
    return m, cfg, U


def test_three_stages_are_one_step():
    m, cfg, U = _case("weno5_hex")
    a, b = Engine(m, cfg), Engine(m, cfg)
    try:
        a.set_state(U)
        b.set_state(U)
        dt = a.calculate_cfl(0.5)
        a.runge_kutta3(dt)
        for s in (1, 2, 3):
            b.rk3_stage(s, dt)
        assert np.array_equal(a.get_state(), b.get_state())
    finally:
        a.close()
        b.close()


def test_halo_pack_and_unpack_rows():
    import torch
    m, cfg, U = _case("muscl_bump")
    e = Engine(m, cfg)
    try:
        e.set_state(U)
        send = np.array([5, 0, 17, 5, 3], dtype=np.int32)  # a row may go to several peers
        recv = np.array([9, 2, 40], dtype=np.int32)
        e.halo_set(send, recv)
        buf = torch.empty((len(send), 5), dtype=torch.float64, device="cuda")
        e.halo_pack(1, buf.data_ptr())
        e.synchronize()
        assert np.array_equal(buf.cpu().numpy(), U[send])
        rows = torch.arange(15, dtype=torch.float64, device="cuda").reshape(3, 5) + 100.0
        e.halo_unpack(1, rows.data_ptr())
        e.synchronize()
        V = U.copy()
        V[recv] = rows.cpu().numpy()
        assert np.array_equal(e.get_state(), V)
    finally:
        e.close()


def test_halo_and_stage_arguments_are_checked():
    m, cfg, U = _case("muscl_bump")
    e = Engine(m, cfg, upload=False)  # the lists map through the cell order fixed at the geometry upload
    try:
        with pytest.raises(EngineError) as ei:
            e.halo_set(np.array([0]), np.array([1]))
        assert ei.value.code == N.UCG_ESTATE
    finally:
        e.close()
    e = Engine(m, cfg)
    try:
        e.set_state(U)
        for send, recv in (([0, m.ncells], [1]), ([0], [-1]), ([0], [3, 4, 3])):
            with pytest.raises(EngineError) as ei:
                e.halo_set(np.array(send), np.array(recv))
            assert ei.value.code == N.UCG_EINVAL
        for stage in (0, 4):
            with pytest.raises(EngineError):
                e.rk3_stage(stage, 1e-3)
    finally:
        e.close()


def test_stage_refuses_mood():
    from ucns3d_b200.config import EULER, make_config
    from ucns3d_b200.mesh import IC_TGV, SCHEME_WENO, Mesh
    m = Mesh.box_hex(8, 8, 8).prepare(SCHEME_WENO, 4, 0)
    cfg = make_config(m, governing=EULER, mood=1)
    e = Engine(m, cfg)
    try:
        e.set_state(m.initial_condition(IC_TGV, [1.4, 10.0, 1.0]))
        with pytest.raises(EngineError) as ei:
            e.rk3_stage(1, 1e-3)
        assert ei.value.code == N.UCG_EINVAL
    finally:
        e.close()


def test_cell_roles_are_checked():
    from test_partition import _case as case
    m, cfg, U = case("muscl_bump")
    plan = PartitionPlan(m, rcb(m.centres(), 2))
    from ucns3d_b200.partition import PartitionMesh
    pm = PartitionMesh(plan, 0)
    roles = plan.roles(0)
    for bad in (np.where(roles == 0, 3, roles), np.full_like(roles, 2)):
        with pytest.raises(EngineError) as ei:
            Engine(pm, cfg, roles=bad)
        assert ei.value.code == N.UCG_EINVAL
    e = Engine(pm, cfg)  # geometry uploaded: too late for roles
    try:
        r = np.ascontiguousarray(roles)
        import ctypes as C
        assert e.lib.ucg_set_cell_roles(e._h, r.ctypes.data_as(C.POINTER(C.c_int8))) == N.UCG_ESTATE
    finally:
        e.close()
    e = Engine(pm, cfg, roles=roles)  # the adjoint covers whole meshes
    try:
        e.set_state(plan.local(0, U))
        with pytest.raises(EngineError) as ei:
            e.force()
        assert ei.value.code == N.UCG_EINVAL
    finally:
        e.close()


@pytest.mark.parametrize("restrict", [True, False])
@pytest.mark.parametrize("name", ["weno5_hex", "cweno4_ns_mixed", "muscl_ns_bump"])
def test_owned_residual_rows_equal_whole_mesh(name, restrict):
    m, cfg, U = _case(name)
    plan = PartitionPlan(m, rcb(m.centres(), 3))
    whole = Engine(m, cfg)
    cluster = LocalCluster(plan, cfg, restrict=restrict)
    try:
        whole.set_state(U)
        R = whole.residual()
        cluster.set_state(U)
        cluster.exchange(1)
        got = plan.assemble([h.engine.residual()[plan.owned[h.rank]] for h in cluster.ranks])
        assert np.array_equal(got, R)
    finally:
        cluster.close()
        whole.close()


@pytest.mark.parametrize("restrict", [True, False])
@pytest.mark.parametrize("precision", [N.UCG_FP64, N.UCG_MIXED])
@pytest.mark.parametrize("nparts", [2, 3])
@pytest.mark.parametrize("name", ["weno5_hex", "weno3_tet", "cweno4_tet", "cweno4_ns_mixed", "muscl_ns_bump"])
def test_partitioned_steps_equal_whole_mesh(name, nparts, precision, restrict):
    m, cfg, U = _case(name, precision)
    plan = PartitionPlan(m, rcb(m.centres(), nparts))
    whole = Engine(m, cfg)
    cluster = LocalCluster(plan, cfg, restrict=restrict)
    try:
        whole.set_state(U)
        cluster.set_state(U)
        for _ in range(3):
            dt = whole.calculate_cfl(0.5)
            assert cluster.compute_dt(0.5) == dt
            whole.runge_kutta3(dt)
            cluster.rk3_step(dt)
        assert np.array_equal(cluster.get_state(), whole.get_state())
    finally:
        cluster.close()
        whole.close()
