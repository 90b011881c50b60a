"""Partitions (ucns3d_b200.partition) on the CPU: the plan's invariants, the
owned cells' residual of every rank equal to the whole mesh's (the oracle on
each rank's sliced mesh, bit for bit), and two gloo ranks stepping RK3 with
CFL time steps through the same transfer code as the engine path, equal to
the whole mesh's steps bit for bit.  The engine path with several ranks on
one device is in tests/test_partition_gpu.py."""
import os
import socket

import numpy as np
import pytest

from ucns3d_b200.config import EULER, NAVIER_STOKES, make_config
from ucns3d_b200.mesh import IC_TGV, IC_UNIFORM, SCHEME_MUSCL, SCHEME_WENO, Mesh
from ucns3d_b200.partition import HaloLists, PartitionMesh, PartitionPlan, rcb, transfer

CASES = {
    "muscl_ns_hex": (lambda: Mesh.box_hex(8, 8, 8), SCHEME_MUSCL, 1, 0, NAVIER_STOKES),
    # long in x with cubic cells (the stencil search goes by distance), so
    # that the bisections cut along x and the halos stop short of the far
    # side: cut faces and cut stencils in every part
    "weno3_tet": (lambda: Mesh.box_tet(16, 4, 4, L=(16.0, 4.0, 4.0), seed=3), SCHEME_WENO, 2, 0, EULER),
    "weno5_hex": (lambda: Mesh.box_hex(40, 6, 6, L=(40.0, 6.0, 6.0)), SCHEME_WENO, 4, 0, EULER),
    "cweno4_tet": (lambda: Mesh.box_tet(14, 4, 4, L=(14.0, 4.0, 4.0), seed=5), SCHEME_WENO, 3, 5, EULER),
    "cweno4_ns_mixed": (lambda: Mesh.mixed_box(6, seed=4), SCHEME_WENO, 3, 5, NAVIER_STOKES),
    "muscl_bump": (lambda: Mesh.bump_channel(24, 10, 2, seed=2), SCHEME_MUSCL, 1, 0, EULER),
    "muscl_ns_bump": (lambda: Mesh.bump_channel(24, 10, 2, seed=2), SCHEME_MUSCL, 1, 0, NAVIER_STOKES),
}


def _case(name):
    mk, scheme, iorder, ees, gov = CASES[name]
    m = mk().prepare(scheme, iorder, ees)
    bump = "bump" in name
    cfg = make_config(m, governing=gov, reynolds=200.0 if bump else 1600.0,
                      pres=1.0 if bump or gov == EULER else 71.43, bc_state=(1.0, 0.8, 0.0, 0.0, 1.0))
    if bump:
        U = m.initial_condition(IC_UNIFORM, [1.4, 1.0, 0.8, 0.0, 0.0, 1.0])
        c = m.centres()
        U[:, 0] *= 1.0 + 0.05 * np.sin(2 * np.pi * c[:, 0] / 3.0) * np.sin(np.pi * c[:, 1])
    else:
        U = m.initial_condition(IC_TGV, [1.4, 71.43 if gov == NAVIER_STOKES else 10.0, 1.0])
    return m, cfg, U


@pytest.mark.parametrize("n,k", [(1000, 2), (1000, 3), (1001, 4), (997, 7)])
def test_rcb_sizes_and_determinism(n, k):
    c = np.random.default_rng(5).uniform(size=(n, 3))
    p = rcb(c, k)
    sizes = np.bincount(p, minlength=k)
    assert sizes.max() - sizes.min() <= 1, sizes
    assert np.array_equal(p, rcb(c.copy(), k))


@pytest.mark.parametrize("name", ["weno5_hex", "muscl_bump"])
def test_plan_invariants(name):
    m, cfg, U = _case(name)
    plan = PartitionPlan(m, rcb(m.centres(), 3))
    owned = np.concatenate([plan.cells[k][plan.owned[k]] for k in range(3)])
    assert np.array_equal(np.sort(owned), np.arange(m.ncells))  # each cell owned once
    for k in range(3):
        assert np.all(np.diff(plan.cells[k]) > 0)  # increasing global index
        halo = np.flatnonzero(~plan.owned[k])
        got = np.concatenate([plan.recv[k][q] for q in sorted(plan.recv[k])])
        assert np.array_equal(np.sort(got), halo)  # every halo row has one source
        lists = HaloLists(plan, k)
        assert len(lists.recv) == len(halo)


@pytest.mark.parametrize("nparts", [2, 3, 4])
@pytest.mark.parametrize("name", list(CASES))
def test_owned_residual_equals_whole_mesh(name, nparts):
    from oracle import Oracle
    m, cfg, U = _case(name)
    R = Oracle(m, cfg).residual(U)
    plan = PartitionPlan(m, rcb(m.centres(), nparts))
    parts = []
    for k in range(nparts):
        pm = PartitionMesh(plan, k)
        Rk = Oracle(pm, cfg).residual(plan.local(k, U))
        parts.append(Rk[plan.owned[k]])
    assert np.array_equal(plan.assemble(parts), R)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, name, nsteps, out_dir):
    import torch
    import torch.distributed as dist
    from oracle import Oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m, cfg, U0 = _case(name)
        plan = PartitionPlan(m, rcb(m.centres(), world))
        lists = HaloLists(plan, rank)
        o = Oracle(PartitionMesh(plan, rank), cfg)
        U = plan.local(rank, U0)
        recvbuf = torch.empty((len(lists.recv), 5), dtype=torch.float64)
        dts = []
        for _ in range(nsteps):
            for s in (1, 2, 3):
                sendbuf = torch.from_numpy(np.ascontiguousarray(U[lists.send]))
                transfer(lists, sendbuf, recvbuf)
                U[lists.recv] = recvbuf.numpy()
                if s == 1:
                    t = torch.tensor([o.compute_dt(U, 0.5)], dtype=torch.float64)
                    dist.all_reduce(t, op=dist.ReduceOp.MIN)
                    dt = float(t.item())
                    dts.append(dt)
                    Un = U.copy()
                o.rk3_stage(Un, U, dt, s)
        np.save(os.path.join(out_dir, f"u{rank}.npy"), U[plan.owned[rank]])
        np.save(os.path.join(out_dir, f"dt{rank}.npy"), np.array(dts))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("name", ["weno5_hex", "muscl_ns_bump"])
def test_two_gloo_ranks_step_like_whole_mesh(name, tmp_path):
    import torch.multiprocessing as mp
    from oracle import Oracle
    nsteps, world = 3, 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, name, nsteps, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
        assert p.exitcode == 0
    m, cfg, U = _case(name)
    o = Oracle(m, cfg)
    dts = []
    for _ in range(nsteps):
        dt = o.compute_dt(U, 0.5)
        dts.append(dt)
        Un = U.copy()
        for s in (1, 2, 3):
            o.rk3_stage(Un, U, dt, s)
    plan = PartitionPlan(m, rcb(m.centres(), world))
    got = plan.assemble([np.load(tmp_path / f"u{r}.npy") for r in range(world)])
    assert np.array_equal(got, U)
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"dt{r}.npy"), np.array(dts))


def test_plan_refuses_an_empty_part():
    m, cfg, U = _case("muscl_bump")
    part = rcb(m.centres(), 2)
    part[part == 1] = 2  # parts 0 and 2: part 1 owns nothing
    with pytest.raises(ValueError):
        PartitionPlan(m, part)
