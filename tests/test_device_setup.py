"""Reconstruction tables built on the device (ucg_build_recon) against the
host set-up library (ucp_prepare + ucg_upload_recon).

The device set-up evaluates the host's operations in the host's order
without fused multiply-adds (setup.cu is compiled with -fmad=false, the
host library with -ffp-contract=off), so the tables are the same doubles
and the residuals and RK3 steps of the two engines are equal bit for bit:
on shared matrix sets (the periodic hexahedra), one set per cell (jittered
tetrahedra), all four cell shapes (the mixed box), CWENO's lower-order
stencils, MUSCL with boundaries, both precision forms and a renumbered
engine."""
import numpy as np
import pytest

from ucns3d_b200 import _native as N
from ucns3d_b200.config import EULER, NAVIER_STOKES, make_config
from ucns3d_b200.mesh import IC_TGV, IC_UNIFORM, SCHEME_MUSCL, SCHEME_WENO, Mesh, RenumberedMesh

CASES = {
    "weno5_hex": (lambda: Mesh.box_hex(10, 10, 10), SCHEME_WENO, 4, 0, EULER),
    "weno3_tet": (lambda: Mesh.box_tet(6, 6, 6, seed=3), SCHEME_WENO, 2, 0, EULER),
    "weno5_tet": (lambda: Mesh.box_tet(5, 5, 5, seed=7), SCHEME_WENO, 4, 0, EULER),
    "cweno4_tet": (lambda: Mesh.box_tet(5, 5, 5, seed=5), SCHEME_WENO, 3, 5, EULER),
    "cweno4_ns_mixed": (lambda: Mesh.mixed_box(8, seed=4), SCHEME_WENO, 3, 5, NAVIER_STOKES),
    "muscl_bump": (lambda: Mesh.bump_channel(24, 10, 2, seed=2), SCHEME_MUSCL, 1, 0, EULER),
}


def _meshes(name):
    mk, scheme, iorder, ees, gov = CASES[name]
    return mk().prepare(scheme, iorder, ees), mk().prepare(scheme, iorder, ees, tables=False), gov


def _state(m, name):
    if name == "muscl_bump":
        U = m.initial_condition(IC_UNIFORM, [1.4, 1.0, 0.8, 0.0, 0.0, 1.0])
        c = m.centres()
        U[:, 0] *= 1.0 + 0.05 * np.sin(2 * np.pi * c[:, 0] / 3.0) * np.sin(np.pi * c[:, 1])
        return U
    return m.initial_condition(IC_TGV, [1.4, 5.0, 1.0])


@pytest.mark.parametrize("name", ["weno5_hex", "weno3_tet", "cweno4_ns_mixed"])
def test_geometry_only_preparation(name):
    """ucp_prepare_geometry: the same geometry, stencils and matrix-set
    numbering as ucp_prepare, no basis means or matrices; ucp_shapes gives
    the cells' volumes and frames of the geometry."""
    mh, md, _ = _meshes(name)
    gh, gd = mh.geometry(), md.geometry()
    assert gd["basis_mean"] is None
    for k, v in gh.items():
        if k != "basis_mean" and isinstance(v, np.ndarray):
            assert np.array_equal(v, gd[k]), k
    rh, rd = mh.recon(), md.recon()
    assert np.array_equal(rh["stencil"], rd["stencil"])
    assert np.array_equal(rh["table_id"], rd["table_id"]) and rh["ntables"] == rd["ntables"]
    assert rd["invmat"] is None
    sh = md.shapes()
    assert np.array_equal(sh["volume"], gh["volume"]) and np.array_equal(sh["frame"], gh["invccjac"])
    assert set(np.unique(sh["shape"])) <= {1, 2, 3, 4}
    if name == "cweno4_ns_mixed":
        assert set(np.unique(sh["shape"])) == {1, 2, 3, 4}


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [N.UCG_FP64, N.UCG_MIXED])
@pytest.mark.parametrize("name", list(CASES))
def test_device_tables_give_the_host_residual_bitwise(name, precision):
    from ucns3d_b200.engine import Engine
    mh, md, gov = _meshes(name)
    kw = dict(reynolds=1600.0, pres=71.43) if gov == NAVIER_STOKES else {}
    cfg = make_config(mh, governing=gov, precision=precision, **kw)
    U = _state(mh, name)
    eh, ed = Engine(mh, cfg), Engine(md, cfg, tables="device")
    out = []
    for e in (eh, ed):
        e.set_state(U)
        r = e.call_flux_subroutines_3d()
        e.runge_kutta3(1e-3)
        e.runge_kutta3(1e-3)
        e.check_health()
        out.append((r, e.get_state()))
    print(f"{name}: {mh.ncells} cells, {mh.ntables} matrix sets")
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["weno3_tet", "weno5_hex"])
def test_device_tables_on_a_renumbered_engine(name):
    """A mesh in shuffled order on an engine that renumbers its cells: the
    device set-up reads shapes and stencils in the caller's order and fills
    the tables of the device order."""
    from ucns3d_b200.engine import Engine
    mh, md, gov = _meshes(name)
    order = np.random.default_rng(11).permutation(mh.ncells)
    sh, sd = RenumberedMesh(mh, order), RenumberedMesh(md, order)
    cfg = make_config(mh, governing=gov, reorder=1)
    U = _state(mh, name)[order]
    res = []
    for m, tables in ((sh, "host"), (sd, "device")):
        e = Engine(m, cfg, tables=tables)
        assert e.cell_order()["renumbered"]
        e.set_state(U)
        res.append(e.call_flux_subroutines_3d())
    if name == "weno5_hex":  # shared sets: the first cell of each set differs between the numberings
        assert np.abs(res[0] - res[1]).max() <= 1e-12 * np.abs(res[0]).max()
    else:
        assert np.array_equal(res[0], res[1])
