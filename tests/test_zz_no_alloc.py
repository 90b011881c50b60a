"""The allocation-free entry point ucg_residual_muscl_static, through the C
ABI, against the engine's ucg_residual and the oracle on the same inputs.

Callers of ucg_residual_muscl_static cannot allocate device memory; the test
itself is not such a caller, so it uses torch to place the inputs and
outputs on the device.  The entry point's only scratch is a fixed device
array in the library; this file runs last so that a failure here leaves the
rest of the suite's results intact, and it passes both alone in a fresh
process and after the other tests.  Tolerance: 1e-12 of the per-cell flux
scale, as the engine-vs-oracle residual tests."""
import ctypes as C

import numpy as np
import pytest

from ucns3d_b200 import _native as N
from ucns3d_b200 import cases
from ucns3d_b200.engine import Engine

pytestmark = pytest.mark.gpu

F, Q = N.UCG_MAX_FACES, N.UCG_MAX_QP


def _flux_scale(mesh, U):
    """Magnitude of the face fluxes of each cell (uniform-state estimate): the
    residual is a sum of such fluxes that largely cancel."""
    g = mesh.geometry()
    r, u = U[:, 0], U[:, 1:4] / U[:, :1]
    p = 0.4 * (U[:, 4] - 0.5 * r * (u * u).sum(1))
    area = (g["face_area"] * (np.arange(F)[None, :] < g["nfaces"][:, None])).sum(1)
    s = np.abs(U).max(1) * (np.abs(u).max(1) + np.sqrt(1.4 * p / r)) + p
    return (s * area)[:, None]


def _device_structs(mesh, dev):
    """Device copies of the ABI-layout geometry and tables (torch owns them)."""
    import torch
    g, r = mesh.geometry(), mesh.recon()
    keep = {}

    def put(name, a, ctype):
        t = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        keep[name] = t
        return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ctype))

    gd = N.UcgGeometry()
    gd.ncells = g["ncells"]
    for name in ("nfaces", "face_type", "neigh", "neigh_face", "bc", "qperm", "admis", "full"):
        setattr(gd, name, put(name, g[name].astype(np.int32), C.c_int32))
    for name in ("face_angle", "face_area", "dih", "qpoints", "volume", "minedge", "invccjac", "basis_mean"):
        setattr(gd, name, put(name, g[name].astype(np.float64), C.c_double))
    rd = N.UcgRecon()
    rd.first, rd.count = 0, g["ncells"]
    rd.stencil = put("stencil", r["stencil"].astype(np.int32), C.c_int32)
    rd.ntables = r["ntables"]
    rd.table_id = put("table_id", r["table_id"].astype(np.int32), C.c_int32)
    rd.invmat = put("invmat", r["invmat"].astype(np.float64), C.c_double)
    return gd, rd, keep


def _static_fn():
    lib = N.engine()
    fn = lib.ucg_residual_muscl_static
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(N.UcgConfig), C.POINTER(N.UcgGeometry), C.POINTER(N.UcgRecon),
                   C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


def _state(which, c):
    U = c.U0.copy()
    cc = c.mesh.centres()
    if which == "bump_euler":
        U[:, 0] *= 1.0 + 0.05 * np.sin(2 * np.pi * cc[:, 0] / 3.0) * np.sin(np.pi * cc[:, 1])
    elif which == "bump_shock_tube":
        # a density and pressure jump of 8x and 10x across x = 1.5: the limited
        # face values next to it move the cell's density by more than 95 %,
        # so CHECKSOLX sends those cells back to first order
        hi = cc[:, 0] < 1.5
        prim = np.where(hi[:, None], [1.0, 0.3, 0.0, 0.0, 1.0], [0.125, 0.3, 0.0, 0.0, 0.1])
        U = np.stack([prim[:, 0], prim[:, 0] * prim[:, 1], prim[:, 0] * prim[:, 2], prim[:, 0] * prim[:, 3],
                      prim[:, 4] / 0.4 + 0.5 * prim[:, 0] * (prim[:, 1:4] ** 2).sum(1)], axis=1)
    return U


@pytest.mark.parametrize("which", ["tgv_ns", "bump_euler", "bump_shock_tube"])
def test_static_scratch_residual_matches_engine_and_oracle(which):
    """Two calls in a row through the C ABI, each against the engine's
    ucg_residual and the oracle's residual on the same inputs."""
    import torch
    from oracle import Oracle
    fn = _static_fn()
    c = cases.tgv_hex_muscl(n=16) if which == "tgv_ns" else cases.bump_muscl(nx=60, ny=20, nlayers=2)
    U = _state(which, c)
    e = Engine(c.mesh, c.cfg)
    e.set_state(U)
    ref = e.call_flux_subroutines_3d()
    e.close()
    orc = Oracle(c.mesh, c.cfg).residual(U)
    dev = torch.device("cuda:0")
    gd, rd, keep = _device_structs(c.mesh, dev)
    scale = _flux_scale(c.mesh, U)
    for call in range(2):  # two calls in a row share the static scratch
        u = torch.from_numpy(U).to(dev)
        rhs = torch.full_like(u, float("nan"))
        rc = fn(C.byref(c.cfg), C.byref(gd), C.byref(rd), C.c_void_p(u.data_ptr()), C.c_void_p(rhs.data_ptr()), None)
        assert rc == N.UCG_OK
        torch.cuda.synchronize()
        got = rhs.cpu().numpy()
        err = (np.abs(got - ref) / scale).max()
        err_o = (np.abs(got - orc) / scale).max()
        assert err < 1e-12, (call, err)
        assert err_o < 1e-12, (call, err_o)


def test_static_scratch_unsupported_faces_give_nan():
    """Faces the allocation-free path does not treat come back as NaN rows,
    not as a plausible residual: every boundary cell of a Navier-Stokes
    channel (the viscous wall treatment is not in this path), and a cell
    whose boundary code is not one of 1, 2, 3, 4, 6.  Other rows stay
    finite and equal to the engine's."""
    import torch
    from ucns3d_b200.config import NAVIER_STOKES, make_config
    fn = _static_fn()
    c = cases.bump_muscl(nx=30, ny=10, nlayers=2)
    dev = torch.device("cuda:0")
    g = c.mesh.geometry()
    nf = g["nfaces"]
    phys = ((g["neigh"] < 0) & (np.arange(F)[None, :] < nf[:, None])).any(1)
    # Navier-Stokes with walls, inflow and outflow
    cfg_ns = make_config(c.mesh, governing=NAVIER_STOKES, reynolds=1000.0, pres=1.0, prandtl=0.72,
                         bc_state=tuple(c.cfg.bc_state))
    gd, rd, keep = _device_structs(c.mesh, dev)
    u = torch.from_numpy(c.U0).to(dev)
    rhs = torch.zeros_like(u)
    assert fn(C.byref(cfg_ns), C.byref(gd), C.byref(rd), C.c_void_p(u.data_ptr()), C.c_void_p(rhs.data_ptr()),
              None) == N.UCG_OK
    torch.cuda.synchronize()
    got = rhs.cpu().numpy()
    assert np.array_equal(np.isnan(got).any(1), phys)
    assert np.isfinite(got[~phys]).all()
    # Euler, one boundary face given code 5 (not a BOUNDARYS case here)
    cell, face = [(i, f) for i in range(len(nf)) for f in range(nf[i]) if g["neigh"][i, f] < 0][3]
    keep["bc"].view(-1)[cell * F + face] = 5
    rhs = torch.zeros_like(u)
    assert fn(C.byref(c.cfg), C.byref(gd), C.byref(rd), C.c_void_p(u.data_ptr()), C.c_void_p(rhs.data_ptr()),
              None) == N.UCG_OK
    torch.cuda.synchronize()
    got = rhs.cpu().numpy()
    bad_rows = np.nonzero(np.isnan(got).any(1))[0].tolist()
    assert bad_rows == [cell]
    e = Engine(c.mesh, c.cfg)
    e.set_state(c.U0)
    ref = e.call_flux_subroutines_3d()
    e.close()
    ok = np.ones(len(nf), bool)
    ok[cell] = False
    assert (np.abs(got[ok] - ref[ok]) / _flux_scale(c.mesh, c.U0)[ok]).max() < 1e-12


def test_static_scratch_rejects_oversize_and_wrong_scheme():
    lib = N.engine()
    fn = lib.ucg_residual_muscl_static
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(N.UcgConfig), C.POINTER(N.UcgGeometry), C.POINTER(N.UcgRecon),
                   C.c_void_p, C.c_void_p, C.c_void_p]
    c = cases.tgv_hex_muscl(n=8)
    g, r = N.UcgGeometry(), N.UcgRecon()
    g.ncells = 10_000_000  # beyond the fixed scratch (checked before any device access)
    r.first, r.count = 0, g.ncells
    r.stencil = C.cast(C.c_void_p(16), C.POINTER(C.c_int32))
    r.invmat = C.cast(C.c_void_p(16), C.POINTER(C.c_double))
    assert fn(C.byref(c.cfg), C.byref(g), C.byref(r), C.c_void_p(16), C.c_void_p(16), None) == N.UCG_EINVAL
    bad = N.UcgConfig.from_buffer_copy(c.cfg)
    bad.scheme = 3
    g.ncells = 8
    r.count = 8
    assert fn(C.byref(bad), C.byref(g), C.byref(r), C.c_void_p(16), C.c_void_p(16), None) == N.UCG_EINVAL


def test_static_scratch_index_out_of_range_gives_nan():
    """An out-of-range stencil index in caller memory is caught by the
    kernel's own bounds check: that cell's residual row is NaN, the call
    returns UCG_OK and nothing outside the arrays is read."""
    import torch
    lib = N.engine()
    fn = lib.ucg_residual_muscl_static
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(N.UcgConfig), C.POINTER(N.UcgGeometry), C.POINTER(N.UcgRecon),
                   C.c_void_p, C.c_void_p, C.c_void_p]
    c = cases.bump_muscl(nx=60, ny=20, nlayers=2)
    dev = torch.device("cuda:0")
    gd, rd, keep = _device_structs(c.mesh, dev)
    n = c.mesh.ncells
    bad_cell = 5
    W = c.cfg.imax + 1
    keep["stencil"].view(-1)[bad_cell * W + 1] = n + 7
    u = torch.from_numpy(c.U0).to(dev)
    rhs = torch.zeros_like(u)
    assert fn(C.byref(c.cfg), C.byref(gd), C.byref(rd), C.c_void_p(u.data_ptr()), C.c_void_p(rhs.data_ptr()),
              None) == N.UCG_OK
    torch.cuda.synchronize()
    got = rhs.cpu().numpy()
    assert np.isnan(got[bad_cell]).all()
    # only the bad cell and the face neighbours that read its face values
    nb = c.mesh.geometry()["neigh"][bad_cell]
    touched = set([bad_cell] + [int(x) for x in nb if x >= 0])
    rows = np.isnan(got).any(1)
    assert set(np.nonzero(rows)[0].tolist()) <= touched
