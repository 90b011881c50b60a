"""CUDA engine against the oracle, through the C ABI, on a B200.

Tolerances (FP64 engine): the residual agrees with the oracle to 1e-12
relative to the largest flux magnitude of the cell's faces (per variable,
max over cells); after several RK3 steps the state agrees to 1e-10 relative.
Differences come only from floating-point contraction/ordering (the GPU fuses
multiply-adds).  The mixed form (FP32 tables and reconstruction on
differences, FP64 fluxes/accumulation/update) agrees with the FP64 engine to
2e-5 relative in the residual."""
import numpy as np
import pytest

from oracle import Oracle
from ucns3d_b200 import _native as N
from ucns3d_b200.config import EULER, NAVIER_STOKES, make_config
from ucns3d_b200.engine import Engine, EngineError
from ucns3d_b200.mesh import IC_TGV, IC_VORTEX, SCHEME_MUSCL, SCHEME_WENO, Mesh
from ucns3d_b200 import cases

pytestmark = pytest.mark.gpu

SMALL = {
    "muscl_ns_hex": (lambda: Mesh.box_hex(10, 10, 10), SCHEME_MUSCL, 1, 0, NAVIER_STOKES),
    "muscl_euler_tet": (lambda: Mesh.box_tet(5, 5, 5, seed=9), SCHEME_MUSCL, 1, 0, EULER),
    "weno3_tet": (lambda: Mesh.box_tet(5, 5, 5, seed=3), SCHEME_WENO, 2, 0, EULER),
    "weno5_hex": (lambda: Mesh.box_hex(12, 12, 12), SCHEME_WENO, 4, 0, EULER),
    "cweno4_tet": (lambda: Mesh.box_tet(5, 5, 5, seed=5), SCHEME_WENO, 3, 5, EULER),
    "cweno4_ns_mixed": (lambda: Mesh.mixed_box(8, seed=4), SCHEME_WENO, 3, 5, NAVIER_STOKES),
    "weno3_ns_hex": (lambda: Mesh.box_hex(8, 8, 8), SCHEME_WENO, 2, 0, NAVIER_STOKES),
    "muscl_bump": (lambda: Mesh.bump_channel(24, 10, 2, seed=2), SCHEME_MUSCL, 1, 0, EULER),
    "muscl_p2_hex": (lambda: Mesh.box_hex(8, 8, 8), SCHEME_MUSCL, 2, 0, EULER),
}


# far-field boundaries (code 6) on the two x sides of a box and, for the
# tetrahedra, the two y sides; and the bump channel under BOUNDTYPE 0
# (inflow faces take the free stream, outflow faces their own state)
SMALL["muscl_farfield_hex"] = (lambda: Mesh.box_hex(10, 6, 6, L=(3.0, 1.0, 1.0), periodic=(0, 1, 1),
                                                   bc=(6, 6, 0, 0, 0, 0)), SCHEME_MUSCL, 1, 0, EULER)
SMALL["weno3_farfield_tet"] = (lambda: Mesh.box_tet(6, 6, 4, L=(3.0, 2.0, 1.0), periodic=(0, 0, 1),
                                                    bc=(6, 6, 6, 6, 0, 0), seed=8), SCHEME_WENO, 2, 0, EULER)
SMALL["muscl_bump_bt0"] = (lambda: Mesh.bump_channel(24, 10, 2, seed=2), SCHEME_MUSCL, 1, 0, EULER)
FARFIELD = ("muscl_farfield_hex", "weno3_farfield_tet")
# Navier-Stokes on the bump channel: no-slip walls, inflow, outflow and
# symmetry faces (the bounded viscous fluxes of CALCULATE_BOUNDED_VISCOUS)
SMALL["muscl_ns_bump"] = (lambda: Mesh.bump_channel(24, 10, 2, seed=2), SCHEME_MUSCL, 1, 0, NAVIER_STOKES)
SMALL["weno3_ns_bump"] = (lambda: Mesh.bump_channel(16, 8, 8, seed=2), SCHEME_WENO, 2, 0, NAVIER_STOKES)
SMALL["cweno4_ns_bump"] = (lambda: Mesh.bump_channel(16, 8, 8, seed=2), SCHEME_WENO, 3, 5, NAVIER_STOKES)
BUMPLIKE = ("muscl_bump", "weno3_channel", "muscl_bump_bt0", "weno5_channel", "muscl_ns_bump", "weno3_ns_bump",
            "cweno4_ns_bump")

# characteristic-variable WENO (WENWRT 2) on the WENO cases, and on a
# channel with inflow/outflow/slip walls (boundary ghosts in the eigenvectors)
SMALL["weno3_channel"] = (lambda: Mesh.bump_channel(16, 8, 8, seed=2), SCHEME_WENO, 2, 0, EULER)
SMALL["weno5_channel"] = (lambda: Mesh.bump_channel(24, 12, 12, seed=2), SCHEME_WENO, 4, 0, EULER)
CHAR = ["weno3_tet", "weno5_hex", "cweno4_tet", "cweno4_ns_mixed", "weno3_channel", "weno3_ns_bump"]


def _setup(name, precision=N.UCG_FP64, wenwrt=1):
    mk, scheme, iorder, ees, gov = SMALL[name]
    m = mk().prepare(scheme, iorder, ees)
    p0 = 71.43
    bc = (1.0, 0.675 * np.sqrt(1.4), 0.0, 0.0, 1.0)
    cfg = make_config(m, governing=gov, precision=precision, reynolds=1600.0,
                      pres=p0 if gov == NAVIER_STOKES and name not in BUMPLIKE else 1.0,
                      prandtl=0.71, bc_state=bc, wenwrt=wenwrt, boundtype=0 if name.endswith("_bt0") else 1)
    if name in FARFIELD:
        # a stream along x whose density and speed vary across the box: the
        # far-field faces see inflow and outflow, subsonic and supersonic
        # (in the reference's test on the normal momentum |rho u_n| >= c)
        c = m.centres()
        rho = 1.0 + 0.5 * np.sin(2 * np.pi * c[:, 1] / 2.0 + 0.3)
        ux = np.sqrt(1.4) * (0.55 + 0.45 * np.cos(2 * np.pi * c[:, 1] / 2.0)) + 0.1 * np.sin(2 * np.pi * c[:, 0] / 3.0)
        uy = 0.3 * np.sin(2 * np.pi * c[:, 0] / 3.0)
        p = 1.0 + 0.1 * np.cos(2 * np.pi * c[:, 2])
        U = np.stack([rho, rho * ux, rho * uy, 0.0 * rho, p / 0.4 + 0.5 * rho * (ux * ux + uy * uy)], axis=1)
    elif name in BUMPLIKE:
        U = m.initial_condition(1, [1.4, *bc])
        # a smooth disturbance so that every branch sees non-trivial data
        c = m.centres()
        U[:, 0] *= 1.0 + 0.05 * np.sin(2 * np.pi * c[:, 0] / 3.0) * np.sin(np.pi * c[:, 1])
    else:
        U = m.initial_condition(IC_TGV, [1.4, p0 if gov == NAVIER_STOKES else 5.0, 1.0])
    return m, cfg, U


def _flux_scale(o, m, U):
    # magnitude of the face fluxes of a cell: |R| of a one-sided evaluation is
    # not available, so use the uniform-state flux scale of each cell
    g = m.geometry()
    r, u = U[:, 0], U[:, 1:4] / U[:, :1]
    p = 0.4 * (U[:, 4] - 0.5 * r * (u * u).sum(1))
    area = (g["face_area"] * (np.arange(6)[None, :] < g["nfaces"][:, None])).sum(1)
    s = np.abs(U).max(1) * (np.abs(u).max(1) + np.sqrt(1.4 * p / r)) + p
    return (s * area)[:, None]


@pytest.mark.parametrize("name", list(SMALL))
def test_residual_matches_oracle(name):
    m, cfg, U = _setup(name)
    o = Oracle(m, cfg)
    e = Engine(m, cfg)
    e.set_state(U)
    Rg = e.call_flux_subroutines_3d()
    Ro = o.residual(U)
    scale = _flux_scale(o, m, U)
    err = (np.abs(Rg - Ro) / scale).max()
    print(f"{name}: residual rel err {err:.3e}")
    assert err < 1e-12


@pytest.mark.parametrize("name", CHAR)
def test_characteristic_weno_residual_matches_oracle(name):
    """WENWRT 2: per-face eigenvector projection, indicators and weights per
    characteristic variable (CHARACTERISTIC_RECONSTRUCTION)."""
    m, cfg, U = _setup(name, wenwrt=2)
    o = Oracle(m, cfg)
    e = Engine(m, cfg)
    e.set_state(U)
    Rg = e.call_flux_subroutines_3d()
    Ro = o.residual(U)
    err = (np.abs(Rg - Ro) / _flux_scale(o, m, U)).max()
    print(f"{name} (characteristic): residual rel err {err:.3e}")
    assert err < 1e-12
    e.check_health()
    # the characteristic reconstruction is a different scheme: not the conserved one
    cfg1 = N.UcgConfig.from_buffer_copy(cfg)
    cfg1.wenwrt = 1
    assert np.abs(Rg - Oracle(m, cfg1).residual(U)).max() > 1e-10 * np.abs(Rg).max()


@pytest.mark.parametrize("riemann", [2, 3, 4, 5, 9])
@pytest.mark.parametrize("name", ["weno3_tet", "muscl_bump", "muscl_ns_hex"])
def test_rusanov_and_hll_match_oracle(name, riemann):
    """iRiemann 2 (Rusanov), 3 (Roe), 4 (rotated Roe-HLL), 5 (t-Roe) and 9
    (HLL) on the same kernels; on the bump's walls the mirrored velocity jump
    lies along n, the degenerate direction of the rotated solver."""
    m, cfg, U = _setup(name)
    cfg.riemann = riemann
    e = Engine(m, cfg)
    e.set_state(U)
    Rg = e.call_flux_subroutines_3d()
    o = Oracle(m, cfg)
    err = (np.abs(Rg - o.residual(U)) / _flux_scale(o, m, U)).max()
    print(f"{name} (riemann {riemann}): residual rel err {err:.3e}")
    assert err < 1e-12
    e.close()


@pytest.mark.parametrize("limiter", [1, 2, 4, 5, 6, 9])
@pytest.mark.parametrize("name", ["muscl_euler_tet", "muscl_bump", "muscl_p2_hex"])
def test_slope_limiters_match_oracle(name, limiter):
    """SLOPE_LIMITERS codes 1-9 in the MUSCL kernels (IORDER 1 and the
    high-order MUSCL of k_wpost)."""
    m, cfg, U = _setup(name)
    cfg.limiter = limiter
    e = Engine(m, cfg)
    e.set_state(U)
    Rg = e.call_flux_subroutines_3d()
    o = Oracle(m, cfg)
    err = (np.abs(Rg - o.residual(U)) / _flux_scale(o, m, U)).max()
    print(f"{name} (limiter {limiter}): residual rel err {err:.3e}")
    assert err < 1e-12
    e.close()


@pytest.mark.parametrize("name", ["weno3_tet", "weno5_hex"])
def test_characteristic_weno_mixed_close_to_fp64(name):
    m, cfg, U = _setup(name, wenwrt=2)
    _, cfgm, _ = _setup(name, precision=N.UCG_MIXED, wenwrt=2)
    out = []
    for c in (cfg, cfgm):
        e = Engine(m, c)
        e.set_state(U)
        out.append(e.call_flux_subroutines_3d())
        e.close()
    err = (np.abs(out[0] - out[1]) / _flux_scale(None, m, U)).max()
    print(f"{name} (characteristic): mixed vs fp64 residual rel err {err:.3e}")
    assert err < 2e-5


@pytest.mark.parametrize("name", ["muscl_ns_hex", "weno3_tet", "weno5_hex", "cweno4_tet", "muscl_bump", "muscl_ns_bump",
                                  "weno3_ns_bump"])
def test_rk3_steps_match_oracle(name):
    m, cfg, U = _setup(name)
    o = Oracle(m, cfg)
    e = Engine(m, cfg)
    e.set_state(U)
    Uo = U.copy()
    for _ in range(3):
        dt_g = e.calculate_cfl(0.5)
        dt_o = o.compute_dt(Uo, 0.5)
        assert abs(dt_g - dt_o) <= 1e-14 * dt_o
        e.runge_kutta3(dt_o)
        Uo = o.rk3_step(Uo, dt_o)
    Ug = e.get_state()
    err = (np.abs(Ug - Uo) / np.abs(Uo).max(0)).max()
    print(f"{name}: 3-step state rel err {err:.3e}")
    assert err < 1e-10
    e.check_health()


def test_device_dt_stepping_matches_host_dt():
    m, cfg, U = _setup("weno3_tet")
    a, b = Engine(m, cfg), Engine(m, cfg)
    a.set_state(U)
    b.set_state(U)
    for _ in range(2):
        dt = b.calculate_cfl(0.5)
        b.runge_kutta3(dt)
    a.time_marching(2, 0.5)
    np.testing.assert_array_equal(a.get_state(), b.get_state())


@pytest.mark.parametrize("name", ["weno5_hex", "cweno4_tet", "weno3_tet"])
@pytest.mark.parametrize("precision", [N.UCG_FP64, N.UCG_MIXED])
def test_bulk_copy_lsq_is_bitwise_equal(name, precision, monkeypatch):
    """The opt-in least squares through the shared-memory bulk-copy ring
    (UCG_LSQ_BULK=1 at engine creation) forms the same products in the same
    order as the default kernel: residuals equal bit for bit."""
    m, cfg, U = _setup(name, precision)
    out = []
    for bulk in ("0", "1"):
        monkeypatch.setenv("UCG_LSQ_BULK", bulk)
        e = Engine(m, cfg)
        e.set_state(U)
        out.append(e.residual())
        e.check_health()
        e.close()
    assert np.array_equal(out[0], out[1])


def test_bulk_copy_wait_timeout_is_reported_and_recoverable(monkeypatch):
    """The bounded waits of the opt-in bulk-copy least squares: with a wait
    limit of 0 polls every stage wait gives up, the warps drain their copies
    in flight and return, ucg_check_health reports UCG_ETIMEOUT, and with the
    default limit restored the same handle gives the normal residual bit for
    bit."""
    m, cfg, U = _setup("weno5_hex", N.UCG_MIXED)
    monkeypatch.setenv("UCG_LSQ_BULK", "1")
    e = Engine(m, cfg)
    e.set_state(U)
    ref = e.residual()
    e.check_health()
    assert e.lib.ucg_set_wait_limit(e._h, 0) == N.UCG_OK
    e.residual()
    with pytest.raises(EngineError) as ei:
        e.check_health()
    assert ei.value.code == N.UCG_ETIMEOUT
    assert e.lib.ucg_set_wait_limit(e._h, -1) == N.UCG_OK
    e.set_state(U)
    again = e.residual()
    e.check_health()
    assert np.array_equal(again, ref)
    e.close()


def test_bitwise_deterministic():
    m, cfg, U = _setup("weno3_tet")
    out = []
    for _ in range(2):
        e = Engine(m, cfg)
        e.set_state(U)
        e.time_marching(3, 0.5)
        out.append(e.get_state())
        e.close()
    assert np.array_equal(out[0], out[1])


def test_enstrophy_matches_oracle():
    m, cfg, U = _setup("muscl_ns_hex")
    e = Engine(m, cfg)
    e.set_state(U)
    a, b = e.enstrophy(), Oracle(m, cfg).enstrophy(U)
    assert abs(a - b) <= 1e-12 * abs(b), (a, b)
    m2, cfg2, U2 = _setup("weno3_ns_hex")
    e2 = Engine(m2, cfg2)
    e2.set_state(U2)
    with pytest.raises(EngineError) as ei:
        e2.enstrophy()
    assert ei.value.code == N.UCG_EINVAL


def test_reductions_match_oracle():
    m, cfg, U = _setup("weno5_hex")
    o = Oracle(m, cfg)
    e = Engine(m, cfg)
    e.set_state(U)
    for what in (N.UCG_REDUCE_KE, N.UCG_REDUCE_MASS, N.UCG_REDUCE_ENERGY):
        a, b = e.reduce(what), o.reduce(U, what)
        assert abs(a - b) <= 1e-13 * abs(b)


@pytest.mark.parametrize("name", ["weno5_hex", "weno3_tet", "muscl_ns_hex", "cweno4_tet", "cweno4_ns_mixed",
                                  "weno3_ns_hex", "weno3_ns_bump"])
def test_mixed_precision_close_to_fp64(name):
    m, cfg64, U = _setup(name, N.UCG_FP64)
    _, cfg32, _ = _setup(name, N.UCG_MIXED)
    cfg32 = N.UcgConfig.from_buffer_copy(cfg64)
    cfg32.precision = N.UCG_MIXED
    a, b = Engine(m, cfg64), Engine(m, cfg32)
    a.set_state(U)
    b.set_state(U)
    Ra, Rb = a.call_flux_subroutines_3d(), b.call_flux_subroutines_3d()
    err = (np.abs(Ra - Rb) / _flux_scale(None, m, U)).max()
    print(f"{name}: mixed vs fp64 residual rel err {err:.3e}")
    assert err < 2e-5


def test_mixed_weno5_vortex_density_error():
    """Isentropic vortex, WENO5: after 20 RK3 steps the mixed form's density
    stays within 1e-6 relative L2 of the FP64 form."""
    c64 = cases.vortex_hex_weno5(n=16)
    c32 = cases.vortex_hex_weno5(n=16, precision=N.UCG_MIXED)
    a, b = Engine(c64.mesh, c64.cfg), Engine(c32.mesh, c32.cfg)
    a.set_state(c64.U0)
    b.set_state(c32.U0)
    a.time_marching(20, 0.5)
    b.time_marching(20, 0.5)
    ra, rb = a.get_state()[:, 0], b.get_state()[:, 0]
    l2 = np.sqrt(np.mean((ra - rb) ** 2)) / np.sqrt(np.mean(ra ** 2))
    print(f"vortex mixed vs fp64 density L2 {l2:.3e}")
    assert l2 < 1e-6


def test_mixed_weno5_vortex_100_steps_against_fp64_and_analytic():
    """Isentropic vortex, WENO5, 100 RK3 steps at one fixed dt: the mixed
    form's density stays within 1e-6 relative L2 of the FP64 form, and its
    error against the analytic solution (the vortex advected by the free
    stream) is the FP64 form's error to within 1 %."""
    from ucns3d_b200.cases import vortex_params
    c64 = cases.vortex_hex_weno5(n=16)
    c32 = cases.vortex_hex_weno5(n=16, precision=N.UCG_MIXED)
    a, b = Engine(c64.mesh, c64.cfg), Engine(c32.mesh, c32.cfg)
    a.set_state(c64.U0)
    b.set_state(c32.U0)
    dt = a.calculate_cfl(0.5)
    for _ in range(100):
        a.runge_kutta3(dt)
        b.runge_kutta3(dt)
    ra, rb = a.get_state()[:, 0], b.get_state()[:, 0]
    ex = c64.mesh.initial_condition(IC_VORTEX, vortex_params(c64.meta["L"], t=100 * dt))[:, 0]

    def rel_l2(x, y):
        return np.sqrt(np.mean((x - y) ** 2)) / np.sqrt(np.mean(y ** 2))

    l2, ea, eb = rel_l2(rb, ra), rel_l2(ra, ex), rel_l2(rb, ex)
    print(f"100 steps: mixed vs fp64 {l2:.3e}, fp64 vs analytic {ea:.3e}, mixed vs analytic {eb:.3e}")
    assert l2 < 1e-6
    assert abs(eb - ea) <= 0.01 * ea


def test_nonphysical_state_is_reported_not_trapped():
    m, cfg, U = _setup("muscl_ns_hex")
    e = Engine(m, cfg)
    bad = U.copy()
    bad[5, 0] = -1.0
    e.set_state(bad)
    e.runge_kutta3(1e-3)
    with pytest.raises(EngineError) as ei:
        e.check_health()
    assert ei.value.code == N.UCG_ENONPHYS
    # the context stays usable
    e.set_state(U)
    e.runge_kutta3(1e-3)
    e.check_health()


def test_call_order_is_checked():
    m, cfg, U = _setup("weno3_tet")
    e = Engine(m, cfg, upload=False)
    with pytest.raises(EngineError) as ei:
        e.runge_kutta3(1e-3)
    assert ei.value.code == N.UCG_ESTATE
    import ctypes as C
    assert e.lib.ucg_set_state(e._h, N.ptr(U, C.c_double), m.ncells - 1) == N.UCG_EINVAL
    e.upload_geometry(m.geometry_struct())
    e.upload_recon(m.recon_struct())
    e.set_state(U)
    e.runge_kutta3(1e-3)
    e.check_health()


@pytest.mark.parametrize("name", ["weno5_hex", "weno5_channel"])
@pytest.mark.parametrize("precision", [N.UCG_FP64, N.UCG_MIXED])
def test_indicator_kernel_is_bitwise_equal(name, precision, monkeypatch):
    """WENO5: the smoothness indicators formed by k_wis (one warp per
    stencil of a 32-cell group, the default at IORDER 4) and inside k_wpost
    (UCG_WENO_IS=0 at engine creation) are the same quadratic forms in the
    same order: residuals equal bit for bit (the channel adds cells on the
    MUSCL fall-back, which k_wis skips)."""
    m, cfg, U = _setup(name, precision)
    monkeypatch.setenv("UCG_WENO_FACE", "0")
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("UCG_WENO_IS", flag)
        e = Engine(m, cfg)
        e.set_state(U)
        out.append(e.residual())
        e.check_health()
        e.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("name", ["weno5_hex", "weno5_channel", "weno5_shock"])
@pytest.mark.parametrize("precision", [N.UCG_FP64, N.UCG_MIXED])
def test_variable_warp_face_values_match_lane_per_cell(name, precision, monkeypatch):
    """WENO5: the weights, combined polynomial and face values formed one
    warp per conserved variable (k_wface, then the MUSCL fall-back of the
    cells it flags) against one lane per cell (k_wpost, UCG_WENO_FACE=0).
    Both take the same operations in the same order; only the compiler's
    multiply-add contraction may differ, so the residuals agree to the
    rounding of the reconstruction's type: 1e-12 of the flux scale in FP64,
    2e-6 in the mixed form.  The shock case (a Sod-like jump across the
    box) sends the cells beside the jump to the fall-back through CHECKSOL."""
    m, cfg, U = _setup("weno5_hex" if name == "weno5_shock" else name, precision)
    if name == "weno5_shock":
        x = m.centres()[:, 0]
        left = x < 0.5 * (x.min() + x.max())
        rho, pr = np.where(left, 1.0, 0.125), np.where(left, 1.0, 0.1)
        U = np.zeros_like(U)
        U[:, 0], U[:, 4] = rho, pr / 0.4
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("UCG_WENO_FACE", flag)
        e = Engine(m, cfg)
        e.set_state(U)
        out.append(e.residual())
        e.check_health()
        e.close()
    err = (np.abs(out[0] - out[1]) / _flux_scale(None, m, U)).max()
    print(f"{name}: k_wface vs k_wpost rel err {err:.3e}, bitwise {np.array_equal(out[0], out[1])}")
    assert err < (1e-12 if precision == N.UCG_FP64 else 2e-6)
