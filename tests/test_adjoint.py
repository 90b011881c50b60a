"""Discrete adjoint (VJP) and tangent (JVP) of the MUSCL residual, the wall
force and SSP-RK3 steps on the bump channel (hexahedra + prisms, inflow,
outflow, slip walls), FP64 form, through the C ABI.

Checks, as the adjoint's contract asks:
  * force J against the oracle's COMPUTEFORCE restatement (1e-12 relative);
  * residual JVP against central finite differences of the oracle's FP64
    residual, in the state and in the free-stream state (FD step 1e-6 of the
    perturbation scale; truncation error O(eps^2));
  * dot-product test <lam, JVP(du, dp)> = <VJP_U(lam), du> + <VJP_p(lam), dp>
    (1e-12 relative: both sides are the same derivatives);
  * through RK3 steps with checkpoints: tangent run vs adjoint run (dot
    product), adjoint run vs finite differences of J after the same steps of
    the oracle, and independence of the checkpoint stride.
Base states: the free stream marched from the inflow (limiters active at the
bump) plus a seeded 3D perturbation, so that no two states tie (see
_generic_state).
"""
import numpy as np
import pytest

from ucns3d_b200 import _native as N
from ucns3d_b200 import cases
from ucns3d_b200.engine import Engine, EngineError

pytestmark = pytest.mark.gpu


def _generic_state(c, nsteps, seed):
    """The free stream marched `nsteps` steps (limiters active at the bump),
    then a 3% perturbation that varies in x, y and z: the base state must be
    generic, since at exactly equal states (a z-invariant flow on a layered
    mesh) the Einfeldt wave-speed min/max of HLLC and the FIND_BOUNDS min/max
    have ties where the residual has no derivative."""
    e = Engine(c.mesh, c.cfg)
    e.set_state(c.U0)
    e.time_marching(nsteps, 0.5)
    U = e.get_state()
    rng = np.random.default_rng(seed)
    cc = c.mesh.centres()
    U = U * (1.0 + 0.03 * np.sin(3.1 * cc[:, :1] + 1.7 * cc[:, 1:2] + 40.0 * cc[:, 2:3] + rng.uniform(0, 6.3, (1, 5))))
    e.set_state(U)
    return e, U


@pytest.fixture(scope="module")
def bump():
    from oracle import Oracle
    c = cases.bump_muscl(nx=60, ny=20, nlayers=4)
    e, U = _generic_state(c, 40, 7)
    dt = e.calculate_cfl(0.5)
    yield dict(case=c, engine=e, U=U, dt=dt, oracle=Oracle(c.mesh, c.cfg))
    e.close()


@pytest.fixture(scope="module")
def short_bump():
    """A short channel, so that the inflow state reaches the bump within the
    200 steps of the adjoint runs."""
    c = cases.bump_muscl(nx=24, ny=8, nlayers=4)
    e, U = _generic_state(c, 20, 11)
    dt = e.calculate_cfl(0.5)
    yield dict(case=c, engine=e, U=U, dt=dt)
    e.close()


def _cfg_with_bc(cfg, bc):
    out = N.UcgConfig.from_buffer_copy(cfg)
    for k in range(5):
        out.bc_state[k] = bc[k]
    return out


def _directions(U, seed):
    rng = np.random.default_rng(seed)
    du = rng.standard_normal(U.shape) * np.abs(U).max(0) * 1e-2
    dp = rng.standard_normal(5) * np.array([1.0, 0.8, 0.0, 0.0, 1.0]) * 1e-2
    return du, dp


def test_force_matches_oracle(bump):
    e, o, U = bump["engine"], bump["oracle"], bump["U"]
    e.set_state(U)
    a, b = e.force(), o.force(U)
    assert abs(a - b) <= 1e-12 * max(1.0, abs(b)), (a, b)


def test_residual_jvp_matches_oracle_fd(bump):
    from oracle import Oracle
    c, e, U = bump["case"], bump["engine"], bump["U"]
    e.set_state(U)
    du, dp = _directions(U, 1)
    jvp = e.residual_jvp(du, dp)
    eps = 1e-6
    bc = np.array([c.cfg.bc_state[k] for k in range(5)])
    op = Oracle(c.mesh, _cfg_with_bc(c.cfg, bc + eps * dp))
    om = Oracle(c.mesh, _cfg_with_bc(c.cfg, bc - eps * dp))
    fd = (op.residual(U + eps * du) - om.residual(U - eps * du)) / (2 * eps)
    scale = np.abs(fd).max(0) + 1e-300
    err = (np.abs(jvp - fd) / scale).max(1)
    # measured: median 3e-9, max 3e-8 (the FD's own roundoff at this step)
    assert err.max() < 1e-6, np.sort(err)[-5:]
    assert np.median(err) < 1e-7


def test_vjp_jvp_dot_product(bump):
    e, U = bump["engine"], bump["U"]
    e.set_state(U)
    du, dp = _directions(U, 2)
    lam = np.random.default_rng(3).standard_normal(U.shape)
    jvp = e.residual_jvp(du, dp)
    mu, pbar = e.residual_vjp(lam)
    a = float(np.sum(lam * jvp))
    b = float(np.sum(mu * du) + np.sum(pbar * dp))
    assert abs(a - b) <= 1e-12 * (np.abs(lam * jvp).sum()), (a, b)


def test_force_vjp_matches_fd(bump):
    e, U = bump["engine"], bump["U"]
    du, _ = _directions(U, 4)
    e.set_state(U)
    g = e.force_vjp()
    eps = 1e-6
    e.set_state(U + eps * du)
    jp = e.force()
    e.set_state(U - eps * du)
    jm = e.force()
    e.set_state(U)
    fd = (jp - jm) / (2 * eps)
    ad = float(np.sum(g * du))
    assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1e-30), (ad, fd)


NSTEPS, EVERY = 200, 20


def test_adjoint_run_matches_tangent_run(short_bump):
    e, U, dt = short_bump["engine"], short_bump["U"], short_bump["dt"]
    du, dp = _directions(U, 5)
    e.set_state(U)
    J1, dJ = e.tangent_run(NSTEPS, dt, du, dp)
    e.set_state(U)
    J2, g, gp = e.adjoint_run(NSTEPS, dt, every=EVERY)
    assert J1 == J2
    ad = float(np.sum(g * du) + np.sum(gp * dp))
    assert abs(ad - dJ) <= 1e-10 * max(abs(dJ), 1e-30), (ad, dJ)


def test_adjoint_run_matches_oracle_fd(short_bump):
    from oracle import Oracle
    c, e, U, dt = short_bump["case"], short_bump["engine"], short_bump["U"], short_bump["dt"]
    e.set_state(U)
    J, g, gp = e.adjoint_run(NSTEPS, dt, every=EVERY)
    bc = np.array([c.cfg.bc_state[k] for k in range(5)])

    def J_oracle(U0, bcs):
        o = Oracle(c.mesh, _cfg_with_bc(c.cfg, bcs))
        W = U0.copy()
        for _ in range(NSTEPS):
            W = o.rk3_step(W, dt)
        return o.force(W)

    assert abs(J_oracle(U, bc) - J) <= 1e-10 * max(1.0, abs(J))
    eps = 1e-6
    du, dp = _directions(U, 6)
    fd_u = (J_oracle(U + eps * du, bc) - J_oracle(U - eps * du, bc)) / (2 * eps)
    fd_p = (J_oracle(U, bc + eps * dp) - J_oracle(U, bc - eps * dp)) / (2 * eps)
    ad_u, ad_p = float(np.sum(g * du)), float(np.sum(gp * dp))
    assert abs(ad_u - fd_u) <= 1e-5 * max(abs(fd_u), 1e-30), (ad_u, fd_u)
    assert abs(ad_p - fd_p) <= 1e-5 * max(abs(fd_p), 1e-30), (ad_p, fd_p)


def test_checkpoint_stride_does_not_change_gradients(short_bump):
    e, U, dt = short_bump["engine"], short_bump["U"], short_bump["dt"]
    out = []
    for every in (1, 7, EVERY, NSTEPS):
        e.set_state(U)
        out.append(e.adjoint_run(NSTEPS, dt, every=every))
    for J, g, gp in out[1:]:
        assert J == out[0][0]
        assert np.array_equal(g, out[0][1]) and np.array_equal(gp, out[0][2])


def test_torch_autograd_function(bump):
    """The residual as a torch.autograd.Function (test harness only):
    backward is the engine's VJP; the gradient of a scalar built on it
    matches finite differences."""
    import torch
    e, U = bump["engine"], bump["U"]

    class Residual(torch.autograd.Function):
        @staticmethod
        def forward(ctx, u):
            e.set_state(u.detach().cpu().numpy())
            ctx.save_for_backward(u)
            return torch.from_numpy(e.residual())

        @staticmethod
        def backward(ctx, g):
            (u,) = ctx.saved_tensors
            e.set_state(u.detach().cpu().numpy())
            mu, _ = e.residual_vjp(g.detach().cpu().numpy())
            return torch.from_numpy(mu)

    w = torch.from_numpy(np.random.default_rng(8).standard_normal(U.shape))
    u = torch.from_numpy(U.copy()).requires_grad_(True)
    Jt = (w * Residual.apply(u)).sum()
    (gu,) = torch.autograd.grad(Jt, u)
    du, _ = _directions(U, 9)
    eps = 1e-6
    with torch.no_grad():
        jp = float((w * Residual.apply(torch.from_numpy(U + eps * du))).sum())
        jm = float((w * Residual.apply(torch.from_numpy(U - eps * du))).sum())
    fd = (jp - jm) / (2 * eps)
    ad = float((gu * torch.from_numpy(du)).sum())
    assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)
    e.set_state(U)


@pytest.mark.parametrize("name", ["weno3_tet", "weno5_hex", "cweno4_tet", "cweno4_tet_wenoz"])
def test_weno_vjp_matches_oracle_fd(name):
    """VJP and JVP of the WENO and CWENO residuals (nonlinear weights, WENO-Z
    weights for CWENO, smoothness indicators, stencil least squares, HLLC at
    every face point) against central differences of the oracle's FP64
    residual, and the dot-product test between them, on periodic meshes
    whose cells are all on the WENO branch."""
    from oracle import Oracle
    from ucns3d_b200.config import make_config
    from ucns3d_b200.mesh import IC_TGV, SCHEME_WENO, Mesh
    if name == "weno3_tet":
        m = Mesh.box_tet(5, 5, 5, seed=3).prepare(SCHEME_WENO, 2)
    elif name.startswith("cweno4_tet"):
        m = Mesh.box_tet(5, 5, 5, seed=5).prepare(SCHEME_WENO, 3, 5)
    else:
        m = Mesh.box_hex(10, 10, 10).prepare(SCHEME_WENO, 4)
    cfg = make_config(m, governing=2, wenoz=int(name.endswith("wenoz")))
    U = m.initial_condition(IC_TGV, [1.4, 5.0, 1.0])
    rng = np.random.default_rng(12)
    cc = m.centres()
    U = U * (1.0 + 0.02 * np.sin(1.3 * cc[:, :1] + 0.7 * cc[:, 1:2] + 2.1 * cc[:, 2:3] + rng.uniform(0, 6.3, (1, 5))))
    e = Engine(m, cfg)
    e.set_state(U)
    lam = rng.standard_normal(U.shape)
    mu, pbar = e.residual_vjp(lam)
    assert np.all(pbar == 0.0)  # periodic: no free-stream dependence
    o = Oracle(m, cfg)
    if name.endswith("wenoz"):  # the WENO-Z weights give another residual
        R0 = Oracle(m, make_config(m, governing=2)).residual(U)
        assert np.abs(o.residual(U) - R0).max() > 1e-8 * np.abs(R0).max()
    eps = 1e-6
    for trial in range(2):
        du = rng.standard_normal(U.shape) * np.abs(U).max(0) * 1e-2
        fdv = (o.residual(U + eps * du) - o.residual(U - eps * du)) / (2 * eps)
        fd = float(np.sum(lam * fdv))
        ad = float(np.sum(mu * du))
        assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1e-30), (trial, ad, fd)
        # the tangent: against the same differences, and the dot-product test
        jvp = e.residual_jvp(du)
        err = (np.abs(jvp - fdv) / (np.abs(fdv).max(0) + 1e-300)).max()
        print(f"{name}: WENO JVP vs oracle differences {err:.2e}")
        assert err < 1e-6
        a, b = float(np.sum(lam * jvp)), ad
        assert abs(a - b) <= 1e-12 * np.abs(lam * jvp).sum(), (a, b)
    e.close()


@pytest.mark.parametrize("order,ees", [(2, 0), (3, 5)])
def test_weno_adjoint_with_muscl_fall_back(order, ees):
    """WENO3 and CWENO4 on the bump channel (slip walls, inflow/outflow):
    the cells next to the boundaries are not FULL and take the MUSCL
    fall-back (the central stencil polynomial limited by Venkatakrishnan
    with FIND_BOUNDS over the face neighbours), others may fail CHECKSOL.
    VJP and JVP in the state and the free-stream state against central
    differences of the oracle's FP64 residual, and the dot-product test."""
    from oracle import Oracle
    from ucns3d_b200.config import make_config
    from ucns3d_b200.mesh import SCHEME_WENO, Mesh
    m = Mesh.bump_channel(16, 8, 8, seed=2).prepare(SCHEME_WENO, order, ees)
    g = m.geometry_struct()
    full = np.ctypeslib.as_array(g.full, shape=(m.ncells,))
    assert 0 < full.sum() < m.ncells  # both branches present
    bc = np.array([1.0, 0.8, 0.0, 0.0, 1.0])
    cfg = make_config(m, governing=2, bc_state=tuple(bc))
    rng = np.random.default_rng(17)
    cc = m.centres()
    U = np.tile([1.0, 0.8, 0.0, 0.0, 1.0 / 0.4 + 0.32], (m.ncells, 1))
    U = U * (1.0 + 0.03 * np.sin(3.1 * cc[:, :1] + 1.7 * cc[:, 1:2] + 9.0 * cc[:, 2:3] + rng.uniform(0, 6.3, (1, 5))))
    e = Engine(m, cfg)
    e.set_state(U)
    lam = rng.standard_normal(U.shape)
    mu, pbar = e.residual_vjp(lam)
    eps = 1e-6
    for trial in range(2):
        du, dp = _directions(U, 30 + trial)
        fdv = (Oracle(m, _cfg_with_bc(cfg, bc + eps * dp)).residual(U + eps * du) -
               Oracle(m, _cfg_with_bc(cfg, bc - eps * dp)).residual(U - eps * du)) / (2 * eps)
        fd = float(np.sum(lam * fdv))
        ad = float(np.sum(mu * du) + np.sum(pbar * dp))
        assert abs(ad - fd) <= 1e-6 * abs(fd), (trial, ad, fd)
        jvp = e.residual_jvp(du, dp)
        err = (np.abs(jvp - fdv) / (np.abs(fdv).max(0) + 1e-300)).max()
        print(f"order {order} ees {ees}: WENO JVP vs oracle differences {err:.2e}")
        assert err < 1e-6
        a = float(np.sum(lam * jvp))
        assert abs(a - ad) <= 1e-12 * np.abs(lam * jvp).sum(), (a, ad)
    e.close()


@pytest.mark.parametrize("name", ["weno3_tet_ns", "cweno4_ns_mixed", "bump_cweno4_ns"])
def test_weno_ns_vjp_jvp_match_oracle_fd(name):
    """Navier-Stokes WENO/CWENO: the reverse of the viscous fluxes at every
    face point, of the face-point gradients (SOLUTIONTRIAV2 on both sides,
    averaged), of the viscous coefficients and least squares, on top of the
    inviscid WENO reverse.  VJP and JVP in the state (and, on the channel,
    the free-stream state) against central differences of the oracle's FP64
    residual, and the dot-product test between them.  Re 50, so that the
    viscous terms are a sizeable part of the derivative."""
    from oracle import Oracle
    from ucns3d_b200.config import NAVIER_STOKES, make_config
    from ucns3d_b200.mesh import IC_TGV, SCHEME_WENO, Mesh
    rng = np.random.default_rng(18)
    bc = np.array([1.0, 0.8, 0.0, 0.0, 1.0])
    if name == "bump_cweno4_ns":  # no-slip walls, inflow/outflow, MUSCL fall-back next to the walls
        m = Mesh.bump_channel(16, 8, 8, seed=2).prepare(SCHEME_WENO, 3, 5)
        U = np.tile([1.0, 0.8, 0.0, 0.0, 1.0 / 0.4 + 0.32], (m.ncells, 1))
        cfg = make_config(m, governing=NAVIER_STOKES, reynolds=50.0, pres=1.0, bc_state=tuple(bc))
    else:
        if name == "weno3_tet_ns":
            m = Mesh.box_tet(5, 5, 5, seed=3).prepare(SCHEME_WENO, 2)
        else:
            m = Mesh.mixed_box(6, seed=4).prepare(SCHEME_WENO, 3, 5)
        U = m.initial_condition(IC_TGV, [1.4, 5.0, 1.0])
        cfg = make_config(m, governing=NAVIER_STOKES, reynolds=50.0, pres=5.0, bc_state=tuple(bc))
    cc = m.centres()
    U = U * (1.0 + 0.03 * np.sin(3.1 * cc[:, :1] + 1.7 * cc[:, 1:2] + 2.3 * cc[:, 2:3] + rng.uniform(0, 6.3, (1, 5))))
    e = Engine(m, cfg)
    e.set_state(U)
    lam = rng.standard_normal(U.shape)
    mu, pbar = e.residual_vjp(lam)
    # the viscous part matters: the Euler residual's derivative differs
    cfg_e = make_config(m, governing=2, bc_state=tuple(bc))
    eps = 1e-6
    for trial in range(2):
        du, dp = _directions(U, 50 + trial)
        if not name.startswith("bump"):
            dp = np.zeros(5)
        Rp = Oracle(m, _cfg_with_bc(cfg, bc + eps * dp)).residual(U + eps * du)
        Rm = Oracle(m, _cfg_with_bc(cfg, bc - eps * dp)).residual(U - eps * du)
        fdv = (Rp - Rm) / (2 * eps)
        if trial == 0:
            fde = (Oracle(m, _cfg_with_bc(cfg_e, bc + eps * dp)).residual(U + eps * du) -
                   Oracle(m, _cfg_with_bc(cfg_e, bc - eps * dp)).residual(U - eps * du)) / (2 * eps)
            assert np.abs(fdv - fde).max() > 1e-2 * np.abs(fdv).max()
        fd = float(np.sum(lam * fdv))
        ad = float(np.sum(mu * du) + np.sum(pbar * dp))
        print(f"{name}: NS WENO VJP {ad:.12e} vs oracle differences {fd:.12e}")
        assert abs(ad - fd) <= 1e-6 * abs(fd), (trial, ad, fd)
        jvp = e.residual_jvp(du, dp)
        scale = np.abs(fdv).max(0) + 1e-300
        err = (np.abs(jvp - fdv) / scale).max(1)
        # a limiter branch switch (the MUSCL fall-back's FIND_BOUNDS and
        # Venkatakrishnan min) within the step: there the tangent must match
        # the one-sided difference from the side without the switch
        R0 = Oracle(m, cfg).residual(U)
        one = np.minimum((np.abs(jvp - (Rp - R0) / eps) / scale).max(1), (np.abs(jvp - (R0 - Rm) / eps) / scale).max(1))
        kink = err >= 1e-6
        print(f"{name}: NS WENO JVP vs oracle differences max {err.max():.2e}, median {np.median(err):.2e}; "
              f"{kink.sum()} cells with a branch switch within eps")
        assert kink.sum() <= max(4, len(err) // 200), np.sort(err)[-10:]
        assert (one[kink] < 1e-5).all(), one[kink]
        a = float(np.sum(lam * jvp))
        assert abs(a - ad) <= 1e-12 * np.abs(lam * jvp).sum(), (a, ad)
    e.close()


def test_adjoint_rejects_other_configurations():
    c = cases.vortex_hex_weno5(n=8, wenwrt=2)  # characteristic variables
    e = Engine(c.mesh, c.cfg)
    e.set_state(c.U0)
    with pytest.raises(EngineError) as ei:
        e.force()
    assert ei.value.code == N.UCG_EINVAL
    e.close()


def _weno_run_case(name):
    """Small WENO/CWENO cases for the adjoint runs: periodic tetrahedra
    (every cell on the WENO branch) and the bump channel (MUSCL fall-back
    next to the walls, inflow/outflow ghosts), Euler, or Navier-Stokes at
    Re 50 (`_ns`: no-slip walls on the channel), with a generic perturbed
    state."""
    from ucns3d_b200.config import NAVIER_STOKES, make_config
    from ucns3d_b200.mesh import IC_TGV, SCHEME_WENO, Mesh
    rng = np.random.default_rng(21)
    ns = name.endswith("_ns")
    gov = dict(governing=NAVIER_STOKES, reynolds=50.0, pres=1.0) if ns else dict(governing=2)
    if name.startswith("bump"):
        order, ees = (3, 5) if "cweno4" in name else (2, 0)
        m = Mesh.bump_channel(16, 8, 4, seed=2).prepare(SCHEME_WENO, order, ees)
        bc = (1.0, 0.8, 0.0, 0.0, 1.0)
        cfg = make_config(m, bc_state=bc, **gov)
        U = np.tile([1.0, 0.8, 0.0, 0.0, 1.0 / 0.4 + 0.32], (m.ncells, 1))
    elif ns:
        m = Mesh.box_tet(4, 4, 4, seed=3).prepare(SCHEME_WENO, 3, 5)
        cfg = make_config(m, governing=NAVIER_STOKES, reynolds=50.0, pres=5.0)
        U = m.initial_condition(IC_TGV, [1.4, 5.0, 1.0])
    else:
        m = Mesh.box_tet(4, 4, 4, seed=3).prepare(SCHEME_WENO, *((2, 0) if name == "weno3_tet" else (3, 5)))
        cfg = make_config(m, governing=2)
        U = m.initial_condition(IC_TGV, [1.4, 5.0, 1.0])
    cc = m.centres()
    U = U * (1.0 + 0.02 * np.sin(1.3 * cc[:, :1] + 0.7 * cc[:, 1:2] + 2.1 * cc[:, 2:3] + rng.uniform(0, 6.3, (1, 5))))
    return m, cfg, U


WENO_RUN_STEPS, WENO_RUN_EVERY = 12, 5


@pytest.mark.parametrize("name", ["weno3_tet", "cweno4_tet", "bump_weno3", "cweno4_tet_ns", "bump_cweno4_ns"])
def test_weno_adjoint_run_kinetic_energy(name):
    """Adjoint through 12 SSP-RK3 steps of the WENO/CWENO residual with
    checkpoints every 5 (J = domain kinetic energy): against central
    differences of J after the same steps of the oracle (state and, on the
    channel, free-stream state; 1e-5), against the tangent run (1e-10) and
    independent of the checkpoint stride (bitwise)."""
    from oracle import Oracle
    m, cfg, U = _weno_run_case(name)
    e = Engine(m, cfg)
    e.set_state(U)
    # CWENO4 Navier-Stokes on the channel (every cell on the MUSCL fall-back,
    # Re 50, the no-slip walls started impulsively) diverges within two
    # steps at half the CFL step, in the oracle as in the engine; 0.1 of it
    # keeps the run bounded
    dt = (0.1 if name == "bump_cweno4_ns" else 0.5) * e.calculate_cfl(0.5)
    e.set_state(U)
    J, g, gp = e.adjoint_run(WENO_RUN_STEPS, dt, every=WENO_RUN_EVERY, objective=N.UCG_OBJ_KE)
    bc = np.array([cfg.bc_state[k] for k in range(5)])

    def J_oracle(U0, bcs):
        o = Oracle(m, _cfg_with_bc(cfg, bcs))
        W = U0.copy()
        for _ in range(WENO_RUN_STEPS):
            W = o.rk3_step(W, dt)
        return o.reduce(W, N.UCG_REDUCE_KE)

    assert abs(J_oracle(U, bc) - J) <= 1e-12 * abs(J)
    eps = 1e-6
    du, dp = _directions(U, 41)
    fd_u = (J_oracle(U + eps * du, bc) - J_oracle(U - eps * du, bc)) / (2 * eps)
    ad_u = float(np.sum(g * du))
    print(f"{name}: adjoint run dJ/dU0.du {ad_u:.10e}, oracle differences {fd_u:.10e}")
    assert abs(ad_u - fd_u) <= 1e-5 * abs(fd_u), (ad_u, fd_u)
    if name.startswith("bump"):
        # dJ/dp.dp is ~1e-5 of J here, so the free-stream difference takes a
        # step of 1e-3 (at 1e-6 it carries rounding of ~1e-4 relative; the
        # differences at 1e-3 and 1e-2 agree to 1e-8)
        eps_p = 1e-3
        fd_p = (J_oracle(U, bc + eps_p * dp) - J_oracle(U, bc - eps_p * dp)) / (2 * eps_p)
        ad_p = float(np.sum(gp * dp))
        print(f"{name}: dJ/dp.dp {ad_p:.10e}, oracle differences {fd_p:.10e}")
        assert abs(ad_p - fd_p) <= 1e-5 * abs(fd_p), (ad_p, fd_p)
    else:
        assert np.all(gp == 0.0)
    e.set_state(U)
    J1, dJ = e.tangent_run(WENO_RUN_STEPS, dt, du, dp, objective=N.UCG_OBJ_KE)
    assert J1 == J
    ad = float(np.sum(g * du) + np.sum(gp * dp))
    assert abs(ad - dJ) <= 1e-10 * abs(dJ), (ad, dJ)
    e.set_state(U)
    J2, g2, gp2 = e.adjoint_run(WENO_RUN_STEPS, dt, every=1, objective=N.UCG_OBJ_KE)
    assert J2 == J and np.array_equal(g2, g) and np.array_equal(gp2, gp)
    e.close()


@pytest.mark.parametrize("name", ["bump_weno3", "bump_cweno4_ns"])
def test_weno_wall_force(name):
    """The wall force of WENO/CWENO states, summed over the quadrature points
    of the wall faces (COMPUTEFORCE): J against the oracle (1e-12), its VJP
    against central differences of the engine's J (1e-6), and through 12
    SSP-RK3 steps the adjoint run against the oracle's differences (1e-5)
    and the tangent run (1e-10)."""
    from oracle import Oracle
    m, cfg, U = _weno_run_case(name)
    o = Oracle(m, cfg)
    e = Engine(m, cfg)
    e.set_state(U)
    J0 = e.force()
    assert J0 != 0.0
    assert abs(J0 - o.force(U)) <= 1e-12 * abs(J0), (J0, o.force(U))
    du, dp = _directions(U, 43)
    g = e.force_vjp()
    eps = 1e-6
    e.set_state(U + eps * du)
    jp = e.force()
    e.set_state(U - eps * du)
    jm = e.force()
    fd = (jp - jm) / (2 * eps)
    ad = float(np.sum(g * du))
    assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)
    e.set_state(U)
    dt = (0.1 if name == "bump_cweno4_ns" else 0.5) * e.calculate_cfl(0.5)
    e.set_state(U)
    J, g, gp = e.adjoint_run(WENO_RUN_STEPS, dt, every=WENO_RUN_EVERY, objective=N.UCG_OBJ_FORCE_X)
    bc = np.array([cfg.bc_state[k] for k in range(5)])

    def J_oracle(U0, bcs):
        ob = Oracle(m, _cfg_with_bc(cfg, bcs))
        W = U0.copy()
        for _ in range(WENO_RUN_STEPS):
            W = ob.rk3_step(W, dt)
        return ob.force(W)

    assert abs(J_oracle(U, bc) - J) <= 1e-12 * abs(J)
    fd_u = (J_oracle(U + eps * du, bc) - J_oracle(U - eps * du, bc)) / (2 * eps)
    ad_u = float(np.sum(g * du))
    print(f"{name}: force adjoint run dJ/dU0.du {ad_u:.10e}, oracle differences {fd_u:.10e}")
    assert abs(ad_u - fd_u) <= 1e-5 * abs(fd_u), (ad_u, fd_u)
    # the free stream reaches the wall within 12 steps only through the
    # inflow cells: dJ/dp.dp is 1e-9 (WENO3) and 1e-7 (CWENO4 NS) of J, so
    # the difference carries rounding of ~1e-4 relative at a step of 1e-3
    # (steps 1e-2, 1e-3 and 1e-4 agree to 3e-4 and 4e-4)
    eps_p = 1e-3
    fd_p = (J_oracle(U, bc + eps_p * dp) - J_oracle(U, bc - eps_p * dp)) / (2 * eps_p)
    ad_p = float(np.sum(gp * dp))
    print(f"{name}: force dJ/dp.dp {ad_p:.10e}, oracle differences {fd_p:.10e}")
    assert abs(ad_p - fd_p) <= 2e-3 * abs(fd_p), (ad_p, fd_p)
    e.set_state(U)
    J1, dJ = e.tangent_run(WENO_RUN_STEPS, dt, du, dp, objective=N.UCG_OBJ_FORCE_X)
    assert J1 == J
    ad = float(np.sum(g * du) + np.sum(gp * dp))
    assert abs(ad - dJ) <= 1e-10 * abs(dJ), (ad, dJ)
    e.close()


def test_muscl_adjoint_run_kinetic_energy(short_bump):
    """The kinetic-energy objective on the MUSCL channel: adjoint run
    against the tangent run (1e-10), with a free-stream gradient that is not
    vacuous (the inflow state changes the kinetic energy of the cells next
    to it from the first step)."""
    e, U, dt = short_bump["engine"], short_bump["U"], short_bump["dt"]
    du, dp = _directions(U, 43)
    e.set_state(U)
    J1, dJ = e.tangent_run(NSTEPS, dt, du, dp, objective=N.UCG_OBJ_KE)
    e.set_state(U)
    J2, g, gp = e.adjoint_run(NSTEPS, dt, every=EVERY, objective=N.UCG_OBJ_KE)
    assert J1 == J2
    ad = float(np.sum(g * du) + np.sum(gp * dp))
    assert abs(ad - dJ) <= 1e-10 * abs(dJ), (ad, dJ)
    assert np.abs(gp).max() > 1e-8


# ---------------------------------------------------------------- viscous
# Navier-Stokes MUSCL: the reverse of the viscous fluxes (Dual<1> columns of
# viscous_flux per face and input), of the cells' gradients of (T, u, v, w)
# through the frame and the viscous least squares, and of the no-slip wall
# ghost; the tangent runs the same viscous path on Dual<1> numbers.

def _ns_case(c, reynolds=200.0):
    from ucns3d_b200.config import NAVIER_STOKES, make_config
    cfg = make_config(c.mesh, governing=NAVIER_STOKES, reynolds=reynolds, pres=1.0,
                      bc_state=tuple(c.cfg.bc_state[k] for k in range(5)))
    return cases.Case(c.name + "_ns", c.mesh, cfg, c.U0, c.cfl, c.steps, dict(c.meta, equations="NS"))


def _ns_tgv():
    from ucns3d_b200.config import NAVIER_STOKES, make_config
    from ucns3d_b200.mesh import IC_TGV, SCHEME_MUSCL, Mesh
    m = Mesh.box_hex(8, 8, 8).prepare(SCHEME_MUSCL, 1)
    cfg = make_config(m, governing=NAVIER_STOKES, reynolds=100.0, pres=71.43)
    U0 = m.initial_condition(IC_TGV, [1.4, 71.43, 1.0])
    return cases.Case("tgv_ns", m, cfg, U0, 0.5, 10, dict(equations="NS"))


@pytest.fixture(scope="module", params=["bump", "tgv"])
def ns_case(request):
    from oracle import Oracle
    if request.param == "bump":
        c = _ns_case(cases.bump_muscl(nx=60, ny=20, nlayers=4))
        e, U = _generic_state(c, 40, 17)
    else:
        c = _ns_tgv()
        e, U = _generic_state(c, 5, 19)
    yield dict(case=c, engine=e, U=U, oracle=Oracle(c.mesh, c.cfg), name=request.param)
    e.close()


def test_ns_residual_jvp_matches_oracle_fd(ns_case):
    from oracle import Oracle
    c, e, U = ns_case["case"], ns_case["engine"], ns_case["U"]
    e.set_state(U)
    du, dp = _directions(U, 21)
    jvp = e.residual_jvp(du, dp)
    eps = 1e-6
    bc = np.array([c.cfg.bc_state[k] for k in range(5)])
    op = Oracle(c.mesh, _cfg_with_bc(c.cfg, bc + eps * dp))
    om = Oracle(c.mesh, _cfg_with_bc(c.cfg, bc - eps * dp))
    Rp, Rm = op.residual(U + eps * du), om.residual(U - eps * du)
    R0 = ns_case["oracle"].residual(U)
    fd = (Rp - Rm) / (2 * eps)
    scale = np.abs(fd).max(0) + 1e-300
    err = (np.abs(jvp - fd) / scale).max(1)
    # A branch switch of the limiters (FIND_BOUNDS min/max, the Barth-Jespersen
    # min(1, .)) or of the HLLC wave speeds inside [-eps, eps] along the
    # direction makes the central difference average two slopes; the tangent
    # takes the branch at U itself, so at those cells it must match the
    # one-sided difference from the side without the switch.
    one = np.minimum((np.abs(jvp - (Rp - R0) / eps) / scale).max(1),
                     (np.abs(jvp - (R0 - Rm) / eps) / scale).max(1))
    kink = err >= 1e-6
    print(f"{ns_case['name']}: NS JVP vs oracle FD, max {err.max():.2e}, median {np.median(err):.2e}; "
          f"{kink.sum()} cells with a branch switch within eps, one-sided max "
          f"{one[kink].max() if kink.any() else 0.0:.2e}")
    assert kink.sum() <= max(8, len(err) // 500), np.sort(err)[-10:]
    assert (one[kink] < 1e-5).all(), one[kink]
    assert np.median(err) < 1e-7


def test_ns_vjp_jvp_dot_product(ns_case):
    e, U = ns_case["engine"], ns_case["U"]
    e.set_state(U)
    du, dp = _directions(U, 22)
    lam = np.random.default_rng(23).standard_normal(U.shape)
    jvp = e.residual_jvp(du, dp)
    mu, pbar = e.residual_vjp(lam)
    a = float(np.sum(lam * jvp))
    b = float(np.sum(mu * du) + np.sum(pbar * dp))
    print(f"{ns_case['name']}: NS dot product {a:.15e} vs {b:.15e}")
    assert abs(a - b) <= 1e-12 * (np.abs(lam * jvp).sum()), (a, b)


@pytest.fixture(scope="module")
def short_ns_bump():
    c = _ns_case(cases.bump_muscl(nx=24, ny=8, nlayers=4))
    e, U = _generic_state(c, 20, 31)
    dt = e.calculate_cfl(0.5)
    yield dict(case=c, engine=e, U=U, dt=dt)
    e.close()


def test_ns_adjoint_run_matches_tangent_run_and_oracle_fd(short_ns_bump):
    """100 Navier-Stokes RK3 steps with checkpoints every 20, wall force: the
    adjoint run against the tangent run (dot product) and against central
    differences of J after the same steps of the oracle."""
    from oracle import Oracle
    c, e, U, dt = short_ns_bump["case"], short_ns_bump["engine"], short_ns_bump["U"], short_ns_bump["dt"]
    nsteps = 100
    du, dp = _directions(U, 32)
    e.set_state(U)
    J1, dJ = e.tangent_run(nsteps, dt, du, dp)
    e.set_state(U)
    J2, g, gp = e.adjoint_run(nsteps, dt, every=EVERY)
    assert J1 == J2
    ad = float(np.sum(g * du) + np.sum(gp * dp))
    assert abs(ad - dJ) <= 1e-10 * max(abs(dJ), 1e-30), (ad, dJ)
    bc = np.array([c.cfg.bc_state[k] for k in range(5)])

    def J_oracle(U0, bcs):
        o = Oracle(c.mesh, _cfg_with_bc(c.cfg, bcs))
        W = U0.copy()
        for _ in range(nsteps):
            W = o.rk3_step(W, dt)
        return o.force(W)

    assert abs(J_oracle(U, bc) - J2) <= 1e-10 * max(1.0, abs(J2))
    eps = 1e-6
    fd_u = (J_oracle(U + eps * du, bc) - J_oracle(U - eps * du, bc)) / (2 * eps)
    # the far-field state reaches the wall force only weakly within 100 steps
    # (dJ/dp.dp ~ 5e-7 against J ~ 2e-2), so at eps = 1e-6 the difference is
    # rounding (|J| 1e-16 / eps ~ 4e-12); at 1e-4 and 1e-3 it agrees to 3e-7
    eps_p = 1e-4
    fd_p = (J_oracle(U, bc + eps_p * dp) - J_oracle(U, bc - eps_p * dp)) / (2 * eps_p)
    ad_u, ad_p = float(np.sum(g * du)), float(np.sum(gp * dp))
    print(f"NS adjoint run: dJ/dU.du {ad_u:.9e} vs FD {fd_u:.9e}; dJ/dp.dp {ad_p:.9e} vs FD {fd_p:.9e}")
    assert abs(ad_u - fd_u) <= 1e-5 * max(abs(fd_u), 1e-30), (ad_u, fd_u)
    assert abs(ad_p - fd_p) <= 1e-5 * max(abs(fd_p), 1e-30), (ad_p, fd_p)
