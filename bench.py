"""Benchmark: cell-RK-stage updates per second of the explicit residual
engine on one B200 (or N independent replicas under torchrun; with
--partition, one mesh split over the N ranks).

Default workload: the isentropic vortex on a periodic 64^3 hexahedral box
(262,144 cells), Euler, 5th-order WENO + HLLC, SSP-RK3 - the mixed-precision
form (FP32 tables/reconstruction on differences, FP64 fluxes/accumulation/
update) is the headline `value`; the all-FP64 form is measured in the same
run and the two are compared by their relative L2 density difference.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is device-resident throughput (dt kept on the device, no host sync
inside the timed region); `e2e` goes through the public API with host
buffers (pinned), the host->device copy of the state and the device->host
read of the result inside every timed step.  Inputs are larger than L2 (the
reconstruction tables alone are tens of GB), so no L2 flush is needed.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-RK-stage updates/s"
UNIT = "cell-stage/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default="vortex_hex_weno5")
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--wenwrt", type=int, default=1, choices=[1, 2],
                    help="WENO variables: 1 conserved, 2 characteristic (vortex_hex_weno5)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint timing (bump channel)")
    ap.add_argument("--adjoint-only", action="store_true", help="only the adjoint timing (bump channel)")
    ap.add_argument("--adjoint-steps", type=int, default=200, help="RK3 steps of the adjoint run")
    ap.add_argument("--adjoint-every", type=int, default=20, help="checkpoint stride of the adjoint run")
    ap.add_argument("--adjoint-weno-n", type=int, default=32,
                    help="hexahedra per side of the vortex timed for the WENO VJP/JVP")
    ap.add_argument("--accuracy-steps", type=int, default=None,
                    help="RK3 steps of the accuracy run (mixed against FP64; the vortex also against the analytic "
                         "solution): default 100 for the vortex, the workload's own step count otherwise; 0 skips")
    ap.add_argument("--shuffle", action="store_true",
                    help="hand the mesh over in a seeded random cell numbering (as from a partitioner) and time "
                         "it with the engine's renumbering on (the line's value) and off (shuffle.reorder_off)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--implicit", action="store_true",
                    help="also time implicit steps (ucg_implicit_step) against explicit RK3 on the bump channel")
    ap.add_argument("--setup", action="store_true",
                    help="also time the reconstruction-table set-up: host (ucp_prepare + upload) against the "
                         "device (ucg_build_recon) on meshes with one matrix set per cell")
    ap.add_argument("--partition", action="store_true",
                    help="split the mesh over the ranks (recursive coordinate bisection, a halo of cell states "
                         "moved over NCCL in every RK stage: strong scaling) instead of one replica per rank")
    ap.add_argument("--cpu-n", type=int, default=0,
                    help="mesh size of the CPU baseline and reference arm (0: the benchmarked --n)")
    return ap.parse_args()


def dist_init():
    """One process per GPU under torchrun: replicas (no data exchange), or
    the partitions of one mesh with --partition."""
    import torch
    import torch.distributed as dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws, local):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = f"cuda:{local}" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# nominal HBM3e bandwidth of a B200 (HGX figure), reported beside the
# measured copy peak
NOMINAL_HBM_GBS = 7700.0


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# DRAM traffic of one k_lsq launch per cell, dram__bytes_read.sum +
# dram__bytes_write.sum of a one-kernel ncu capture divided by the cells of
# the captured mesh, keyed by (workload, precision).  Only measured entries
# are listed; other workloads report traffic null.  The k_lsq traffic grows
# in proportion to the cells (no re-reads between cells), so a launch on a
# larger mesh of the same workload moves this times its cells.
#   vortex_hex_weno5, mixed: 32^3 capture, 1.00x the algorithmic bytes
LSQ_DRAM_BYTES_PER_CELL = {("vortex_hex_weno5", 1): 106_700}


def lsq_bytes_per_cell(cfg):
    """Algorithmic bytes of k_lsq per cell: the pseudo-inverse slices and
    stencil indices of every stencil, the cell's own state, and the stencil
    polynomials G written (neighbour states come through L2; they are
    counted once, in the flux kernel)."""
    from ucns3d_b200 import _native as N
    s = 4 if cfg.precision == N.UCG_MIXED else 8
    b = 5 * 8
    for ll in range(cfg.admis_max):
        low = cfg.ees == 5 and ll > 0
        nk, nd = (cfg.imax2, cfg.ideg2) if low else (cfg.imax, cfg.ideg)
        b += s * nk * nd + 4 * nk + s * nd * 5
    return b


def recon_bytes_per_cell(cfg):
    """Algorithmic bytes the reconstruction kernel must move per cell: the
    pseudo-inverses, stencil indices, smoothness matrix, face quadrature
    points and basis means of the cell, its own state and its face values
    written (neighbour state counted once, in the flux kernel)."""
    from ucns3d_b200 import _native as N
    s = 4 if cfg.precision == N.UCG_MIXED else 8
    nq = max(cfg.nq_quad, cfg.nq_tri)
    b = s * cfg.ideg * cfg.imax * cfg.admis_max + 4 * (cfg.imax + 1) * cfg.admis_max
    if cfg.scheme == 3:  # packed upper triangle of the smoothness matrix
        b += s * cfg.ideg * (cfg.ideg + 1) // 2
    b += s * 6 * nq * 3 + s * cfg.ideg + 5 * 8
    b += s * 6 * nq * 5  # face values written
    return b


def recon_kernels(cfg, wenwrt):
    """The kernels of one reconstruction (the launch sequence of launch_weno)."""
    if cfg.scheme == 2 and cfg.iorder == 1:
        return "k_muscl"
    if cfg.scheme == 3 and cfg.iorder == 4 and wenwrt == 1:
        return "k_lsq + k_wis + k_wface + k_wpost fall-back"
    return "k_lsq + k_wpost"


L2_BYTES = 126 * 2 ** 20


def scheme_label(case, wenwrt):
    """e.g. 'WENO5+HLLC SSP-RK3, Euler' from the case's metadata."""
    m = case.meta
    name = {"WENO": f"WENO{m.get('order', '')}", "CWENO": f"CWENO{m.get('order', '')}",
            "MUSCL": "MUSCL"}.get(m.get("scheme"), str(m.get("scheme")))
    s = f"{name}+HLLC SSP-RK3, {m.get('equations', '')}"
    return s + (" (characteristic variables)" if wenwrt == 2 else "")


def make_case(args, precision):
    from ucns3d_b200 import cases
    fn = cases.CASES[args.case]
    kw = {"precision": precision}
    if args.case in ("tgv_hex_muscl", "tgv_tet_weno3", "vortex_hex_weno5", "mixed_cweno4"):
        kw["n"] = args.n
    if args.case == "vortex_hex_weno5" and args.wenwrt != 1:
        kw["wenwrt"] = args.wenwrt
    c = fn(**kw)
    if args.shuffle:
        import numpy as np
        from ucns3d_b200.mesh import RenumberedMesh
        order = np.random.default_rng(2024).permutation(c.mesh.ncells)
        c = cases.Case(c.name, RenumberedMesh(c.mesh, order), c.cfg, np.ascontiguousarray(c.U0[order]), c.cfl,
                       c.steps, dict(c.meta, shuffled=True))
    return c


def run_gpu(args, case, ws, local, timed_e2e=True):
    import numpy as np
    import torch
    from ucns3d_b200.engine import Engine

    eng = Engine(case.mesh, case.cfg, device=local)
    eng.set_state(case.U0)
    # warm-up (also JIT/allocations)
    eng.time_marching(args.warmup, case.cfl)
    eng.synchronize()
    eng.check_health()
    stream = torch.cuda.ExternalStream(eng.stream_ptr, device=f"cuda:{local}")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    barrier(ws)
    torch.cuda.synchronize(local)
    sampler.start()
    l0 = eng.launch_count
    ev0.record(stream)
    eng.time_marching(args.steps, case.cfl)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize(local)
    launches = eng.launch_count - l0
    clocks = sampler.stop()
    barrier(ws)
    ms = ev0.elapsed_time(ev1)
    eng.check_health()
    kern = eng.time_kernels(reps=3)
    state = eng.get_state()
    e2e = None
    if timed_e2e:
        # public API with pinned host buffers: H2D of the state, one step, D2H
        hin = torch.from_numpy(state).pin_memory()
        hout = torch.empty_like(hin).pin_memory()
        nin, nout = hin.numpy(), hout.numpy()
        eng.set_state(nin)
        eng.time_marching(1, case.cfl)
        eng.get_state(nout)
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            eng.set_state(nin)
            eng.time_marching(1, case.cfl)
            eng.get_state(nout)
        t1 = time.perf_counter()
        e2e = dict(seconds=t1 - t0, bytes_in=nin.nbytes, bytes_out=nout.nbytes)
    nbytes_dev = eng.device_bytes
    co = eng.cell_order()
    order = {"renumbered": co["renumbered"], "gather_cost_caller": co["cost_caller"], "gather_cost_rcm": co["cost_rcm"]}
    eng.close()
    return dict(ms=ms, kern=kern, state=state, clocks=clocks, launches=launches, e2e=e2e, device_bytes=nbytes_dev,
                order=order)


def run_accuracy(case, local, steps):
    """`steps` RK3 steps at one fixed dt (CFL from the initial state) in the
    FP64 and the mixed form on the same mesh: the density of mixed against
    FP64 (relative L2 and Linf) and, for the isentropic vortex, of each
    against the analytic solution (the initial vortex advected by the free
    stream for steps * dt)."""
    import numpy as np
    from ucns3d_b200 import _native as N
    from ucns3d_b200.cases import vortex_params
    from ucns3d_b200.engine import Engine
    from ucns3d_b200.mesh import IC_VORTEX

    rho = {}
    dt = None
    for prec in (N.UCG_FP64, N.UCG_MIXED):
        cfg = N.UcgConfig.from_buffer_copy(case.cfg)
        cfg.precision = prec
        eng = Engine(case.mesh, cfg, device=local)
        eng.set_state(case.U0)
        if dt is None:
            dt = eng.calculate_cfl(case.cfl)
        for _ in range(steps):
            eng.runge_kutta3(dt)
        eng.check_health()
        rho[prec] = eng.get_state()[:, 0].copy()
        eng.close()

    def err(a, b):
        return {"rel_l2": float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2))),
                "rel_linf": float(np.abs(a - b).max() / np.abs(b).max())}

    out = {"steps": steps, "dt": dt, "t": steps * dt,
           "density_mixed_vs_fp64": err(rho[N.UCG_MIXED], rho[N.UCG_FP64])}
    if case.name == "vortex_hex_weno5":
        exact = case.mesh.initial_condition(IC_VORTEX, vortex_params(case.meta["L"], t=steps * dt))[:, 0]
        out["density_fp64_vs_analytic"] = err(rho[N.UCG_FP64], exact)
        out["density_mixed_vs_analytic"] = err(rho[N.UCG_MIXED], exact)
    return out


def cpu_case(args):
    """The workload prepared for the oracle (FP64 tables), at the bench's own
    size unless --cpu-n asks for another."""
    from ucns3d_b200 import _native as N
    from ucns3d_b200 import cases
    fn = cases.CASES[args.case]
    kw = {"precision": N.UCG_FP64}
    if args.case in ("tgv_hex_muscl", "tgv_tet_weno3", "vortex_hex_weno5", "mixed_cweno4"):
        kw["n"] = args.cpu_n or args.n
    if args.case == "vortex_hex_weno5" and args.wenwrt != 1:
        kw["wenwrt"] = args.wenwrt
    return fn(**kw)


def cpu_stages(case, cfg, stages):
    """The oracle (FP64 CPU restatement, OpenMP over all host threads) for
    `stages` consecutive SSP-RK3 stages of the workload on its full mesh;
    seconds of the stage calls alone (set-up excluded)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle
    o = Oracle(case.mesh, cfg)
    Un = case.U0.copy()
    U = Un.copy()
    dt = o.compute_dt(Un, case.cfl)
    t = 0.0
    for k in range(stages):
        stage = k % 3 + 1
        if stage == 1:
            Un[:] = U
        t0 = time.perf_counter()
        o.rk3_stage(Un, U, dt, stage)
        t += time.perf_counter() - t0
    return t


def host_cores():
    thr = os.environ.get("OMP_NUM_THREADS")
    return int(thr) if thr else os.cpu_count()


def cpu_sample(args, case=None, stages=3):
    """cpu_baseline: the oracle on one SSP-RK3 step (3 stages) of the same
    workload and mesh, all host threads."""
    from ucns3d_b200 import _native as N
    if case is None:
        case = cpu_case(args)
    cfg = N.UcgConfig.from_buffer_copy(case.cfg)
    cfg.precision = N.UCG_FP64
    t = cpu_stages(case, cfg, stages)
    n = case.mesh.ncells
    return dict(value=n * stages / t, cores=host_cores(), seconds=t, ncells=n,
                sample=f"{args.case}, {n} cells (the benchmarked mesh), {stages} SSP-RK3 stage(s), "
                       f"oracle FP64 CPU restatement, OpenMP")


def main_reference(args, ws, rank, local):
    """The reference arm: the CPU restatement of the reference path (the
    Fortran reference cannot be built on this image) on the host cores, on
    the benchmarked workload and mesh; each step is one SSP-RK3 stage of
    that mesh (a full RK3 step takes three), one stage of warm-up."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from ucns3d_b200 import _native as N
    orc.build()
    case = cpu_case(args)
    cfg = N.UcgConfig.from_buffer_copy(case.cfg)
    cfg.precision = N.UCG_FP64
    cpu_stages(case, cfg, 1)
    t = cpu_stages(case, cfg, args.steps)
    n = case.mesh.ncells
    value = n * args.steps / t
    sample = (f"{args.case}, {n} cells (the benchmarked mesh), {args.steps} SSP-RK3 stages timed after 1 "
              f"warm-up stage, oracle FP64 CPU restatement, OpenMP")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.case, "cells": n, "n": args.cpu_n or args.n,
                   "scheme": scheme_label(case, args.wenwrt),
                   "step": "one SSP-RK3 stage of the full mesh (the metric counts cell-stages); "
                           "1 warm-up stage whatever --warmup says"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": host_cores(), "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_adjoint(local, steps=200, every=20, weno_n=32):
    """Adjoint cost on the bump channel (240x80 quads half split into
    triangles, 4 layers: hexahedra + prisms, MUSCL + HLLC, FP64): device
    times of the residual, its VJP and JVP at a marched state, then a
    checkpointed adjoint run of `steps` RK3 steps (checkpoints every
    `every`) against the same steps of the primal alone."""
    import torch
    from ucns3d_b200 import cases
    from ucns3d_b200.engine import Engine
    c = cases.bump_muscl()
    eng = Engine(c.mesh, c.cfg, device=local)
    eng.set_state(c.U0)
    eng.time_marching(50, c.cfl)
    U = eng.get_state()
    dt = eng.calculate_cfl(c.cfl)
    t = eng.time_adjoint(reps=10)
    stream = torch.cuda.ExternalStream(eng.stream_ptr, device=f"cuda:{local}")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    eng.set_state(U)
    ev[0].record(stream)
    for _ in range(steps):
        eng.runge_kutta3(dt)
    ev[1].record(stream)
    ev[1].synchronize()
    eng.set_state(U)
    ev[2].record(stream)
    J, g, gp = eng.adjoint_run(steps, dt, every)
    ev[3].record(stream)
    ev[3].synchronize()
    primal, adj = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3])
    eng.close()
    # the same run on the short channel (24x8 quads, 4 layers), where the
    # inflow state reaches the bump within the window, so that dJ/dp is not
    # vacuous; checked against the tangent run along a seeded direction
    import numpy as np
    cs = cases.bump_muscl(nx=24, ny=8, nlayers=4)
    es = Engine(cs.mesh, cs.cfg, device=local)
    es.set_state(cs.U0)
    es.time_marching(20, cs.cfl)
    Us = es.get_state()
    dts = es.calculate_cfl(cs.cfl)
    es.set_state(Us)
    Js, gs, gps = es.adjoint_run(steps, dts, every)
    rng = np.random.default_rng(5)
    du = rng.standard_normal(Us.shape) * np.abs(Us).max(0) * 1e-2
    dp = rng.standard_normal(5) * np.array([1.0, 0.8, 0.0, 0.0, 1.0]) * 1e-2
    es.set_state(Us)
    _, dJs = es.tangent_run(steps, dts, du, dp)
    es.close()
    short = {"workload": "bump_muscl 24x8x4", "cells": cs.mesh.ncells, "run_steps": steps, "J": Js,
             "dJdp": [float(x) for x in gps],
             "adjoint_vs_tangent_rel": abs(float(np.sum(gs * du) + np.sum(gps * dp)) - dJs) / abs(dJs)}
    out = {"workload": "bump_muscl", "cells": c.mesh.ncells, "dtype": "f64", "residual_ms": t["residual"],
           "vjp_ms": t["vjp"], "jvp_ms": t["jvp"], "vjp_over_residual": t["vjp"] / t["residual"],
           "run_steps": steps, "checkpoint_every": every, "primal_run_ms": primal, "adjoint_run_ms": adj,
           "adjoint_run_over_primal_run": adj / primal, "J": J,
           "dJdp": [float(x) for x in gp],
           "dJdp_note": "inflow changes reach the bump only after about 500 steps at this size, so dJ/dp is "
                        "physically near zero over the 200-step window; see short_channel",
           "short_channel": short}
    # the Navier-Stokes residual's VJP/JVP on the same channel (Re 200,
    # no-slip walls on BC 4), at the free stream marched 50 steps
    from ucns3d_b200.config import NAVIER_STOKES, make_config
    cfg_ns = make_config(c.mesh, governing=NAVIER_STOKES, reynolds=200.0, pres=1.0,
                         bc_state=tuple(c.cfg.bc_state[k] for k in range(5)))
    en = Engine(c.mesh, cfg_ns, device=local)
    en.set_state(c.U0)
    en.time_marching(50, c.cfl)
    tn = en.time_adjoint(reps=10)
    en.close()
    out["ns"] = {"workload": "bump_muscl_ns Re 200", "cells": c.mesh.ncells, "dtype": "f64",
                 "residual_ms": tn["residual"], "vjp_ms": tn["vjp"], "jvp_ms": tn["jvp"],
                 "vjp_over_residual": tn["vjp"] / tn["residual"]}
    # the CWENO4 Navier-Stokes residual's VJP/JVP on the mixed-element box
    # (the 2.1 M-cell workload's scheme at n = 24)
    from ucns3d_b200 import _native as N
    cm = cases.mixed_cweno4(n=24, precision=N.UCG_FP64)
    em = Engine(cm.mesh, cm.cfg, device=local)
    em.set_state(cm.U0)
    tm = em.time_adjoint(reps=5)
    em.close()
    out["weno_ns"] = {"workload": "mixed_cweno4 n=24", "cells": cm.mesh.ncells, "dtype": "f64",
                      "residual_ms": tm["residual"], "vjp_ms": tm["vjp"], "jvp_ms": tm["jvp"],
                      "vjp_over_residual": tm["vjp"] / tm["residual"]}
    # the WENO residual's VJP/JVP (FP64 form) on the vortex, weno_n^3 hexahedra
    from ucns3d_b200 import _native as N
    from ucns3d_b200.engine import EngineError
    cw = cases.vortex_hex_weno5(n=weno_n, precision=N.UCG_FP64)
    ew = Engine(cw.mesh, cw.cfg, device=local)
    ew.set_state(cw.U0)
    try:
        tw = ew.time_adjoint(reps=5)
        out["weno"] = {"workload": "vortex_hex_weno5", "cells": cw.mesh.ncells, "dtype": "f64",
                       "residual_ms": tw["residual"], "vjp_ms": tw["vjp"], "jvp_ms": tw["jvp"],
                       "vjp_over_residual": tw["vjp"] / tw["residual"]}
        # checkpointed adjoint run of the WENO5 vortex (J = kinetic energy)
        # against the primal steps alone
        dtw = ew.calculate_cfl(cw.cfl)
        nw, kw = 20, 5
        stream_w = torch.cuda.ExternalStream(ew.stream_ptr, device=f"cuda:{local}")
        evw = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ew.set_state(cw.U0)
        evw[0].record(stream_w)
        for _ in range(nw):
            ew.runge_kutta3(dtw)
        evw[1].record(stream_w)
        evw[1].synchronize()
        ew.set_state(cw.U0)
        evw[2].record(stream_w)
        Jw, _, _ = ew.adjoint_run(nw, dtw, kw, objective=N.UCG_OBJ_KE)
        evw[3].record(stream_w)
        evw[3].synchronize()
        pw, aw = evw[0].elapsed_time(evw[1]), evw[2].elapsed_time(evw[3])
        out["weno"].update({"run_steps": nw, "checkpoint_every": kw, "objective": "kinetic energy",
                            "primal_run_ms": pw, "adjoint_run_ms": aw, "adjoint_run_over_primal_run": aw / pw,
                            "J": Jw})
    except EngineError as err:
        out["weno"] = {"unavailable": str(err)}
    ew.close()
    return out


def run_implicit(local):
    """The bump channel (MUSCL + HLLC, Euler, 240 x 80 x 4 layers) from the
    free stream toward its steady state: implicit steps at CFL 50
    (IMPLICIT_TIMEs, 10 relaxation sweeps) against explicit RK3 steps at CFL
    0.9, each timed with CUDA events on the engine stream; the residual norm
    relative to the free stream's after each run."""
    import numpy as np
    import torch
    from ucns3d_b200 import cases
    from ucns3d_b200.engine import Engine
    c = cases.bump_muscl()
    out = {"workload": "bump_muscl 240x80x4", "cells": c.mesh.ncells}
    for kind, steps in (("implicit", 200), ("explicit_rk3", 2000)):
        e = Engine(c.mesh, c.cfg, device=local)
        e.set_state(c.U0)
        r0 = float(np.linalg.norm(e.call_flux_subroutines_3d()))
        stream = torch.cuda.ExternalStream(e.stream_ptr, device=f"cuda:{local}")
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e.synchronize()
        ev0.record(stream)
        if kind == "implicit":
            e.implicit_step(50.0, steps, 10)
        else:
            e.time_marching(steps, 0.9)
        ev1.record(stream)
        ev1.synchronize()
        e.check_health()
        r1 = float(np.linalg.norm(e.call_flux_subroutines_3d()))
        ms = ev0.elapsed_time(ev1)
        out[kind] = {"steps": steps, "cfl": 50.0 if kind == "implicit" else 0.9, "ms": ms, "ms_per_step": ms / steps,
                     "residual_ratio": r1 / r0}
        e.close()
    return out


def run_setup(local):
    """Start-up time of the reconstruction tables on meshes whose cells all
    have their own matrix sets (jittered tetrahedra): the host set-up
    library's tables (the difference between ucp_prepare and
    ucp_prepare_geometry, all host threads) plus their upload
    (ucg_upload_recon), against ucg_build_recon on the device; wall-clock
    seconds of each synchronous call, and whether the residuals agree bit
    for bit."""
    import os
    import numpy as np
    from ucns3d_b200.config import make_config, EULER
    from ucns3d_b200.engine import Engine
    from ucns3d_b200.mesh import IC_TGV, SCHEME_WENO, Mesh
    out = []
    for name, mk, io in (("tets 16^3x6, WENO5", lambda: Mesh.box_tet(16, 16, 16, seed=7), 4),
                         ("tets 24^3x6, WENO3", lambda: Mesh.box_tet(24, 24, 24, seed=7), 2)):
        mg, mh = mk(), mk()
        t0 = time.perf_counter()
        mg.prepare(SCHEME_WENO, io, tables=False)
        t1 = time.perf_counter()
        mh.prepare(SCHEME_WENO, io)
        t2 = time.perf_counter()
        cfg = make_config(mh, governing=EULER)
        U = mh.initial_condition(IC_TGV, [1.4, 5.0, 1.0])
        eh, ed = Engine(mh, cfg, device=local, upload=False), Engine(mg, cfg, device=local, upload=False)
        eh.upload_geometry(mh.geometry_struct())
        ed.upload_geometry(mg.geometry_struct())
        t3 = time.perf_counter()
        eh.upload_recon(mh.recon_struct())
        t4 = time.perf_counter()
        ed.build_recon(mg.shapes_struct(), mg.recon_struct())
        t5 = time.perf_counter()
        res = []
        for e in (eh, ed):
            e.set_state(U)
            res.append(e.call_flux_subroutines_3d())
            e.close()
        host_tables = (t2 - t1) - (t1 - t0)
        out.append({"workload": name, "cells": mh.ncells, "matrix_sets": mh.ntables, "host_threads": os.cpu_count(),
                    "host_tables_s": host_tables, "upload_s": t4 - t3, "host_total_s": host_tables + (t4 - t3),
                    "device_build_s": t5 - t4, "speedup": (host_tables + (t4 - t3)) / (t5 - t4),
                    "residual_bitwise_equal": bool(np.array_equal(res[0], res[1]))})
    return out


def main_partition(args, ws, rank, local):
    """The workload split over the ranks (ucns3d_b200.partition): every rank
    builds the same mesh and plan, steps its partition with halo transfers in
    each stage and CFL time steps reduced over the ranks; value = the whole
    mesh's cell-stages per second, timed on the device as the slowest rank."""
    import numpy as np
    import torch
    from ucns3d_b200 import _native as N
    from ucns3d_b200.partition import HaloEngine, PartitionPlan, rcb

    case = make_case(args, N.UCG_MIXED)
    ncells = case.mesh.ncells
    plan = PartitionPlan(case.mesh, rcb(case.mesh.centres(), ws))
    h = HaloEngine(plan, rank, case.cfg, device=local)
    h.set_state(case.U0)
    for _ in range(args.warmup):
        h.rk3_step(h.compute_dt(case.cfl))
    h.engine.synchronize()
    h.engine.check_health()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    barrier(ws)
    torch.cuda.synchronize(local)
    sampler.start()
    l0 = h.engine.launch_count
    ev0.record(h.stream)
    for _ in range(args.steps):
        h.rk3_step(h.compute_dt(case.cfl))
    ev1.record(h.stream)
    ev1.synchronize()
    torch.cuda.synchronize(local)
    launches = h.engine.launch_count - l0
    clocks = sampler.stop()
    barrier(ws)
    ms = max_over_ranks(ev0.elapsed_time(ev1), ws, local)
    h.engine.check_health()
    # end to end: the rank's rows from pinned host memory, one step, its
    # owned rows back, every step
    U = plan.local(rank, case.U0)
    hin = torch.from_numpy(U).pin_memory()
    hout = torch.empty((int(plan.owned[rank].sum()), 5), dtype=torch.float64).pin_memory()
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        h.engine.set_state(hin.numpy())
        h.rk3_step(h.compute_dt(case.cfl))
        hout.numpy()[:] = h.owned_state()
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(t1 - t0, ws, local)
    local_cells = len(plan.cells[rank])
    owned = int(plan.owned[rank].sum())
    halo_rows = max_over_ranks(float(len(h.lists.recv)), ws, local)
    h.close()
    if rank == 0:
        value = ncells * 3 * args.steps / (ms / 1000.0)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "mixed: f32 tables/reconstruction, f64 flux/accumulate/update",
            "data": "synthetic (seeded mesh and analytic initial condition)",
            "config": {"workload": args.case, "cells": ncells, "n": args.n, "scheme": scheme_label(case, 1),
                       "parallelism": f"partitions x{ws} (recursive coordinate bisection; cell-state halo "
                                      f"over NCCL each stage)",
                       "rank0_cells": {"owned": owned, "local": local_cells},
                       "max_halo_rows": int(halo_rows)},
            "e2e": {"value": ncells * 3 * args.steps / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": int(hin.numpy().nbytes), "d2h_bytes_per_step": int(hout.numpy().nbytes)},
            "gpu_launches": launches, "clocks": clocks,
        }
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    ws, rank, local = dist_init()
    if args.impl == "reference":
        main_reference(args, ws, rank, local)
        return
    if args.partition:
        main_partition(args, ws, rank, local)
        return
    import numpy as np
    from ucns3d_b200 import _native as N

    if args.adjoint_only:
        adj = run_adjoint(local, args.adjoint_steps, args.adjoint_every, args.adjoint_weno_n)
        if rank == 0:
            print(json.dumps({"adjoint": adj}), flush=True)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    peak, peak_kind = load_peaks()
    c32 = make_case(args, N.UCG_MIXED)
    ncells = c32.mesh.ncells
    r32 = run_gpu(args, c32, ws, local, timed_e2e=True)
    cfg32 = c32.cfg
    r64 = None
    if not args.no_fp64:
        # same mesh, tables and initial state; FP64 engine
        from ucns3d_b200.cases import Case
        cfg64 = N.UcgConfig.from_buffer_copy(cfg32)
        cfg64.precision = N.UCG_FP64
        c64 = Case(c32.name, c32.mesh, cfg64, c32.U0, c32.cfl, c32.steps, c32.meta)
        r64 = run_gpu(args, c64, ws, local, timed_e2e=False)
        del c64
    shuffle = None
    if args.shuffle:
        # the same shuffled numbering with the engine's renumbering off
        from ucns3d_b200.cases import Case
        cfg0 = N.UcgConfig.from_buffer_copy(c32.cfg)
        cfg0.reorder = 0
        r0 = run_gpu(args, Case(c32.name, c32.mesh, cfg0, c32.U0, c32.cfl, c32.steps, c32.meta), ws, local,
                     timed_e2e=False)
        ms0 = max_over_ranks(r0["ms"], ws, local)
        shuffle = {"numbering": "seeded random permutation of the cells",
                   "reorder_on": {"ms_per_step": None, "kernel_ms": r32["kern"]},
                   "reorder_off": {"value": ws * ncells * 3 * args.steps / (ms0 / 1000.0),
                                   "ms_per_step": ms0 / args.steps, "kernel_ms": r0["kern"]}}
    ms = max_over_ranks(r32["ms"], ws, local)
    value = ws * ncells * 3 * args.steps / (ms / 1000.0)
    e2e_s = max_over_ranks(r32["e2e"]["seconds"], ws, local)
    e2e_value = ws * ncells * 3 * args.steps / e2e_s
    # roofline of the dominant kernel (k_lsq), achieved from its CUDA-event
    # duration on the engine stream; the whole reconstruction beside it
    bpc = lsq_bytes_per_cell(cfg32)
    table_bytes = bpc * ncells
    lsq_ms = r32["kern"]["lsq"]
    achieved = bpc * ncells / (lsq_ms / 1000.0) / 1e9
    rbpc = recon_bytes_per_cell(cfg32)
    per_cell = LSQ_DRAM_BYTES_PER_CELL.get((args.case, int(cfg32.precision)))
    traffic = per_cell * ncells if per_cell is not None and args.wenwrt == 1 else None
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "mixed: f32 tables/reconstruction, f64 flux/accumulate/update",
        "data": "synthetic (seeded mesh and analytic initial condition)",
        "config": {"workload": args.case, "cells": ncells, "n": args.n,
                   "scheme": scheme_label(c32, args.wenwrt),
                   "parallelism": f"replicas x{ws}",
                   "l2": ("inputs larger than L2 (tables)" if table_bytes > L2_BYTES
                          else "tables smaller than L2: not an HBM-roofline case")},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "nominal_peak": NOMINAL_HBM_GBS, "frac_nominal": achieved / NOMINAL_HBM_GBS,
                     "traffic": traffic, "traffic_unit": "bytes per launch",
                     "kernel": "k_lsq (stencil least squares)",
                     "bytes_per_cell": bpc, "kernel_ms": lsq_ms,
                     "reconstruction": {"kernels": recon_kernels(cfg32, args.wenwrt), "bytes_per_cell": rbpc,
                                        "ms": r32["kern"]["recon"],
                                        "frac": rbpc * ncells / (r32["kern"]["recon"] / 1000.0) / 1e9 / peak}},
        "kernel_ms": r32["kern"],
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": r32["e2e"]["bytes_in"],
                "d2h_bytes_per_step": r32["e2e"]["bytes_out"]},
        "gpu_launches": r32["launches"],
        "clocks": r32["clocks"],
        "device_bytes": r32["device_bytes"],
        "cell_order": r32["order"],
    }
    if shuffle is not None:
        shuffle["reorder_on"]["ms_per_step"] = ms / args.steps
        out["shuffle"] = shuffle
        out["config"]["numbering"] = "shuffled (engine renumbering on)"
    if r64 is not None:
        ms64 = max_over_ranks(r64["ms"], ws, local)
        v64 = ws * ncells * 3 * args.steps / (ms64 / 1000.0)
        ra, rb = r64["state"][:, 0], r32["state"][:, 0]
        l2 = float(np.sqrt(np.mean((ra - rb) ** 2)) / np.sqrt(np.mean(ra ** 2)))
        linf = float(np.abs(ra - rb).max() / np.abs(ra).max())
        bpc64 = lsq_bytes_per_cell(cfg64)
        out["fp64"] = {"value": v64, "ms_per_step": ms64 / args.steps, "kernel_ms": r64["kern"],
                       "roofline_frac": bpc64 * ncells / (r64["kern"]["lsq"] / 1000.0) / 1e9 / peak,
                       "mixed_speedup": value / v64,
                       "density_rel_l2_mixed_vs_fp64": l2, "density_rel_linf_mixed_vs_fp64": linf,
                       "after_steps": args.warmup + args.steps}
    acc_steps = args.accuracy_steps if args.accuracy_steps is not None else (
        100 if args.case == "vortex_hex_weno5" else c32.steps)
    if acc_steps > 0:
        out["accuracy"] = run_accuracy(c32, local, acc_steps)
    if not args.no_adjoint:
        out["adjoint"] = run_adjoint(local, args.adjoint_steps, args.adjoint_every, args.adjoint_weno_n)
    if args.setup:
        out["setup"] = run_setup(local)
    if args.implicit:
        out["implicit"] = run_implicit(local)
    if rank == 0 and ws == 1 and not args.no_cpu:
        cb = cpu_sample(args, case=c32 if not args.cpu_n else None)
        out["cpu_baseline"] = {"value": cb["value"], "unit": UNIT, "cores": cb["cores"], "kind": "port",
                               "sample": cb["sample"]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
