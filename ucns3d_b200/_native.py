"""ctypes bindings of the engine (include/ucns3d_gpu.h) and of the host set-up
library (include/ucns3d_prep.h).

The shared libraries are built in-tree into ``ucns3d_b200/lib`` by
``ucns3d_b200.build``.  Loading fails loudly when a library is missing: there
is no Python or CPU fallback for the engine.
"""
from __future__ import annotations

import ctypes as C
import os

LIBDIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")

UCG_NV = 5
UCG_MAX_FACES = 6
UCG_MAX_QP = 16

UCG_OK, UCG_EINVAL, UCG_ECUDA, UCG_ENONPHYS, UCG_ESTATE, UCG_ENOMEM, UCG_ETIMEOUT = range(7)
UCG_FP64, UCG_MIXED = 0, 1
UCG_OBJ_FORCE_X, UCG_OBJ_KE = 1, 2
UCG_REDUCE_KE, UCG_REDUCE_MASS, UCG_REDUCE_ENERGY, UCG_REDUCE_ENSTROPHY = 1, 2, 3, 4

ERROR_NAMES = {
    UCG_EINVAL: "UCG_EINVAL",
    UCG_ECUDA: "UCG_ECUDA",
    UCG_ENONPHYS: "UCG_ENONPHYS",
    UCG_ESTATE: "UCG_ESTATE",
    UCG_ENOMEM: "UCG_ENOMEM",
    UCG_ETIMEOUT: "UCG_ETIMEOUT",
}

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)


class UcgConfig(C.Structure):
    _fields_ = [
        ("governing", C.c_int32), ("scheme", C.c_int32), ("iorder", C.c_int32),
        ("ees", C.c_int32), ("wenwrt", C.c_int32), ("limiter", C.c_int32),
        ("riemann", C.c_int32), ("precision", C.c_int32), ("wenoz", C.c_int32),
        ("ideg", C.c_int32), ("imax", C.c_int32), ("admis_max", C.c_int32),
        ("ideg2", C.c_int32), ("imax2", C.c_int32), ("nq_quad", C.c_int32),
        ("nq_tri", C.c_int32),
        ("gamma", C.c_double), ("prandtl", C.c_double), ("visc", C.c_double),
        ("r_gas", C.c_double), ("pres", C.c_double), ("rres", C.c_double),
        ("lwci", C.c_double), ("weno_eps", C.c_double), ("kappa_ven", C.c_double),
        ("lamx", C.c_double),
        ("quad_w", C.c_double * UCG_MAX_QP), ("tri_w", C.c_double * UCG_MAX_QP),
        ("bc_state", C.c_double * UCG_NV),
        ("boundtype", C.c_int32), ("reorder", C.c_int32),
        ("mood", C.c_int32), ("mood_mode", C.c_int32), ("mood_var", C.c_double * 4),
    ]


class UcgGeometry(C.Structure):
    _fields_ = [
        ("ncells", C.c_int64),
        ("nfaces", _i32p), ("face_type", _i32p), ("neigh", _i32p), ("neigh_face", _i32p),
        ("bc", _i32p), ("qperm", _i32p),
        ("face_angle", _f64p), ("face_area", _f64p), ("dih", _f64p), ("qpoints", _f64p),
        ("volume", _f64p), ("minedge", _f64p), ("invccjac", _f64p), ("basis_mean", _f64p),
        ("admis", _i32p), ("full", _i32p),
    ]


class UcgRecon(C.Structure):
    _fields_ = [
        ("first", C.c_int64), ("count", C.c_int64),
        ("stencil", _i32p),
        ("ntables", C.c_int64), ("table_id", _i32p),
        ("invmat", _f64p), ("invmat2", _f64p), ("indicator", _f64p), ("indicator2", _f64p),
    ]


class UcgShapes(C.Structure):
    _fields_ = [
        ("ncells", C.c_int64),
        ("shape", _i32p), ("vertices", _f64p), ("centre", _f64p), ("volume", _f64p),
        ("frame", _f64p), ("frame_origin", _f64p), ("frame_det", _f64p),
        ("period", C.c_double * 3),
    ]


class UcpScheme(C.Structure):
    _fields_ = [("scheme", C.c_int32), ("iorder", C.c_int32), ("ees", C.c_int32),
                ("nthreads", C.c_int32)]


def _load(name: str) -> C.CDLL:
    path = os.path.join(LIBDIR, name)
    if not os.path.exists(path):
        raise RuntimeError(
            f"{name} is not built (expected {path}); run `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `python -m ucns3d_b200.build`")
    return C.CDLL(path)


_prep = None
_engine = None


def prep() -> C.CDLL:
    """The host set-up library (meshes, geometry, stencils, tables)."""
    global _prep
    if _prep is None:
        lib = _load("libucns3d_prep.so")
        vp = C.c_void_p
        lib.ucp_box_hex.restype = vp
        lib.ucp_box_hex.argtypes = [C.c_int32] * 3 + [_f64p, _f64p, _i32p, _i32p]
        lib.ucp_box_tet.restype = vp
        lib.ucp_box_tet.argtypes = [C.c_int32] * 3 + [_f64p, _f64p, _i32p, _i32p, C.c_double, C.c_uint64]
        lib.ucp_bump_channel.restype = vp
        lib.ucp_bump_channel.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                         C.c_double, C.c_uint64]
        lib.ucp_mixed_box.restype = vp
        lib.ucp_mixed_box.argtypes = [C.c_int32, C.c_double, C.c_uint64]
        lib.ucp_read_grid.restype = vp
        lib.ucp_read_grid.argtypes = [C.c_char_p]
        lib.ucp_write_grid.restype = C.c_int32
        lib.ucp_write_grid.argtypes = [vp, C.c_char_p]
        lib.ucp_prepare.restype = C.c_int32
        lib.ucp_prepare.argtypes = [vp, C.POINTER(UcpScheme)]
        lib.ucp_prepare_geometry.restype = C.c_int32
        lib.ucp_prepare_geometry.argtypes = [vp, C.POINTER(UcpScheme)]
        lib.ucp_shapes.restype = C.c_int32
        lib.ucp_shapes.argtypes = [vp, C.POINTER(UcgShapes)]
        lib.ucp_ncells.restype = C.c_int64
        lib.ucp_ncells.argtypes = [vp]
        lib.ucp_ntables.restype = C.c_int64
        lib.ucp_ntables.argtypes = [vp]
        lib.ucp_fill_config.restype = C.c_int32
        lib.ucp_fill_config.argtypes = [vp, C.POINTER(UcgConfig)]
        lib.ucp_geometry.restype = C.c_int32
        lib.ucp_geometry.argtypes = [vp, C.POINTER(UcgGeometry)]
        lib.ucp_recon.restype = C.c_int32
        lib.ucp_recon.argtypes = [vp, C.POINTER(UcgRecon)]
        lib.ucp_cell_centres.restype = C.c_int32
        lib.ucp_cell_centres.argtypes = [vp, _f64p]
        lib.ucp_initial_condition.restype = C.c_int32
        lib.ucp_initial_condition.argtypes = [vp, C.c_int32, _f64p, C.c_int32, _f64p]
        lib.ucp_last_error.restype = C.c_char_p
        lib.ucp_last_error.argtypes = []
        lib.ucp_free.restype = None
        lib.ucp_free.argtypes = [vp]
        _prep = lib
    return _prep


ENGINE_SYMBOLS = [
    "ucg_create", "ucg_destroy", "ucg_upload_geometry", "ucg_upload_recon",
    "ucg_set_state", "ucg_get_state", "ucg_compute_dt", "ucg_residual", "ucg_rk3_step",
    "ucg_step", "ucg_last_dt", "ucg_reduce", "ucg_check_health", "ucg_synchronize",
    "ucg_time_kernels", "ucg_get_stream", "ucg_launch_count", "ucg_device_bytes", "ucg_last_error",
    "ucg_create_error", "ucg_force", "ucg_force_vjp", "ucg_residual_vjp", "ucg_residual_jvp", "ucg_adjoint_run",
    "ucg_tangent_run", "ucg_time_adjoint", "ucg_cell_order", "ucg_adjoint_run_obj", "ucg_tangent_run_obj",
    "ucg_set_wait_limit", "ucg_mood_state", "ucg_build_recon", "ucg_implicit_step",
    "ucg_dual_time_step", "ucg_rk3_stage", "ucg_halo_set", "ucg_halo_pack", "ucg_halo_unpack",
    "ucg_set_cell_roles", "ucg_dual_time_step_explicit", "ucg_wall_loads",
]


def engine() -> C.CDLL:
    """The CUDA engine library.  Raises when it is not built."""
    global _engine
    if _engine is None:
        lib = _load("libucns3d_gpu.so")
        vp = C.c_void_p
        lib.ucg_create.restype = C.c_int
        lib.ucg_create.argtypes = [C.POINTER(UcgConfig), C.c_int64, C.c_int, C.POINTER(vp)]
        lib.ucg_destroy.restype = None
        lib.ucg_destroy.argtypes = [vp]
        lib.ucg_upload_geometry.restype = C.c_int
        lib.ucg_upload_geometry.argtypes = [vp, C.POINTER(UcgGeometry)]
        lib.ucg_upload_recon.restype = C.c_int
        lib.ucg_upload_recon.argtypes = [vp, C.POINTER(UcgRecon)]
        lib.ucg_set_state.restype = C.c_int
        lib.ucg_set_state.argtypes = [vp, _f64p, C.c_int64]
        lib.ucg_get_state.restype = C.c_int
        lib.ucg_get_state.argtypes = [vp, _f64p, C.c_int64]
        lib.ucg_compute_dt.restype = C.c_int
        lib.ucg_compute_dt.argtypes = [vp, C.c_double, _f64p]
        lib.ucg_residual.restype = C.c_int
        lib.ucg_residual.argtypes = [vp, _f64p]
        lib.ucg_rk3_step.restype = C.c_int
        lib.ucg_rk3_step.argtypes = [vp, C.c_double]
        lib.ucg_step.restype = C.c_int
        lib.ucg_step.argtypes = [vp, C.c_double, C.c_int32]
        lib.ucg_last_dt.restype = C.c_int
        lib.ucg_last_dt.argtypes = [vp, _f64p]
        lib.ucg_reduce.restype = C.c_int
        lib.ucg_reduce.argtypes = [vp, C.c_int32, _f64p]
        lib.ucg_check_health.restype = C.c_int
        lib.ucg_check_health.argtypes = [vp]
        lib.ucg_synchronize.restype = C.c_int
        lib.ucg_synchronize.argtypes = [vp]
        lib.ucg_time_kernels.restype = C.c_int
        lib.ucg_time_kernels.argtypes = [vp, C.c_int32, _f64p]
        lib.ucg_get_stream.restype = vp
        lib.ucg_get_stream.argtypes = [vp]
        lib.ucg_launch_count.restype = C.c_int64
        lib.ucg_launch_count.argtypes = [vp]
        lib.ucg_device_bytes.restype = C.c_int64
        lib.ucg_device_bytes.argtypes = [vp]
        lib.ucg_last_error.restype = C.c_int
        lib.ucg_last_error.argtypes = [vp, C.c_char_p, C.c_int32]
        lib.ucg_create_error.restype = C.c_char_p
        lib.ucg_create_error.argtypes = []
        lib.ucg_force.restype = C.c_int
        lib.ucg_force.argtypes = [vp, _f64p]
        lib.ucg_force_vjp.restype = C.c_int
        lib.ucg_force_vjp.argtypes = [vp, _f64p]
        lib.ucg_wall_loads.restype = C.c_int
        lib.ucg_wall_loads.argtypes = [vp, _f64p, _f64p]
        lib.ucg_residual_vjp.restype = C.c_int
        lib.ucg_residual_vjp.argtypes = [vp, _f64p, _f64p, _f64p]
        lib.ucg_residual_jvp.restype = C.c_int
        lib.ucg_residual_jvp.argtypes = [vp, _f64p, _f64p, _f64p]
        lib.ucg_adjoint_run.restype = C.c_int
        lib.ucg_adjoint_run.argtypes = [vp, C.c_int32, C.c_double, C.c_int32, _f64p, _f64p, _f64p]
        lib.ucg_time_adjoint.restype = C.c_int
        lib.ucg_time_adjoint.argtypes = [vp, C.c_int32, _f64p]
        lib.ucg_adjoint_run_obj.restype = C.c_int
        lib.ucg_adjoint_run_obj.argtypes = [vp, C.c_int32, C.c_int32, C.c_double, C.c_int32, _f64p, _f64p, _f64p]
        lib.ucg_tangent_run_obj.restype = C.c_int
        lib.ucg_tangent_run_obj.argtypes = [vp, C.c_int32, C.c_int32, C.c_double, _f64p, _f64p, _f64p, _f64p]
        lib.ucg_set_wait_limit.restype = C.c_int
        lib.ucg_set_wait_limit.argtypes = [vp, C.c_int64]
        lib.ucg_cell_order.restype = C.c_int
        lib.ucg_cell_order.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _f64p]
        lib.ucg_mood_state.restype = C.c_int
        lib.ucg_mood_state.argtypes = [vp, _i32p, _i32p]
        lib.ucg_implicit_step.restype = C.c_int
        lib.ucg_implicit_step.argtypes = [vp, C.c_double, C.c_int32, C.c_int32]
        lib.ucg_dual_time_step.restype = C.c_int
        lib.ucg_dual_time_step.argtypes = [vp, C.c_double, C.c_double, C.c_int32, C.c_double, C.c_int32,
                                           C.POINTER(C.c_int32)]
        lib.ucg_build_recon.restype = C.c_int
        lib.ucg_build_recon.argtypes = [vp, C.POINTER(UcgShapes), C.POINTER(UcgRecon)]
        lib.ucg_dual_time_step_explicit.restype = C.c_int
        lib.ucg_dual_time_step_explicit.argtypes = [vp, C.c_double, C.c_double, C.c_int32, C.c_double,
                                                    C.POINTER(C.c_int32)]
        lib.ucg_set_cell_roles.restype = C.c_int
        lib.ucg_set_cell_roles.argtypes = [vp, C.POINTER(C.c_int8)]
        lib.ucg_rk3_stage.restype = C.c_int
        lib.ucg_rk3_stage.argtypes = [vp, C.c_int32, C.c_double]
        lib.ucg_halo_set.restype = C.c_int
        lib.ucg_halo_set.argtypes = [vp, _i32p, C.c_int64, _i32p, C.c_int64]
        # device buffers, passed as addresses
        lib.ucg_halo_pack.restype = C.c_int
        lib.ucg_halo_pack.argtypes = [vp, C.c_int32, vp]
        lib.ucg_halo_unpack.restype = C.c_int
        lib.ucg_halo_unpack.argtypes = [vp, C.c_int32, vp]
        lib.ucg_tangent_run.restype = C.c_int
        lib.ucg_tangent_run.argtypes = [vp, C.c_int32, C.c_double, _f64p, _f64p, _f64p, _f64p]
        _engine = lib
    return _engine


def ptr(a, ctype):
    """Pointer to the data of a contiguous numpy array (None for None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))
