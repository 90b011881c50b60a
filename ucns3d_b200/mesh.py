"""Synthetic meshes and their set-up tables (wrapper of libucns3d_prep).

UCNS3D builds these tables in its Fortran set-up (src/main.f90:151-767); a
driver that keeps that set-up passes its own tables to the engine.  This
module is the standalone path: seeded synthetic meshes for the benchmark and
the tests, with geometry, stencils, pseudo-inverses and smoothness matrices
computed in FP64 on the host.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

SCHEME_MUSCL = 2
SCHEME_WENO = 3

IC_TGV = 95
IC_VORTEX = 201
IC_UNIFORM = 1


def _check(rc: int, what: str):
    if rc != 0:
        msg = N.prep().ucp_last_error().decode()
        raise RuntimeError(f"{what} failed ({N.ERROR_NAMES.get(rc, rc)}): {msg}")


class Mesh:
    """A mesh owned by the set-up library.  Build with one of the class
    methods, then ``prepare`` it for a scheme."""

    def __init__(self, handle, kind: str, params: dict):
        if not handle:
            raise RuntimeError("mesh construction failed: " + N.prep().ucp_last_error().decode())
        self._h = C.c_void_p(handle)
        self.kind = kind
        self.params = params
        self.prepared = False

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                N.prep().ucp_free(h)
            except TypeError:  # interpreter shutdown: the module is already torn down
                pass
            self._h = None

    # -------------------------------------------------------- constructors
    @classmethod
    def box_hex(cls, nx, ny, nz, L=(2 * np.pi,) * 3, origin=(0.0, 0.0, 0.0), periodic=(1, 1, 1),
                bc=(0, 0, 0, 0, 0, 0)):
        Ls = (C.c_double * 3)(*L)
        o = (C.c_double * 3)(*origin)
        p = (C.c_int32 * 3)(*periodic)
        b = (C.c_int32 * 6)(*bc)
        h = N.prep().ucp_box_hex(nx, ny, nz, Ls, o, p, b)
        return cls(h, "box_hex", dict(n=(nx, ny, nz), L=tuple(L), periodic=tuple(periodic)))

    @classmethod
    def box_tet(cls, nx, ny, nz, L=(2 * np.pi,) * 3, origin=(0.0, 0.0, 0.0), periodic=(1, 1, 1),
                bc=(0, 0, 0, 0, 0, 0), jitter=0.15, seed=1234):
        Ls = (C.c_double * 3)(*L)
        o = (C.c_double * 3)(*origin)
        p = (C.c_int32 * 3)(*periodic)
        b = (C.c_int32 * 6)(*bc)
        h = N.prep().ucp_box_tet(nx, ny, nz, Ls, o, p, b, float(jitter), int(seed))
        return cls(h, "box_tet", dict(n=(nx, ny, nz), L=tuple(L), periodic=tuple(periodic),
                                      jitter=jitter, seed=seed))

    @classmethod
    def bump_channel(cls, nx=240, ny=80, nlayers=4, bump=0.1, dz=None, split_frac=0.5, seed=1234):
        dz = (1.0 / ny) if dz is None else dz
        h = N.prep().ucp_bump_channel(nx, ny, nlayers, bump, dz, split_frac, int(seed))
        return cls(h, "bump_channel", dict(nx=nx, ny=ny, nlayers=nlayers, bump=bump, seed=seed))

    @classmethod
    def read_grid(cls, prefix: str):
        """A mesh from UCNS3D's ASCII grid files <prefix>GRID.vrt, GRID.cel
        and GRID.bnd (non-periodic)."""
        h = N.prep().ucp_read_grid(prefix.encode())
        return cls(h, "grid", dict(prefix=prefix))

    def write_grid(self, prefix: str):
        """Write this prepared, non-periodic mesh as <prefix>GRID.vrt,
        GRID.cel and GRID.bnd."""
        _check(N.prep().ucp_write_grid(self._h, prefix.encode()), "ucp_write_grid")

    @classmethod
    def mixed_box(cls, n, L=2 * np.pi, seed=1234):
        h = N.prep().ucp_mixed_box(n, L, int(seed))
        return cls(h, "mixed_box", dict(n=n, L=L, seed=seed))

    # ------------------------------------------------------------- set-up
    @property
    def ncells(self) -> int:
        return int(N.prep().ucp_ncells(self._h))

    def prepare(self, scheme: int, iorder: int, ees: int = 0, nthreads: int = 0, tables: bool = True) -> "Mesh":
        """Connectivity, geometry, stencils and (``tables``) the
        reconstruction tables; without them the engine builds the tables on
        the device (``Engine(..., tables="device")``)."""
        s = N.UcpScheme(scheme, iorder, ees, nthreads)
        if tables:
            _check(N.prep().ucp_prepare(self._h, C.byref(s)), "ucp_prepare")
        else:
            _check(N.prep().ucp_prepare_geometry(self._h, C.byref(s)), "ucp_prepare_geometry")
        self.prepared = True
        self.tables = tables
        self.scheme, self.iorder, self.ees = scheme, iorder, ees
        cfg = N.UcgConfig()
        _check(N.prep().ucp_fill_config(self._h, C.byref(cfg)), "ucp_fill_config")
        self.sizes = dict(ideg=cfg.ideg, imax=cfg.imax, admis_max=cfg.admis_max, ideg2=cfg.ideg2,
                          imax2=cfg.imax2, nq_quad=cfg.nq_quad, nq_tri=cfg.nq_tri,
                          quad_w=list(cfg.quad_w), tri_w=list(cfg.tri_w))
        return self

    def fill_config(self, cfg: N.UcgConfig) -> N.UcgConfig:
        _check(N.prep().ucp_fill_config(self._h, C.byref(cfg)), "ucp_fill_config")
        return cfg

    def geometry_struct(self) -> N.UcgGeometry:
        g = N.UcgGeometry()
        _check(N.prep().ucp_geometry(self._h, C.byref(g)), "ucp_geometry")
        return g

    def recon_struct(self) -> N.UcgRecon:
        r = N.UcgRecon()
        _check(N.prep().ucp_recon(self._h, C.byref(r)), "ucp_recon")
        return r

    def shapes_struct(self) -> N.UcgShapes:
        """Cell shapes, frames and periods for ucg_build_recon."""
        s = N.UcgShapes()
        _check(N.prep().ucp_shapes(self._h, C.byref(s)), "ucp_shapes")
        return s

    @property
    def ntables(self) -> int:
        return int(N.prep().ucp_ntables(self._h))

    # ------------------------------------------------ numpy views (copies)
    def geometry(self) -> dict:
        """Copies of the geometry arrays as numpy arrays (for tests)."""
        g = self.geometry_struct()
        n = g.ncells
        F, Q = N.UCG_MAX_FACES, N.UCG_MAX_QP
        ideg = self.sizes["ideg"]

        def arr(p, shape, dt):
            if not p:
                return None
            count = int(np.prod(shape))
            ct = C.c_int32 if dt == np.int32 else C.c_double
            buf = (ct * count).from_address(C.cast(p, C.c_void_p).value)
            return np.frombuffer(buf, dtype=dt).reshape(shape).copy()

        return dict(
            ncells=n,
            nfaces=arr(g.nfaces, (n,), np.int32), face_type=arr(g.face_type, (n, F), np.int32),
            neigh=arr(g.neigh, (n, F), np.int32), neigh_face=arr(g.neigh_face, (n, F), np.int32),
            bc=arr(g.bc, (n, F), np.int32), qperm=arr(g.qperm, (n, F, Q), np.int32),
            face_angle=arr(g.face_angle, (n, F, 2), np.float64), face_area=arr(g.face_area, (n, F), np.float64),
            dih=arr(g.dih, (n, F), np.float64), qpoints=arr(g.qpoints, (n, F, Q, 3), np.float64),
            volume=arr(g.volume, (n,), np.float64), minedge=arr(g.minedge, (n,), np.float64),
            invccjac=arr(g.invccjac, (n, 3, 3), np.float64), basis_mean=arr(g.basis_mean, (n, ideg), np.float64),
            admis=arr(g.admis, (n,), np.int32), full=arr(g.full, (n,), np.int32),
        )

    def shapes(self) -> dict:
        """Copies of the cell shapes of ucp_shapes (for tests and
        renumbered views)."""
        sh = self.shapes_struct()
        n = sh.ncells

        def arr(p, shape, dt):
            count = int(np.prod(shape))
            ct = C.c_int32 if dt == np.int32 else C.c_double
            buf = (ct * count).from_address(C.cast(p, C.c_void_p).value)
            return np.frombuffer(buf, dtype=dt).reshape(shape).copy()

        return dict(shape=arr(sh.shape, (n,), np.int32), vertices=arr(sh.vertices, (n, 8, 3), np.float64),
                    centre=arr(sh.centre, (n, 3), np.float64), volume=arr(sh.volume, (n,), np.float64),
                    frame=arr(sh.frame, (n, 3, 3), np.float64), frame_origin=arr(sh.frame_origin, (n, 3), np.float64),
                    frame_det=arr(sh.frame_det, (n,), np.float64), period=list(sh.period))

    def recon(self) -> dict:
        """Copies of the reconstruction tables (for tests)."""
        r = self.recon_struct()
        s = self.sizes
        n, nt = r.count, r.ntables
        A, W, D = s["admis_max"], s["imax"] + 1, s["ideg"]

        def arr(p, shape, dt):
            if not p:
                return None
            count = int(np.prod(shape))
            ct = C.c_int32 if dt == np.int32 else C.c_double
            buf = (ct * count).from_address(C.cast(p, C.c_void_p).value)
            return np.frombuffer(buf, dtype=dt).reshape(shape).copy()

        out = dict(stencil=arr(r.stencil, (n, A, W), np.int32), table_id=arr(r.table_id, (n,), np.int32),
                   ntables=nt, invmat=arr(r.invmat, (nt, A, s["imax"], D), np.float64),
                   indicator=arr(r.indicator, (nt, D, D), np.float64))
        if s["ideg2"]:
            out["invmat2"] = arr(r.invmat2, (nt, A, s["imax2"], s["ideg2"]), np.float64)
            out["indicator2"] = arr(r.indicator2, (nt, s["ideg2"], s["ideg2"]), np.float64)
        return out

    def centres(self) -> np.ndarray:
        out = np.zeros((self.ncells, 3))
        _check(N.prep().ucp_cell_centres(self._h, N.ptr(out, C.c_double)), "ucp_cell_centres")
        return out

    def initial_condition(self, kind: int, params) -> np.ndarray:
        """Cell averages of the conserved variables, shape (n, 5)."""
        p = np.ascontiguousarray(params, dtype=np.float64)
        out = np.zeros((self.ncells, 5))
        _check(N.prep().ucp_initial_condition(self._h, kind, N.ptr(p, C.c_double), len(p),
                                              N.ptr(out, C.c_double)), "ucp_initial_condition")
        return out


class RenumberedMesh:
    """A prepared mesh seen through another cell numbering: caller cell i is
    the base mesh's cell ``order[i]``.  Neighbour and stencil indices are
    renumbered, per-cell rows moved; the shared matrix sets (``table_id``)
    are kept.  It stands in for a mesh that arrives in partitioner or file
    order, as UCNS3D's cells do after METIS and the grid reader
    (src/main.f90:103-137), and offers the interface the engine, the oracle
    and the benchmarks use."""

    def __init__(self, base: Mesh, order: np.ndarray):
        if not getattr(base, "prepared", False):
            raise ValueError("mesh must be prepared first")
        n = base.ncells
        order = np.asarray(order, dtype=np.int64)
        if order.shape != (n,) or not np.array_equal(np.sort(order), np.arange(n)):
            raise ValueError("order must be a permutation of the cells")
        self.base, self.order = base, order
        self.inverse = np.empty(n, dtype=np.int64)
        self.inverse[order] = np.arange(n)
        self.prepared = True
        self.sizes = base.sizes
        self.scheme, self.iorder, self.ees = base.scheme, base.iorder, base.ees
        remap = lambda a: np.where(a >= 0, self.inverse[np.maximum(a, 0)], -1).astype(np.int32)  # noqa: E731
        g = base.geometry()
        self._g = {k: (np.ascontiguousarray(v[order]) if isinstance(v, np.ndarray) else v) for k, v in g.items()}
        self._g["neigh"] = remap(self._g["neigh"])
        self._s = {k: (np.ascontiguousarray(v[order]) if isinstance(v, np.ndarray) else v)
                   for k, v in base.shapes().items()}
        r = base.recon()
        self._r = dict(r)
        self._r["stencil"] = np.ascontiguousarray(remap(r["stencil"][order]))
        if r["table_id"] is not None:
            self._r["table_id"] = np.ascontiguousarray(r["table_id"][order])
        else:  # per-cell matrix sets: move them with their cells
            for k in ("invmat", "invmat2", "indicator", "indicator2"):
                if r.get(k) is not None:
                    self._r[k] = np.ascontiguousarray(r[k][order])

    @property
    def ncells(self) -> int:
        return len(self.order)

    @property
    def ntables(self) -> int:
        return self._r["ntables"]

    def fill_config(self, cfg: N.UcgConfig) -> N.UcgConfig:
        return self.base.fill_config(cfg)

    def geometry_struct(self) -> N.UcgGeometry:
        g, s = self._g, N.UcgGeometry()
        s.ncells = self.ncells
        for k in ("nfaces", "face_type", "neigh", "neigh_face", "bc", "qperm", "admis", "full"):
            setattr(s, k, N.ptr(g[k], C.c_int32))
        for k in ("face_angle", "face_area", "dih", "qpoints", "volume", "minedge", "invccjac", "basis_mean"):
            if g[k] is not None:  # basis_mean: absent when the engine builds the tables
                setattr(s, k, N.ptr(g[k], C.c_double))
        return s

    def recon_struct(self) -> N.UcgRecon:
        r, s = self._r, N.UcgRecon()
        s.first, s.count = 0, self.ncells
        s.stencil = N.ptr(r["stencil"], C.c_int32)
        s.ntables = r["ntables"]
        if r["table_id"] is not None:
            s.table_id = N.ptr(r["table_id"], C.c_int32)
        for k in ("invmat", "invmat2", "indicator", "indicator2"):
            if r.get(k) is not None:
                setattr(s, k, N.ptr(r[k], C.c_double))
        return s

    def shapes_struct(self) -> N.UcgShapes:
        sh, s = self._s, N.UcgShapes()
        s.ncells = self.ncells
        s.shape = N.ptr(sh["shape"], C.c_int32)
        for k in ("vertices", "centre", "volume", "frame", "frame_origin", "frame_det"):
            setattr(s, k, N.ptr(sh[k], C.c_double))
        for k in range(3):
            s.period[k] = sh["period"][k]
        return s

    def geometry(self) -> dict:
        return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self._g.items()}

    def recon(self) -> dict:
        return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self._r.items()}

    def centres(self) -> np.ndarray:
        return self.base.centres()[self.order]

    def initial_condition(self, kind: int, params) -> np.ndarray:
        return self.base.initial_condition(kind, params)[self.order]

    def to_base(self, a: np.ndarray) -> np.ndarray:
        """Per-cell rows of this numbering in the base mesh's numbering."""
        out = np.empty_like(a)
        out[self.order] = a
        return out
