"""Host set-up library: meshes, connectivity, geometry and reconstruction
tables (CPU only)."""
import numpy as np
import pytest

from ucns3d_b200.mesh import SCHEME_MUSCL, SCHEME_WENO, Mesh

L = 2 * np.pi


def _normals(g):
    a = g["face_angle"]
    return np.stack([np.cos(a[..., 0]) * np.sin(a[..., 1]), np.sin(a[..., 0]) * np.sin(a[..., 1]),
                     np.cos(a[..., 1])], -1)


MESHES = {
    "hex": lambda: Mesh.box_hex(6, 5, 4),
    "tet": lambda: Mesh.box_tet(4, 4, 3, jitter=0.15, seed=7),
    "bump": lambda: Mesh.bump_channel(12, 6, 2, seed=3),
    "mixed": lambda: Mesh.mixed_box(8, seed=5),
}


@pytest.mark.parametrize("kind", list(MESHES))
def test_connectivity_and_closure(kind):
    m = MESHES[kind]().prepare(SCHEME_MUSCL, 1)
    g = m.geometry()
    n = g["ncells"]
    assert n == m.ncells > 0
    assert (g["volume"] > 0).all()
    # neighbour relation is symmetric and normals/areas match across faces
    nrm = _normals(g)
    for c in range(n):
        for f in range(g["nfaces"][c]):
            nb, nf = g["neigh"][c, f], g["neigh_face"][c, f]
            if nb < 0:
                assert g["bc"][c, f] in (1, 2, 3, 4)
                continue
            assert g["neigh"][nb, nf] == c and g["neigh_face"][nb, nf] == f
            assert abs(g["face_area"][c, f] - g["face_area"][nb, nf]) < 1e-12 * g["face_area"][c, f]
            np.testing.assert_allclose(nrm[c, f], -nrm[nb, nf], atol=1e-12)
    # closed cells: sum of n A over the faces vanishes
    mask = np.arange(6)[None, :] < g["nfaces"][:, None]
    s = (nrm * (g["face_area"] * mask)[..., None]).sum(1)
    assert np.abs(s).max() < 1e-13 * g["face_area"].max()


def test_box_volume_and_periodic_pairing():
    m = Mesh.box_tet(3, 3, 3, jitter=0.15, seed=11).prepare(SCHEME_WENO, 2)
    g = m.geometry()
    assert abs(g["volume"].sum() - L ** 3) < 1e-10 * L ** 3
    assert (g["neigh"][:, :4] >= 0).all()  # periodic box: no boundary faces
    # quadrature point pairing is an involution
    for c in range(g["ncells"]):
        for f in range(4):
            nb, nf = g["neigh"][c, f], g["neigh_face"][c, f]
            for q in range(3):
                qq = g["qperm"][c, f, q]
                assert g["qperm"][nb, nf, qq] == q


def test_mixed_box_has_all_shapes():
    m = Mesh.mixed_box(8, seed=5).prepare(SCHEME_MUSCL, 1)
    g = m.geometry()
    nf = np.bincount(g["nfaces"])
    assert nf[4] > 0 and nf[5] > 0 and nf[6] > 0  # tets; pyramids+prisms; hexahedra
    assert abs(g["volume"].sum() - L ** 3) < 1e-9 * L ** 3


@pytest.mark.parametrize("kind,scheme,iorder,ees", [
    ("hex", SCHEME_MUSCL, 1, 0), ("tet", SCHEME_WENO, 2, 0), ("hex12", SCHEME_WENO, 4, 0), ("tet", SCHEME_WENO, 3, 5)])
def test_lsq_reproduces_linear_fields(kind, scheme, iorder, ees):
    """invmat_stencilt recovers the exact coefficients of a linear field from
    cell averages (LSQ exactness, prestore.f90:434-523)."""
    mk = {"hex": lambda: Mesh.box_hex(8, 8, 8), "tet": lambda: Mesh.box_tet(4, 4, 4, seed=3),
          "hex12": lambda: Mesh.box_hex(12, 12, 12)}[kind]
    m = mk().prepare(scheme, iorder, ees)
    g, r, c = m.geometry(), m.recon(), m.centres()
    worst = 0.0
    for i in range(g["ncells"]):
        J = np.linalg.inv(g["invccjac"][i])
        t = r["table_id"][i]
        for ll in range(g["admis"][i]):
            low = ees == 5 and ll > 0
            M = r["invmat2"][t, ll] if low else r["invmat"][t, ll]
            nk = M.shape[0]
            st = r["stencil"][i, ll, 1:nk + 1]
            d = c[st] - c[i]
            d -= L * np.round(d / L)
            for comp in range(3):
                gg = M.T @ d[:, comp]
                worst = max(worst, np.abs(gg[:3] - J[comp]).max(), np.abs(gg[3:]).max() if gg.size > 3 else 0.0)
    assert worst < 1e-8


def test_weno_stencils_admissible_and_shared_tables():
    m = Mesh.box_hex(12, 12, 12).prepare(SCHEME_WENO, 4)
    g, r = m.geometry(), m.recon()
    assert (g["admis"] == 7).all() and (g["full"] == 1).all()
    assert r["ntables"] == 1  # translation-invariant stencils share one matrix set
    st = r["stencil"]
    assert (st[:, :, 0] == np.arange(g["ncells"])[:, None]).all()
    assert (st >= 0).all()
    # indicator matrices are symmetric positive semi-definite
    S = r["indicator"][0]
    np.testing.assert_allclose(S, S.T, rtol=1e-12, atol=1e-12 * np.abs(S).max())
    assert np.linalg.eigvalsh(S).min() > -1e-10 * np.abs(S).max()


def test_initial_condition_averages():
    m = Mesh.box_hex(16, 16, 16).prepare(SCHEME_MUSCL, 1)
    U = m.initial_condition(95, [1.4, 100.0, 1.0])
    g = m.geometry()
    assert abs((U[:, 0] * g["volume"]).sum() - L ** 3) < 1e-9
    # TGV momentum integrates to zero
    assert np.abs((U[:, 1:4] * g["volume"][:, None]).sum(0)).max() < 1e-9


def test_renumbered_mesh_oracle_residual_is_permuted():
    """The oracle evaluates every cell from its own faces, so a renumbered
    copy of a mesh gives the same residual rows, moved, bit for bit."""
    import sys
    import os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    from oracle import Oracle
    from ucns3d_b200.config import EULER, make_config
    from ucns3d_b200.mesh import IC_TGV, SCHEME_WENO, Mesh, RenumberedMesh
    m = Mesh.box_tet(4, 4, 4, seed=3).prepare(SCHEME_WENO, 2)
    cfg = make_config(m, governing=EULER)
    U = m.initial_condition(IC_TGV, [1.4, 5.0, 1.0])
    order = np.random.default_rng(5).permutation(m.ncells)
    ms = RenumberedMesh(m, order)
    assert np.array_equal(ms.geometry()["volume"], m.geometry()["volume"][order])
    Rb = Oracle(m, cfg).residual(U)
    Rs = Oracle(ms, cfg).residual(U[order])
    assert np.array_equal(ms.to_base(Rs), Rb)


@pytest.mark.parametrize("kind", ["bump", "tet_box"])
def test_grid_files_round_trip(kind, tmp_path):
    """UCNS3D's GRID.vrt/cel/bnd: a mesh written and read back prepares to
    the same geometry, boundary codes and reconstruction tables, bit for bit
    (coordinates are written with 17 significant digits)."""
    if kind == "bump":
        m = Mesh.bump_channel(16, 8, 4, seed=3).prepare(SCHEME_WENO, 2)
    else:
        m = Mesh.box_tet(4, 4, 4, periodic=(0, 0, 0), bc=(1, 2, 3, 3, 4, 6), seed=7).prepare(SCHEME_WENO, 2)
    prefix = str(tmp_path) + "/"
    m.write_grid(prefix)
    r = Mesh.read_grid(prefix).prepare(SCHEME_WENO, 2)
    ga, gb = m.geometry(), r.geometry()
    for k in ("nfaces", "face_type", "neigh", "neigh_face", "bc", "qperm", "face_angle", "face_area", "dih",
              "qpoints", "volume", "minedge", "invccjac", "basis_mean", "admis", "full"):
        assert np.array_equal(ga[k], gb[k]), k
    ra, rb = m.recon(), r.recon()
    assert np.array_equal(ra["stencil"], rb["stencil"])
    ia = ra["invmat"][ra["table_id"]] if ra["table_id"] is not None else ra["invmat"]
    ib = rb["invmat"][rb["table_id"]] if rb["table_id"] is not None else rb["invmat"]
    assert np.array_equal(ia, ib)
    lines = open(prefix + "GRID.bnd").read().split("\n")
    assert len([x for x in lines if x]) == int(((ga["neigh"] < 0) & (np.arange(6)[None, :] < ga["nfaces"][:, None])).sum())


@pytest.mark.parametrize("kind", ["hex", "tet", "mixed", "hex_xz"])
def test_periodic_grid_files_round_trip(kind, tmp_path):
    """Periodic meshes in GRID files: the writer gives each node that a cell
    sees across a periodic side its own image node and writes the faces on
    the periodic sides with code 5; the reader pairs them as APPLY_BOUNDARY
    does (same shape, centroids on opposite sides of the bounding box with
    the same other two coordinates, period = the box's extent) and prepares
    to the same geometry, stencils, tables and oracle residual, bit for bit."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    from oracle import Oracle
    from ucns3d_b200.config import EULER, make_config
    from ucns3d_b200.mesh import IC_TGV
    m = {"hex": lambda: Mesh.box_hex(6, 5, 4),
         "tet": lambda: Mesh.box_tet(4, 4, 4, jitter=0.0, seed=3),
         "mixed": lambda: Mesh.mixed_box(6),
         "hex_xz": lambda: Mesh.box_hex(6, 5, 4, periodic=(1, 0, 1), bc=(0, 0, 4, 4, 0, 0))}[kind]()
    m = m.prepare(SCHEME_WENO, 2)
    prefix = str(tmp_path) + "/"
    m.write_grid(prefix)
    codes = np.loadtxt(prefix + "GRID.bnd", dtype=np.int64, ndmin=2)[:, 5]
    assert (codes == 5).sum() > 0
    r = Mesh.read_grid(prefix).prepare(SCHEME_WENO, 2)
    ga, gb = m.geometry(), r.geometry()
    for k in ("nfaces", "face_type", "neigh", "neigh_face", "bc", "qperm", "face_angle", "face_area", "dih",
              "qpoints", "volume", "minedge", "invccjac", "basis_mean", "admis", "full"):
        assert np.array_equal(ga[k], gb[k]), k
    ra, rb = m.recon(), r.recon()
    assert np.array_equal(ra["stencil"], rb["stencil"])
    ia = ra["invmat"][ra["table_id"]] if ra["table_id"] is not None else ra["invmat"]
    ib = rb["invmat"][rb["table_id"]] if rb["table_id"] is not None else rb["invmat"]
    assert np.array_equal(ia, ib)
    cfg = make_config(m, governing=EULER)
    U = m.initial_condition(IC_TGV, [1.4, 5.0, 1.0])
    assert np.array_equal(Oracle(r, cfg).residual(U), Oracle(m, cfg).residual(U))


def test_periodic_grid_errors(tmp_path):
    """Periodic sides the GRID format cannot pair are refused: a jittered
    periodic box (faces off the box's sides) is not written, and a code 5
    face without a partner on the opposite side is not read."""
    m = Mesh.box_tet(4, 4, 4, jitter=0.15, seed=3).prepare(SCHEME_WENO, 2)
    with pytest.raises(RuntimeError, match="off the sides"):
        m.write_grid(str(tmp_path) + "/j_")
    m = Mesh.box_hex(4, 4, 4).prepare(SCHEME_MUSCL, 1)
    prefix = str(tmp_path) + "/h_"
    m.write_grid(prefix)
    lines = open(prefix + "GRID.bnd").read().split("\n")
    with open(prefix + "GRID.bnd", "w") as f:
        f.write("\n".join(lines[1:]))  # one face of a periodic pair dropped
    with pytest.raises(RuntimeError, match="periodic"):
        Mesh.read_grid(prefix)


def test_grid_reader_shapes_and_errors(tmp_path):
    """The 8-node encoding of the four cell shapes, told apart by repeated
    nodes as FIND_SHAPE does: a pyramid on a hexahedron's top with a
    tetrahedron and a prism beside it is read with the right face counts;
    a boundary face missing from GRID.bnd, and periodic codes, are refused."""
    d = str(tmp_path) + "/"
    # unit cube 1-8, apex 9 above it, 10 beside, 11-12 for a prism
    pts = {1: (0, 0, 0), 2: (1, 0, 0), 3: (1, 1, 0), 4: (0, 1, 0), 5: (0, 0, 1), 6: (1, 0, 1), 7: (1, 1, 1),
           8: (0, 1, 1), 9: (0.5, 0.5, 1.6), 10: (0.5, -0.8, 0.5)}
    with open(d + "GRID.vrt", "w") as f:
        for k, p in pts.items():
            f.write(f"{k} {p[0]} {p[1]} {p[2]}\n")
    with open(d + "GRID.cel", "w") as f:
        f.write("1 1 2 3 4 5 6 7 8\n")        # hexahedron
        f.write("2 5 6 7 8 9 9 9 9\n")        # pyramid on its top
        f.write("3 1 2 6 6 10 10 10 10\n")    # tetrahedron on the face 1-2-6
    # a boundary file that misses most boundary faces: read, refused at prepare
    with open(d + "GRID.bnd", "w") as f:
        f.write("1 1 4 3 2 4\n")
    m = Mesh.read_grid(d)
    assert m.ncells == 3
    with pytest.raises(RuntimeError, match="GRID.bnd"):
        m.prepare(SCHEME_MUSCL, 1)
    with open(d + "GRID.bnd", "w") as f:
        f.write("1 1 4 3 2 5\n")
    with pytest.raises(RuntimeError, match="periodic"):
        Mesh.read_grid(d)
    with open(d + "GRID.bnd", "w") as f:
        f.write("1 1 4 3 2 4\n")
    with open(d + "GRID.cel", "a") as f:
        f.write("4 1 2 3 4 5 5 6 6\n")        # no shape of FIND_SHAPE
    with pytest.raises(RuntimeError, match="none of"):
        Mesh.read_grid(d)
