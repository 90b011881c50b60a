// Host-side set-up: synthetic meshes, connectivity, geometry, stencils and
// the FP64 reconstruction tables consumed by the engine (ucns3d_gpu.h).
//
// The formulas follow UCNS3D's set-up; the search/sort machinery is this
// library's own.  Reference routines restated here:
//   element tet decomposition       DECOMPOSE3         src/grid_t.f90:1027-1074
//   cell volume (sum of tets)        GEOMETRY_CALC      src/grid_t.f90:1192-1365
//   MINEDGE = 3 V / sum(S)                              src/grid_t.f90:1122
//   face normal as two angles        FIND_ROT_ANGLES    src/grid_t.f90:274
//   face quadrature                  QUADRATUREQUAD3D / QUADRATURETRIANG
//                                                       src/grid_t.f90:2834, 2054
//   centre distance DIH              direct_side        src/local_pt.f90:1990-2091
//   reference frame (first tet)      LOCALISE_STEN2     src/local_pt.f90:1040-1133
//   basis = monomials minus mean     BASIS_REC          src/basis.f90:11-1744
//   stencil matrix of integrals      COMPBASEL          src/prestore.f90:3657
//   pseudo-inverse via QR of A^T A   PRESTORE_RECONSTRUCTION3 src/prestore.f90:434-528
//   smoothness matrices              INDICATORMATRIX/WENOTET/PH1-4 src/prestore.f90:1529-2100
//   stencil sizes                    DETERMINE_SIZE     src/grid_p.f90:6097-6288
//   admissible stencils, FULL        STENCILS           src/grid_p.f90:6452-6554
//   initial condition averages       INITIALISE         src/init_p.f90:14, profile.f90:253
#include "ucns3d_prep.h"
#include "../common/rules.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <random>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;
void set_err(const std::string& s) { g_err = s; }
// a message set by an OpenMP worker (inside a critical section) goes to the
// calling thread's error when the parallel loop's result comes back
std::string g_err_par;
void set_err_par(const std::string& s) { g_err_par = s; }
bool par_result(bool ok) {
  if (!ok) set_err(g_err_par);
  return ok;
}

struct V3 {
  double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }

// topology, volume quadrature, monomial order: ../common/rules.h
using ucrules::Topo;
using ucrules::topo;
using ucrules::gauss_legendre;
using ucrules::TetRule;
using ucrules::tet_rule;

// Face rules.  Quadrilaterals: tensor Gauss-Legendre with n = IGQRULES per
// direction, weights w_i w_j / 4 (QUADRATUREQUAD3D).  Triangles: the
// symmetric rules of QUADRATURETRIANG (1, 3, 6, 10 points; published
// Dunavant-type tables, weights summing to 1).
struct FaceRule {
  int nq = 0;
  std::vector<std::array<double, 3>> p;  // (r,s,-) for quads, barycentric for triangles
  std::vector<double> w;
};
FaceRule quad_rule(int ig) {
  std::vector<double> gx, gw;
  gauss_legendre(ig, gx, gw);
  FaceRule r;
  for (int a = 0; a < ig; ++a)
    for (int b = 0; b < ig; ++b) {
      r.p.push_back({gx[a], gx[b], 0.0});
      r.w.push_back(0.25 * gw[a] * gw[b]);
    }
  r.nq = ig * ig;
  return r;
}
FaceRule tri_rule(int ig) {
  FaceRule r;
  auto add3 = [&](double a, double b, double w) {
    r.p.push_back({a, b, b});
    r.w.push_back(w);
    r.p.push_back({b, a, b});
    r.w.push_back(w);
    r.p.push_back({b, b, a});
    r.w.push_back(w);
  };
  auto add6 = [&](double a, double b, double c, double w) {
    const double v[6][3] = {{a, b, c}, {a, c, b}, {c, a, b}, {b, a, c}, {b, c, a}, {c, b, a}};
    for (auto& q : v) {
      r.p.push_back({q[0], q[1], q[2]});
      r.w.push_back(w);
    }
  };
  if (ig <= 1) {
    r.p.push_back({1.0 / 3, 1.0 / 3, 1.0 / 3});
    r.w.push_back(1.0);
  } else if (ig == 2) {
    add3(2.0 / 3.0, 1.0 / 6.0, 1.0 / 3.0);
  } else if (ig == 3) {
    add3(0.816847572980459, 0.091576213509771, 0.109951743655322);
    add3(0.108103018168070, 0.445948490915965, 0.223381589678011);
  } else {
    add3(0.888871894660413, 0.055564052669793, 0.041955512996649);
    add6(0.295533711735893, 0.634210747745723, 0.070255540518384, 0.112098412070887);
    r.p.push_back({1.0 / 3, 1.0 / 3, 1.0 / 3});
    r.w.push_back(0.201542988584730);
  }
  double s = 0.0;
  for (double w : r.w) s += w;
  for (auto& w : r.w) w /= s;
  r.nq = (int)r.w.size();
  return r;
}

using ucrules::Mono;
using ucrules::monomials;

inline double ipow(double x, int e) {
  double r = 1.0;
  for (int i = 0; i < e; ++i) r *= x;
  return r;
}
inline double mono_eval(const Mono& m, const double* p) { return ipow(p[0], m.e[0]) * ipow(p[1], m.e[1]) * ipow(p[2], m.e[2]); }
// all monomials of a point at once: powers tabulated per coordinate
inline void mono_all(const std::vector<Mono>& mono, const double* p, double* out) {
  double px[8], py[8], pz[8];
  px[0] = py[0] = pz[0] = 1.0;
  for (int k = 1; k < 8; ++k) {
    px[k] = px[k - 1] * p[0];
    py[k] = py[k - 1] * p[1];
    pz[k] = pz[k - 1] * p[2];
  }
  for (size_t d = 0; d < mono.size(); ++d) out[d] = px[mono[d].e[0]] * py[mono[d].e[1]] * pz[mono[d].e[2]];
}
// D^alpha of a monomial
inline double mono_deriv(const Mono& m, const int* al, const double* p) {
  double c = 1.0;
  int e[3];
  for (int k = 0; k < 3; ++k) {
    if (al[k] > m.e[k]) return 0.0;
    for (int j = 0; j < al[k]; ++j) c *= (m.e[k] - j);
    e[k] = m.e[k] - al[k];
  }
  return c * ipow(p[0], e[0]) * ipow(p[1], e[1]) * ipow(p[2], e[2]);
}

// ----------------------------------------------------------------- dense
// Householder QR of the normal matrix, then R^{-1} Q^T (the reference's
// QRDECOMPOSITION + INVERT, src/matrix.f90:93-150, prestore.f90:4047).
bool qr_inverse(int n, std::vector<double>& A /*n*n row-major, destroyed*/, std::vector<double>& inv) {
  std::vector<double> Q(n * n, 0.0);
  for (int i = 0; i < n; ++i) Q[i * n + i] = 1.0;
  std::vector<double> v(n);
  for (int k = 0; k < n - 1; ++k) {
    double nrm = 0.0;
    for (int i = k; i < n; ++i) nrm += A[i * n + k] * A[i * n + k];
    nrm = std::sqrt(nrm);
    if (nrm == 0.0) continue;
    double alpha = A[k * n + k] > 0 ? -nrm : nrm;
    for (int i = 0; i < n; ++i) v[i] = 0.0;
    for (int i = k; i < n; ++i) v[i] = A[i * n + k];
    v[k] -= alpha;
    double vn = 0.0;
    for (int i = k; i < n; ++i) vn += v[i] * v[i];
    if (vn == 0.0) continue;
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int i = k; i < n; ++i) s += v[i] * A[i * n + j];
      s = 2.0 * s / vn;
      for (int i = k; i < n; ++i) A[i * n + j] -= s * v[i];
    }
    // Q <- Q H
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int j = k; j < n; ++j) s += Q[i * n + j] * v[j];
      s = 2.0 * s / vn;
      for (int j = k; j < n; ++j) Q[i * n + j] -= s * v[j];
    }
  }
  // inv = R^{-1} Q^T
  std::vector<double> Ri(n * n, 0.0);
  for (int i = n - 1; i >= 0; --i) {
    if (A[i * n + i] == 0.0) return false;
    Ri[i * n + i] = 1.0 / A[i * n + i];
    for (int j = i + 1; j < n; ++j) {
      double s = 0.0;
      for (int k = i + 1; k <= j; ++k) s += A[i * n + k] * Ri[k * n + j];
      Ri[i * n + j] = -s / A[i * n + i];
    }
  }
  inv.assign(n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int k = i; k < n; ++k) s += Ri[i * n + k] * Q[j * n + k];
      inv[i * n + j] = s;
    }
  for (double x : inv)
    if (!std::isfinite(x)) return false;
  return true;
}

// -------------------------------------------------------------- mesh data
struct SchemeSizes {
  int scheme = 2, iorder = 1, ees = 0, igq = 1;
  int ideg = 3, imax = 8, numn = 9, admis_max = 1, ideg2 = 0, imax2 = 0, numn2 = 0, iorder2 = 0;
  int iextend = 2, typesten = 1;
  FaceRule qrule, trule;
};

}  // namespace

struct ucp_mesh {
  // cells
  int64_t nc = 0;
  std::vector<int8_t> type;
  std::vector<int64_t> gnode;   // [nc][8] global node ids, -1 unused
  std::vector<double> vx;       // [nc][8][3] vertex coordinates seen from the cell
  double L[3] = {0, 0, 0};
  int per[3] = {0, 0, 0};
  int box_bc[6] = {0, 0, 0, 0, 0, 0};
  double box_lo[3] = {0, 0, 0}, box_hi[3] = {0, 0, 0};
  bool prepared = false;
  bool tables = false;          // basis means and matrix sets built (ucp_prepare)
  std::vector<int32_t> shape32; // ISHAPE per cell as int32 (ucp_shapes)
  SchemeSizes sz;
  // derived geometry
  std::vector<double> centre;   // [nc][3]
  std::vector<int32_t> nfaces, face_type, neigh, neigh_face, bc, qperm;
  std::vector<int32_t> fnode;   // [nc][6][4] local node indices per face (oriented)
  std::vector<double> face_angle, face_area, dih, qpoints, volume, minedge, invccjac, basis_mean;
  std::vector<double> jac_a, jac_det;  // frame origin [nc][3], det [nc]
  std::vector<int32_t> admis, full;
  // reconstruction
  std::vector<int32_t> stencil, table_id;
  int64_t ntab = 0;
  std::vector<double> invmat, invmat2, indicator, indicator2;
  // boundary codes of a mesh read from GRID files, by the sorted global
  // node ids of the face (the last entry -1 for a triangle)
  bool has_bnd = false;
  std::map<std::array<int64_t, 4>, int32_t> bnd_code;
};

namespace {

inline V3 vtx(const ucp_mesh& m, int64_t c, int k) {
  const double* p = &m.vx[(c * 8 + k) * 3];
  return {p[0], p[1], p[2]};
}

V3 wrap(const ucp_mesh& m, V3 d) {
  if (m.per[0]) d.x -= m.L[0] * std::nearbyint(d.x / m.L[0]);
  if (m.per[1]) d.y -= m.L[1] * std::nearbyint(d.y / m.L[1]);
  if (m.per[2]) d.z -= m.L[2] * std::nearbyint(d.z / m.L[2]);
  return d;
}

ucp_mesh* new_mesh(int64_t nc) {
  auto* m = new ucp_mesh;
  m->nc = nc;
  m->type.assign(nc, 1);
  m->gnode.assign(nc * 8, -1);
  m->vx.assign(nc * 8 * 3, 0.0);
  return m;
}

void set_cell(ucp_mesh* m, int64_t c, int type, const int64_t* ids, const V3* pts) {
  m->type[c] = (int8_t)type;
  int nv = topo(type).nv;
  for (int k = 0; k < nv; ++k) {
    m->gnode[c * 8 + k] = ids[k];
    m->vx[(c * 8 + k) * 3 + 0] = pts[k].x;
    m->vx[(c * 8 + k) * 3 + 1] = pts[k].y;
    m->vx[(c * 8 + k) * 3 + 2] = pts[k].z;
  }
}

double tet_signed_vol(V3 a, V3 b, V3 c, V3 d) { return dot(b - a, cross(c - a, d - a)) / 6.0; }

// Node lattice helper for boxes: (i,j,k) -> id with periodic wrap and the
// vertex position as seen from a cell whose lower corner is (ci,cj,ck).
struct Lattice {
  int nx, ny, nz;
  int per[3];
  double h[3], o[3];
  std::vector<V3> disp;  // jitter displacement per node id
  int64_t id(int i, int j, int k) const {
    int ii = per[0] ? ((i % nx) + nx) % nx : i;
    int jj = per[1] ? ((j % ny) + ny) % ny : j;
    int kk = per[2] ? ((k % nz) + nz) % nz : k;
    int64_t sx = per[0] ? nx : nx + 1, sy = per[1] ? ny : ny + 1;
    return ((int64_t)kk * sy + jj) * sx + ii;
  }
  V3 pos(int i, int j, int k) const {
    V3 p = {o[0] + i * h[0], o[1] + j * h[1], o[2] + k * h[2]};
    if (!disp.empty()) p = p + disp[id(i, j, k)];
    return p;
  }
  int64_t nnodes() const {
    return (int64_t)(per[0] ? nx : nx + 1) * (per[1] ? ny : ny + 1) * (per[2] ? nz : nz + 1);
  }
};

// corner (bx,by,bz) of a hexahedron -> node number of the hexahedron
const int kBitToHex[8] = {0, 1, 3, 2, 4, 5, 7, 6};  // index bx + 2 by + 4 bz

// ---------------------------------------------------------- connectivity
struct FaceRec {
  std::array<int64_t, 4> key;
  int64_t cell;
  int face;
  bool operator<(const FaceRec& o) const { return key < o.key || (key == o.key && cell < o.cell); }
};

int bc_of_boundary_face(const ucp_mesh& m, V3 fc, V3 n) {
  // pick the box side the outward normal points to most
  double a[3] = {n.x, n.y, n.z};
  int ax = 0;
  for (int k = 1; k < 3; ++k)
    if (std::fabs(a[k]) > std::fabs(a[ax])) ax = k;
  int side = ax * 2 + (a[ax] > 0 ? 1 : 0);
  (void)fc;
  return m.box_bc[side];
}

// sorted global node ids of face f of cell c (-1 fills a triangle's 4th slot)
std::array<int64_t, 4> face_key(const ucp_mesh& m, int64_t c, int f) {
  std::array<int64_t, 4> k = {-1, -1, -1, -1};
  const int nv = m.face_type[c * 6 + f] == 5 ? 4 : 3;
  for (int i = 0; i < nv; ++i) k[i] = m.gnode[c * 8 + m.fnode[c * 24 + f * 4 + i]];
  std::sort(k.begin(), k.begin() + nv);
  return k;
}

bool build_connectivity(ucp_mesh& m) {
  const int64_t nc = m.nc;
  m.nfaces.assign(nc, 0);
  m.face_type.assign(nc * 6, 0);
  m.neigh.assign(nc * 6, -1);
  m.neigh_face.assign(nc * 6, -1);
  m.bc.assign(nc * 6, 0);
  m.fnode.assign(nc * 24, -1);
  m.centre.assign(nc * 3, 0.0);
  m.volume.assign(nc, 0.0);
  // centres, orientation of faces
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    const Topo& t = topo(m.type[c]);
    V3 cen = {0, 0, 0};
    for (int k = 0; k < t.nv; ++k) cen = cen + vtx(m, c, k);
    cen = (1.0 / t.nv) * cen;
    m.centre[c * 3 + 0] = cen.x;
    m.centre[c * 3 + 1] = cen.y;
    m.centre[c * 3 + 2] = cen.z;
    double vol = 0.0;
    for (int k = 0; k < t.ntet; ++k)
      vol += std::fabs(tet_signed_vol(vtx(m, c, t.tet[k][0]), vtx(m, c, t.tet[k][1]), vtx(m, c, t.tet[k][2]),
                                      vtx(m, c, t.tet[k][3])));
    m.volume[c] = vol;
    m.nfaces[c] = t.nf;
    for (int f = 0; f < t.nf; ++f) {
      int nv = t.fnv[f];
      int ids[4];
      for (int k = 0; k < nv; ++k) ids[k] = t.fv[f][k];
      V3 nrm = {0, 0, 0}, fc = {0, 0, 0};
      for (int k = 0; k < nv; ++k) {
        V3 a = vtx(m, c, ids[k]), b = vtx(m, c, ids[(k + 1) % nv]);
        nrm = nrm + cross(a, b);
        fc = fc + a;
      }
      fc = (1.0 / nv) * fc;
      if (dot(nrm, fc - cen) < 0) std::reverse(ids, ids + nv);
      for (int k = 0; k < nv; ++k) m.fnode[c * 24 + f * 4 + k] = ids[k];
      m.face_type[c * 6 + f] = (nv == 4) ? 5 : 6;
    }
  }
  // match faces by their sorted global node ids
  std::vector<FaceRec> recs;
  recs.reserve(nc * 6);
  for (int64_t c = 0; c < nc; ++c)
    for (int f = 0; f < m.nfaces[c]; ++f) {
      FaceRec r;
      r.key = {-1, -1, -1, -1};
      int nv = m.face_type[c * 6 + f] == 5 ? 4 : 3;
      for (int k = 0; k < nv; ++k) r.key[k] = m.gnode[c * 8 + m.fnode[c * 24 + f * 4 + k]];
      std::sort(r.key.begin(), r.key.begin() + nv);
      r.cell = c;
      r.face = f;
      recs.push_back(r);
    }
  std::sort(recs.begin(), recs.end());
  for (size_t i = 0; i < recs.size();) {
    size_t j = i + 1;
    while (j < recs.size() && recs[j].key == recs[i].key) ++j;
    if (j - i == 2) {
      const FaceRec &a = recs[i], &b = recs[i + 1];
      m.neigh[a.cell * 6 + a.face] = (int32_t)b.cell;
      m.neigh_face[a.cell * 6 + a.face] = b.face;
      m.neigh[b.cell * 6 + b.face] = (int32_t)a.cell;
      m.neigh_face[b.cell * 6 + b.face] = a.face;
    } else if (j - i > 2) {
      set_err("non-manifold face shared by more than two cells");
      return false;
    }
    i = j;
  }
  return true;
}

// ANGLEX / ANGLEY (grid_t.f90:4440-4508): azimuth in [0, 2 pi) by quadrant,
// polar angle by acos.
double angle_x(double a, double b) {
  if (a != 0.0 && b != 0.0) {
    if (a > 0.0 && b > 0.0) return std::atan(b / a);
    if (a < 0.0) return M_PI + std::atan(b / a);
    return 2.0 * M_PI + std::atan(b / a);
  }
  if (a == 0.0 && b != 0.0) return b > 0.0 ? M_PI / 2.0 : 3.0 * (M_PI / 2.0);
  if (a != 0.0 && b == 0.0) return a > 0.0 ? 0.0 : M_PI;
  return 0.0;
}
// Normals within a few ulp of the poles are snapped onto them: acos is
// ill-conditioned there (acos(1-1e-16) = 1.5e-8), and the 1-ulp error of
// normalising an axis-aligned Newell vector would otherwise tilt the face
// by 1e-8 rad and break free-stream preservation at the 1e-8 level.
double angle_y(double c) {
  if (c == 0.0) return std::acos(0.0);
  if (c >= 1.0 - 4.0e-16) return 0.0;
  if (c <= -1.0 + 4.0e-16) return M_PI;
  return std::acos(c);
}

bool build_geometry(ucp_mesh& m) {
  const int64_t nc = m.nc;
  SchemeSizes& s = m.sz;
  const int Q = UCG_MAX_QP;
  m.face_angle.assign(nc * 12, 0.0);
  m.face_area.assign(nc * 6, 0.0);
  m.dih.assign(nc * 6, 0.0);
  m.qpoints.assign(nc * 6 * Q * 3, 0.0);
  m.qperm.assign(nc * 6 * Q, 0);
  m.minedge.assign(nc, 0.0);
  m.invccjac.assign(nc * 9, 0.0);
  m.jac_a.assign(nc * 3, 0.0);
  m.jac_det.assign(nc, 0.0);
  std::vector<double> gpts(nc * 6 * Q * 3, 0.0);  // global qp coordinates
  bool ok = true;
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    const Topo& t = topo(m.type[c]);
    V3 cen = {m.centre[c * 3], m.centre[c * 3 + 1], m.centre[c * 3 + 2]};
    // reference frame from the first tetrahedron (LOCALISE_STEN2)
    V3 a = vtx(m, c, t.tet[0][0]), b = vtx(m, c, t.tet[0][1]), cc = vtx(m, c, t.tet[0][2]), d = vtx(m, c, t.tet[0][3]);
    V3 c1 = b - a, c2 = cc - a, c3 = d - a;  // columns of J
    double det = dot(c1, cross(c2, c3));
    // J^{-1} rows = (c2 x c3, c3 x c1, c1 x c2) / det
    V3 r1 = cross(c2, c3), r2 = cross(c3, c1), r3 = cross(c1, c2);
    double* J = &m.invccjac[c * 9];
    J[0] = r1.x / det; J[1] = r1.y / det; J[2] = r1.z / det;
    J[3] = r2.x / det; J[4] = r2.y / det; J[5] = r2.z / det;
    J[6] = r3.x / det; J[7] = r3.y / det; J[8] = r3.z / det;
    m.jac_a[c * 3] = a.x; m.jac_a[c * 3 + 1] = a.y; m.jac_a[c * 3 + 2] = a.z;
    m.jac_det[c] = det;
    double ssum = 0.0;
    for (int f = 0; f < t.nf; ++f) {
      int nv = m.face_type[c * 6 + f] == 5 ? 4 : 3;
      V3 p[4];
      for (int k = 0; k < nv; ++k) p[k] = vtx(m, c, m.fnode[c * 24 + f * 4 + k]);
      // Newell normal in the difference form of FIND_ROT_ANGLES
      // (grid_t.f90:330-420): axis-aligned faces get exact zero components.
      V3 nrm = {0, 0, 0}, fc = {0, 0, 0};
      for (int k = 0; k < nv; ++k) {
        V3 a0 = p[k], a1 = p[(k + 1) % nv];
        nrm.x += (a0.y - a1.y) * (a0.z + a1.z);
        nrm.y += (a0.z - a1.z) * (a0.x + a1.x);
        nrm.z += (a0.x - a1.x) * (a0.y + a1.y);
        fc = fc + p[k];
      }
      fc = (1.0 / nv) * fc;
      double area = 0.5 * norm(nrm);
      V3 n = (1.0 / norm(nrm)) * nrm;
      m.face_area[c * 6 + f] = area;
      ssum += area;
      m.face_angle[c * 12 + f * 2 + 0] = angle_x(n.x, n.y);  // FACEANGLEX
      m.face_angle[c * 12 + f * 2 + 1] = angle_y(n.z);       // FACEANGLEY
      const FaceRule& R = nv == 4 ? s.qrule : s.trule;
      for (int q = 0; q < R.nq; ++q) {
        V3 x;
        if (nv == 4) {
          double r = R.p[q][0], ss = R.p[q][1];
          x = 0.25 * ((1 - r) * (1 - ss) * p[0] + (1 + r) * (1 - ss) * p[1] + (1 + r) * (1 + ss) * p[2] +
                      (1 - r) * (1 + ss) * p[3]);
        } else {
          x = R.p[q][0] * p[0] + R.p[q][1] * p[1] + R.p[q][2] * p[2];
        }
        double* g = &gpts[((c * 6 + f) * Q + q) * 3];
        g[0] = x.x; g[1] = x.y; g[2] = x.z;
        V3 rel = x - a;
        double* lq = &m.qpoints[((c * 6 + f) * Q + q) * 3];
        lq[0] = J[0] * rel.x + J[1] * rel.y + J[2] * rel.z;
        lq[1] = J[3] * rel.x + J[4] * rel.y + J[5] * rel.z;
        lq[2] = J[6] * rel.x + J[7] * rel.y + J[8] * rel.z;
      }
      int nb = m.neigh[c * 6 + f];
      if (nb < 0) {
        m.bc[c * 6 + f] = bc_of_boundary_face(m, fc, n);
        m.dih[c * 6 + f] = 2.0 * norm(fc - cen);
      } else {
        V3 cn = {m.centre[nb * 3], m.centre[nb * 3 + 1], m.centre[nb * 3 + 2]};
        m.dih[c * 6 + f] = norm(wrap(m, cn - cen));
      }
    }
    m.minedge[c] = 3.0 * m.volume[c] / ssum;
  }
  // codes of a mesh read from GRID files: from GRID.bnd, by face nodes
  if (m.has_bnd)
    for (int64_t c = 0; c < nc; ++c)
      for (int f = 0; f < m.nfaces[c]; ++f) {
        if (m.neigh[c * 6 + f] >= 0) continue;
        const auto it = m.bnd_code.find(face_key(m, c, f));
        if (it == m.bnd_code.end()) {
          set_err("boundary face of cell " + std::to_string(c + 1) + " has no entry in GRID.bnd");
          return false;
        }
        m.bc[c * 6 + f] = it->second;
      }
  // quadrature point pairing across faces
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    V3 cen = {m.centre[c * 3], m.centre[c * 3 + 1], m.centre[c * 3 + 2]};
    for (int f = 0; f < m.nfaces[c]; ++f) {
      int nb = m.neigh[c * 6 + f];
      int nq = m.face_type[c * 6 + f] == 5 ? s.qrule.nq : s.trule.nq;
      if (nb < 0) {
        for (int q = 0; q < nq; ++q) m.qperm[(c * 6 + f) * Q + q] = q;
        continue;
      }
      int g = m.neigh_face[c * 6 + f];
      V3 cn = {m.centre[nb * 3], m.centre[nb * 3 + 1], m.centre[nb * 3 + 2]};
      V3 T = (cen - cn) - wrap(m, cen - cn);  // translation of the neighbour's image
      double h = std::cbrt(m.volume[c]);
      for (int q = 0; q < nq; ++q) {
        const double* x = &gpts[((c * 6 + f) * Q + q) * 3];
        int best = -1;
        double bd = 1e300;
        for (int p = 0; p < nq; ++p) {
          const double* y = &gpts[((int64_t(nb) * 6 + g) * Q + p) * 3];
          double dx = y[0] + T.x - x[0], dy = y[1] + T.y - x[1], dz = y[2] + T.z - x[2];
          double dd = dx * dx + dy * dy + dz * dz;
          if (dd < bd) { bd = dd; best = p; }
        }
        if (std::sqrt(bd) > 1e-6 * h) {
#pragma omp critical
          {
            ok = false;
            set_err_par("face quadrature points of neighbouring cells do not coincide");
          }
        }
        m.qperm[(c * 6 + f) * Q + q] = best;
      }
    }
  }
  return par_result(ok);
}

// ------------------------------------------------------------- stencils
void stencil_sizes(SchemeSizes& s) {
  // DETERMINE_SIZE (grid_p.f90:6097) with extf = 3 (CODE_PROFILE 0)
  int p = s.iorder;
  int ilx = (p + 1) * (p + 2) * (p + 3) / 6;
  s.ideg = ilx - 1;
  s.numn = (p == 1) ? 9 : ilx * 3;
  s.imax = s.numn - 1;
  if (p <= 3) {
    s.ideg2 = 3; s.iorder2 = 1; s.numn2 = (p == 1) ? 7 : 12;
  } else {
    s.ideg2 = 9; s.iorder2 = 2; s.numn2 = 20;
  }
  s.igq = std::min(p, 6);  // IGQRULES (parameters.f90:1390)
  if (s.scheme == 3) {     // WENO (parameters.f90:1338-1372)
    s.iextend = (s.ees == 5) ? 5 : 12;
    s.typesten = 7;
  } else {
    s.iextend = 2;
    s.typesten = 1;
  }
  if (s.ees != 5) { s.ideg2 = 0; s.imax2 = 0; s.numn2 = 0; }
  else s.imax2 = s.numn2 - 1;
  s.admis_max = s.typesten;
  s.qrule = quad_rule(s.igq);
  s.trule = tri_rule(s.igq);
}

// Cone test: is point P inside the cone with apex C through face polygon?
bool in_cone(V3 C, const V3* fv, int nv, V3 P) {
  V3 fc = {0, 0, 0};
  for (int k = 0; k < nv; ++k) fc = fc + fv[k];
  fc = (1.0 / nv) * fc;
  V3 d = P - C;
  double dn = norm(d);
  if (dot(d, fc - C) <= 0) return false;
  for (int k = 0; k < nv; ++k) {
    V3 nrm = cross(fv[k] - C, fv[(k + 1) % nv] - C);
    double ref = dot(nrm, fc - C);
    double val = dot(nrm, d);
    double tol = 1e-9 * norm(nrm) * dn;
    if (ref > 0 ? val < -tol : val > tol) return false;
  }
  return true;
}

bool build_stencils(ucp_mesh& m) {
  SchemeSizes& s = m.sz;
  const int64_t nc = m.nc;
  const int W = s.imax + 1;
  m.stencil.assign(nc * s.admis_max * W, -1);
  m.admis.assign(nc, 0);
  m.full.assign(nc, 0);
  int64_t want = std::min<int64_t>((int64_t)s.numn * s.iextend, nc);
  bool ok = true;
#pragma omp parallel
  {
    std::vector<int64_t> seen_mark(nc, -1);
    std::vector<int32_t> order;
    std::vector<std::pair<int64_t, int64_t>> keyed;  // (quantized distance, bfs index)
#pragma omp for schedule(dynamic, 256)
    for (int64_t c = 0; c < nc; ++c) {
      order.clear();
      order.push_back((int32_t)c);
      seen_mark[c] = c;
      size_t head = 0;
      int64_t target = std::min<int64_t>(2 * want, nc);
      while (head < order.size() && (int64_t)order.size() < target) {
        int32_t x = order[head++];
        for (int f = 0; f < m.nfaces[x]; ++f) {
          int32_t y = m.neigh[(int64_t)x * 6 + f];
          if (y >= 0 && seen_mark[y] != c) {
            seen_mark[y] = c;
            order.push_back(y);
          }
        }
      }
      V3 cen = {m.centre[c * 3], m.centre[c * 3 + 1], m.centre[c * 3 + 2]};
      double h = std::cbrt(m.volume[c]);
      keyed.clear();
      for (size_t k = 0; k < order.size(); ++k) {
        int32_t y = order[k];
        V3 cy = {m.centre[y * 3], m.centre[y * 3 + 1], m.centre[y * 3 + 2]};
        double dist = norm(wrap(m, cy - cen));
        keyed.push_back({(int64_t)std::llround(dist / (1e-7 * h)), (int64_t)k});
      }
      std::sort(keyed.begin(), keyed.end());
      int64_t ncand = std::min<int64_t>((int64_t)keyed.size(), want);
      int32_t* st = &m.stencil[c * s.admis_max * W];
      int nadm = 0;
      // central stencil: the numn nearest cells
      if (ncand >= s.numn) {
        for (int k = 0; k < s.numn; ++k) st[k] = order[keyed[k].second];
        nadm = 1;
      } else {
#pragma omp critical
        {
          ok = false;
          set_err_par("mesh too small for the central stencil");
        }
      }
      // directional stencils (STENCIILSX): candidates inside the cone of each face
      if (s.typesten > 1 && nadm == 1) {
        int target2 = (s.ees == 5) ? s.numn2 : s.numn;
        for (int f = 0; f < m.nfaces[c]; ++f) {
          if (m.neigh[c * 6 + f] < 0) continue;
          int nv = m.face_type[c * 6 + f] == 5 ? 4 : 3;
          V3 fv[4];
          for (int k = 0; k < nv; ++k) fv[k] = vtx(m, c, m.fnode[c * 24 + f * 4 + k]);
          std::vector<int32_t> cand;
          cand.push_back((int32_t)c);
          for (int64_t k = 1; k < ncand && (int)cand.size() < target2; ++k) {
            int32_t y = order[keyed[k].second];
            V3 cy = {m.centre[y * 3], m.centre[y * 3 + 1], m.centre[y * 3 + 2]};
            V3 P = cen + wrap(m, cy - cen);
            if (in_cone(cen, fv, nv, P)) cand.push_back(y);
          }
          if ((int)cand.size() == target2) {
            int32_t* dst = st + nadm * W;
            for (int k = 0; k < target2; ++k) dst[k] = cand[k];
            ++nadm;
          }
        }
      }
      m.admis[c] = nadm;
      // FULL (STENCILS, grid_p.f90:6499-6518): all face stencils admissible
      m.full[c] = (s.scheme == 3 && nadm >= m.nfaces[c] + 1) ? 1 : 0;
    }
  }
  return par_result(ok);
}

// ------------------------------------------------------------- tables
struct Frame {
  double J[9];
  V3 a;
  double absdet;
};
inline V3 to_local(const Frame& F, V3 x) {
  V3 r = x - F.a;
  return {F.J[0] * r.x + F.J[1] * r.y + F.J[2] * r.z, F.J[3] * r.x + F.J[4] * r.y + F.J[5] * r.z,
          F.J[6] * r.x + F.J[7] * r.y + F.J[8] * r.z};
}

// integral over cell y (shifted by T) of each monomial, in frame F
void cell_moments(const ucp_mesh& m, int64_t y, V3 T, const Frame& F, const std::vector<Mono>& mono,
                  const TetRule& R, double* out /*nmono*/) {
  const Topo& t = topo(m.type[y]);
  int nm = (int)mono.size();
  for (int d = 0; d < nm; ++d) out[d] = 0.0;
  for (int k = 0; k < t.ntet; ++k) {
    V3 p[4];
    for (int j = 0; j < 4; ++j) p[j] = to_local(F, vtx(m, y, t.tet[k][j]) + T);
    double vol = std::fabs(tet_signed_vol(p[0], p[1], p[2], p[3]));
    for (size_t q = 0; q < R.w.size(); ++q) {
      V3 x = p[0] + R.p[q][0] * (p[1] - p[0]) + R.p[q][1] * (p[2] - p[0]) + R.p[q][2] * (p[3] - p[0]);
      double xx[3] = {x.x, x.y, x.z}, mv[64];
      mono_all(mono, xx, mv);
      double wv = R.w[q] * vol;
      for (int d = 0; d < nm; ++d) out[d] += wv * mv[d];
    }
  }
}

// smoothness matrix of cell c for `order` (PH1..PH4): sum over all
// derivatives 1 <= |alpha| <= order of the products, integrated in frame F.
void indicator_matrix(const ucp_mesh& m, int64_t c, const Frame& F, int order, const TetRule& R, double* S) {
  std::vector<Mono> mono = monomials(order);
  int n = (int)mono.size();
  std::vector<std::array<int, 3>> al;
  for (int k = 1; k <= order; ++k)
    for (int cz = 0; cz <= k; ++cz)
      for (int by = 0; by <= k - cz; ++by) al.push_back({k - cz - by, by, cz});
  for (int i = 0; i < n * n; ++i) S[i] = 0.0;
  const Topo& t = topo(m.type[c]);
  std::vector<double> D(al.size() * n);
  for (int k = 0; k < t.ntet; ++k) {
    V3 p[4];
    for (int j = 0; j < 4; ++j) p[j] = to_local(F, vtx(m, c, t.tet[k][j]));
    double vol = std::fabs(tet_signed_vol(p[0], p[1], p[2], p[3]));
    for (size_t q = 0; q < R.w.size(); ++q) {
      V3 x = p[0] + R.p[q][0] * (p[1] - p[0]) + R.p[q][1] * (p[2] - p[0]) + R.p[q][2] * (p[3] - p[0]);
      double xx[3] = {x.x, x.y, x.z};
      for (size_t a = 0; a < al.size(); ++a)
        for (int d = 0; d < n; ++d) D[a * n + d] = mono_deriv(mono[d], al[a].data(), xx);
      double wv = R.w[q] * vol;
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          double sacc = 0.0;
          for (size_t a = 0; a < al.size(); ++a) sacc += D[a * n + i] * D[a * n + j];
          S[i * n + j] += wv * sacc;
        }
    }
  }
}

inline uint64_t mix64(uint64_t h, uint64_t v) {
  h ^= v + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
  h *= 0xff51afd7ed558ccdULL;
  h ^= h >> 33;
  return h;
}

// Matrix sets shared by cells whose stencils look the same: keys from the
// stencil members' shapes and vertex positions relative to the cell
// (quantised at 1e-9 of the cell size); table_id[c] numbers the sets in
// the order of the first cell that uses each, rep[t] = that cell.
void assign_tables(ucp_mesh& m, std::vector<int64_t>& rep) {
  SchemeSizes& s = m.sz;
  const int64_t nc = m.nc;
  const int W = s.imax + 1;
  // geometry keys: cells whose stencils look the same share tables
  std::vector<std::array<uint64_t, 2>> key(nc);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    double h = std::cbrt(m.volume[c]);
    double qs = 1.0 / (1e-9 * h);
    V3 cen = {m.centre[c * 3], m.centre[c * 3 + 1], m.centre[c * 3 + 2]};
    uint64_t h1 = 0x1234567ULL, h2 = 0x89abcdefULL;
    const int32_t* st = &m.stencil[c * s.admis_max * W];
    h1 = mix64(h1, m.admis[c]);
    h2 = mix64(h2, m.admis[c] * 7 + 1);
    for (int ll = 0; ll < m.admis[c]; ++ll)
      for (int k = 0; k < W; ++k) {
        int32_t y = st[ll * W + k];
        h1 = mix64(h1, (uint64_t)(y < 0 ? 0 : 1 + m.type[y]));
        h2 = mix64(h2, (uint64_t)(y < 0 ? 5 : 11 + m.type[y]));
        if (y < 0) continue;
        V3 cy = {m.centre[y * 3], m.centre[y * 3 + 1], m.centre[y * 3 + 2]};
        V3 T = wrap(m, cy - cen) - (cy - cen);
        const Topo& t = topo(m.type[y]);
        for (int v = 0; v < t.nv; ++v) {
          V3 p = vtx(m, y, v) + T - cen;
          int64_t q[3] = {std::llround(p.x * qs), std::llround(p.y * qs), std::llround(p.z * qs)};
          for (int j = 0; j < 3; ++j) {
            h1 = mix64(h1, (uint64_t)q[j]);
            h2 = mix64(h2, (uint64_t)q[j] * 0x9e37ULL + 3);
          }
        }
      }
    key[c] = {h1, h2};
  }
  std::vector<int64_t> idx(nc);
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return key[a] < key[b] || (key[a] == key[b] && a < b); });
  m.table_id.assign(nc, -1);
  rep.clear();
  for (int64_t i = 0; i < nc; ++i) {
    if (i == 0 || key[idx[i]] != key[idx[i - 1]]) rep.push_back(idx[i]);
    m.table_id[idx[i]] = (int32_t)(rep.size() - 1);
  }
  // keep table order following the first cell that uses it
  {
    std::vector<int64_t> first(rep.size(), nc);
    for (int64_t c = 0; c < nc; ++c) first[m.table_id[c]] = std::min(first[m.table_id[c]], c);
    std::vector<int64_t> ord(rep.size());
    std::iota(ord.begin(), ord.end(), 0);
    std::sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return first[a] < first[b]; });
    std::vector<int32_t> remap(rep.size());
    std::vector<int64_t> rep2(rep.size());
    for (size_t k = 0; k < ord.size(); ++k) {
      remap[ord[k]] = (int32_t)k;
      rep2[k] = rep[ord[k]];
    }
    for (int64_t c = 0; c < nc; ++c) m.table_id[c] = remap[m.table_id[c]];
    rep.swap(rep2);
  }
  m.ntab = (int64_t)rep.size();
}

bool build_tables(ucp_mesh& m) {
  SchemeSizes& s = m.sz;
  const int64_t nc = m.nc;
  const int W = s.imax + 1;
  const int ideg = s.ideg;
  std::vector<Mono> mono = monomials(s.iorder);
  TetRule Rm = tet_rule(std::max(2, (s.iorder + 4) / 2));
  TetRule Ri = tet_rule(std::max(2, (2 * s.iorder + 2) / 2 + 1));
  m.basis_mean.assign(nc * ideg, 0.0);
  // frames + cell means
  std::vector<Frame> frames(nc);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    Frame& F = frames[c];
    std::memcpy(F.J, &m.invccjac[c * 9], sizeof(F.J));
    F.a = {m.jac_a[c * 3], m.jac_a[c * 3 + 1], m.jac_a[c * 3 + 2]};
    F.absdet = std::fabs(m.jac_det[c]);
    std::vector<double> mom(ideg);
    cell_moments(m, c, {0, 0, 0}, F, mono, Rm, mom.data());
    double vloc = m.volume[c] / F.absdet;  // VOLUME(1,1)
    for (int d = 0; d < ideg; ++d) m.basis_mean[c * ideg + d] = mom[d] / vloc;
  }
  std::vector<int64_t> rep;
  assign_tables(m, rep);
  const int64_t ntab = m.ntab;
  const int A = s.admis_max;
  m.invmat.assign(ntab * A * s.imax * ideg, 0.0);
  if (s.ees == 5) m.invmat2.assign(ntab * A * s.imax2 * s.ideg2, 0.0);
  else m.invmat2.clear();
  if (s.scheme == 3) m.indicator.assign(ntab * ideg * ideg, 0.0);
  else m.indicator.clear();
  if (s.ees == 5) m.indicator2.assign(ntab * s.ideg2 * s.ideg2, 0.0);
  else m.indicator2.clear();
  bool ok = true;
#pragma omp parallel
  {
    std::vector<double> Amat, N, Ninv, mom(ideg);
#pragma omp for schedule(dynamic, 4)
    for (int64_t t = 0; t < ntab; ++t) {
      int64_t c = rep[t];
      const Frame& F = frames[c];
      V3 cen = {m.centre[c * 3], m.centre[c * 3 + 1], m.centre[c * 3 + 2]};
      const int32_t* st = &m.stencil[c * A * W];
      for (int ll = 0; ll < m.admis[c]; ++ll) {
        bool low = (s.ees == 5 && ll > 0);
        int nd = low ? s.ideg2 : ideg;
        int nk = low ? s.imax2 : s.imax;
        Amat.assign(nk * nd, 0.0);
        std::vector<double> vloc(nk);
        for (int k = 0; k < nk; ++k) {
          int32_t y = st[ll * W + k + 1];
          V3 cy = {m.centre[y * 3], m.centre[y * 3 + 1], m.centre[y * 3 + 2]};
          V3 T = wrap(m, cy - cen) - (cy - cen);
          cell_moments(m, y, T, F, mono, Rm, mom.data());
          vloc[k] = m.volume[y] / F.absdet;  // ILOX_VOLUME
          for (int d = 0; d < nd; ++d) Amat[k * nd + d] = mom[d] - vloc[k] * m.basis_mean[c * ideg + d];
        }
        N.assign(nd * nd, 0.0);
        for (int i = 0; i < nd; ++i)
          for (int j = 0; j < nd; ++j) {
            double acc = 0.0;
            for (int k = 0; k < nk; ++k) acc += Amat[k * nd + i] * Amat[k * nd + j];
            N[i * nd + j] = acc;
          }
        if (!qr_inverse(nd, N, Ninv)) {
#pragma omp critical
          {
            ok = false;
            set_err_par("singular least-squares normal matrix");
          }
          continue;
        }
        double* out = low ? &m.invmat2[((t * A + ll) * s.imax2) * s.ideg2] : &m.invmat[((t * A + ll) * s.imax) * ideg];
        for (int k = 0; k < nk; ++k)
          for (int d = 0; d < nd; ++d) {
            double acc = 0.0;
            for (int e = 0; e < nd; ++e) acc += Ninv[d * nd + e] * Amat[k * nd + e];
            out[k * nd + d] = acc * vloc[k];  // column scaling by ILOX_VOLUME (prestore.f90:520-523)
          }
      }
      if (s.scheme == 3) indicator_matrix(m, c, F, s.iorder, Ri, &m.indicator[t * ideg * ideg]);
      if (s.ees == 5) indicator_matrix(m, c, F, s.iorder2, Ri, &m.indicator2[t * s.ideg2 * s.ideg2]);
    }
  }
  return par_result(ok);
}

// ---------------------------------------------------------- IC helpers
void ic_point(int kind, const double* P, int np, const double x[3], double* u) {
  double gamma = P[0];
  double r, uu, vv, ww, p;
  if (kind == UCP_IC_TGV) {
    double p0 = np > 1 ? P[1] : 100.0, r0 = np > 2 ? P[2] : 1.0;
    r = r0;
    uu = std::sin(x[0]) * std::cos(x[1]) * std::cos(x[2]);
    vv = -std::cos(x[0]) * std::sin(x[1]) * std::cos(x[2]);
    ww = 0.0;
    p = p0 + (r0 / 16.0) * (std::cos(2.0 * x[2]) + 2.0) * (std::cos(2.0 * x[0]) + std::cos(2.0 * x[1]));
  } else if (kind == UCP_IC_VORTEX) {
    double beta = P[1], ui = P[2], vi = P[3], wi = P[4];
    double xc = P[5] + ui * P[8], yc = P[6] + vi * P[8];
    double Lx = P[9], Ly = P[10];
    double dx = x[0] - xc, dy = x[1] - yc;
    if (Lx > 0) dx -= Lx * std::nearbyint(dx / Lx);
    if (Ly > 0) dy -= Ly * std::nearbyint(dy / Ly);
    double r2 = dx * dx + dy * dy;
    double e = std::exp(0.5 * (1.0 - r2));
    double du = -beta / (2.0 * M_PI) * e * dy, dv = beta / (2.0 * M_PI) * e * dx;
    double dT = -(gamma - 1.0) * beta * beta / (8.0 * gamma * M_PI * M_PI) * e * e;
    double T = 1.0 + dT;
    r = std::pow(T, 1.0 / (gamma - 1.0));
    p = r * T;
    uu = ui + du;
    vv = vi + dv;
    ww = wi;
  } else {
    r = P[1]; uu = P[2]; vv = P[3]; ww = P[4]; p = P[5];
  }
  u[0] = r;
  u[1] = r * uu;
  u[2] = r * vv;
  u[3] = r * ww;
  u[4] = p / (gamma - 1.0) + 0.5 * r * (uu * uu + vv * vv + ww * ww);
}

}  // namespace

// ================================================================== C ABI
extern "C" {

const char* ucp_last_error(void) { return g_err.c_str(); }

static ucp_mesh* make_box(int32_t nx, int32_t ny, int32_t nz, const double L[3], const double origin[3],
                          const int32_t periodic[3], const int32_t bc[6], bool tets, double jitter, uint64_t seed) {
  if (nx < 1 || ny < 1 || nz < 1 || !L) {
    set_err("bad box size");
    return nullptr;
  }
  Lattice lat;
  lat.nx = nx; lat.ny = ny; lat.nz = nz;
  for (int k = 0; k < 3; ++k) lat.per[k] = periodic ? periodic[k] : 0;
  lat.h[0] = L[0] / nx; lat.h[1] = L[1] / ny; lat.h[2] = L[2] / nz;
  for (int k = 0; k < 3; ++k) lat.o[k] = origin ? origin[k] : 0.0;
  if (tets && jitter > 0) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    int64_t nn = lat.nnodes();
    lat.disp.assign(nn, {0, 0, 0});
    int sx = lat.per[0] ? nx : nx + 1, sy = lat.per[1] ? ny : ny + 1, sz = lat.per[2] ? nz : nz + 1;
    for (int k = 0; k < sz; ++k)
      for (int j = 0; j < sy; ++j)
        for (int i = 0; i < sx; ++i) {
          V3 d = {U(rng) * jitter * lat.h[0], U(rng) * jitter * lat.h[1], U(rng) * jitter * lat.h[2]};
          if (!lat.per[0] && (i == 0 || i == nx)) d.x = 0;
          if (!lat.per[1] && (j == 0 || j == ny)) d.y = 0;
          if (!lat.per[2] && (k == 0 || k == nz)) d.z = 0;
          lat.disp[lat.id(i, j, k)] = d;
        }
  }
  int64_t nh = (int64_t)nx * ny * nz;
  ucp_mesh* m = new_mesh(tets ? nh * 6 : nh);
  for (int k = 0; k < 3; ++k) {
    m->L[k] = L[k];
    m->per[k] = lat.per[k];
    m->box_lo[k] = lat.o[k];
    m->box_hi[k] = lat.o[k] + L[k];
  }
  for (int k = 0; k < 6; ++k) m->box_bc[k] = bc ? bc[k] : 0;
  // Kuhn split of the cube about the diagonal (0,0,0)-(1,1,1): one tet per
  // ordering of the axes; conforming between neighbouring cubes.
  const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  for (int kk = 0; kk < nz; ++kk)
    for (int jj = 0; jj < ny; ++jj)
      for (int ii = 0; ii < nx; ++ii) {
        int64_t hc = ((int64_t)kk * ny + jj) * nx + ii;
        int64_t ids[8];
        V3 pts[8];
        for (int b = 0; b < 8; ++b) {
          int bx = b & 1, by = (b >> 1) & 1, bz = (b >> 2) & 1;
          int hn = kBitToHex[b];
          ids[hn] = lat.id(ii + bx, jj + by, kk + bz);
          pts[hn] = lat.pos(ii + bx, jj + by, kk + bz);
        }
        if (!tets) {
          set_cell(m, hc, 1, ids, pts);
          continue;
        }
        for (int t = 0; t < 6; ++t) {
          int bits[4];
          bits[0] = 0;
          int cur = 0;
          for (int s = 0; s < 3; ++s) {
            cur |= (1 << perm[t][s]);
            bits[s + 1] = cur;
          }
          int64_t tid[4];
          V3 tp[4];
          for (int s = 0; s < 4; ++s) {
            tid[s] = ids[kBitToHex[bits[s]]];
            tp[s] = pts[kBitToHex[bits[s]]];
          }
          if (tet_signed_vol(tp[0], tp[1], tp[2], tp[3]) < 0) {
            std::swap(tid[2], tid[3]);
            std::swap(tp[2], tp[3]);
          }
          set_cell(m, hc * 6 + t, 2, tid, tp);
        }
      }
  return m;
}

ucp_mesh* ucp_box_hex(int32_t nx, int32_t ny, int32_t nz, const double L[3], const double origin[3],
                      const int32_t periodic[3], const int32_t bc[6]) {
  return make_box(nx, ny, nz, L, origin, periodic, bc, false, 0.0, 0);
}

ucp_mesh* ucp_box_tet(int32_t nx, int32_t ny, int32_t nz, const double L[3], const double origin[3],
                      const int32_t periodic[3], const int32_t bc[6], double jitter, uint64_t seed) {
  return make_box(nx, ny, nz, L, origin, periodic, bc, true, jitter, seed);
}

ucp_mesh* ucp_bump_channel(int32_t nx, int32_t ny, int32_t nlayers, double bump, double dz, double split_frac,
                           uint64_t seed) {
  if (nx < 2 || ny < 1 || nlayers < 1) {
    set_err("bad channel size");
    return nullptr;
  }
  // 2D node (i,j): x = 3 i/nx; lower wall y0(x) = bump*sin^2(pi (x-1)) on [1,2]
  auto node = [&](int i, int j, int k) -> V3 {
    double x = 3.0 * i / nx;
    double y0 = (x > 1.0 && x < 2.0) ? bump * std::pow(std::sin(M_PI * (x - 1.0)), 2) : 0.0;
    double y = y0 + (1.0 - y0) * (double)j / ny;
    return {x, y, k * dz};
  };
  auto nid = [&](int i, int j, int k) -> int64_t { return ((int64_t)k * (ny + 1) + j) * (nx + 1) + i; };
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  std::vector<int> split((size_t)nx * ny);
  for (auto& s : split) s = U(rng) < split_frac ? 1 : 0;
  int64_t nc2 = 0;
  for (int s : split) nc2 += s ? 2 : 1;
  ucp_mesh* m = new_mesh(nc2 * nlayers);
  m->box_lo[0] = 0; m->box_hi[0] = 3;
  m->box_lo[1] = 0; m->box_hi[1] = 1;
  m->box_lo[2] = 0; m->box_hi[2] = nlayers * dz;
  const int bcs[6] = {1, 2, 4, 4, 3, 3};
  for (int k = 0; k < 6; ++k) m->box_bc[k] = bcs[k];
  int64_t c = 0;
  for (int k = 0; k < nlayers; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        int q[4][2] = {{i, j}, {i + 1, j}, {i + 1, j + 1}, {i, j + 1}};
        if (!split[(size_t)j * nx + i]) {
          int64_t ids[8];
          V3 pts[8];
          for (int a = 0; a < 4; ++a) {
            ids[a] = nid(q[a][0], q[a][1], k);
            pts[a] = node(q[a][0], q[a][1], k);
            ids[a + 4] = nid(q[a][0], q[a][1], k + 1);
            pts[a + 4] = node(q[a][0], q[a][1], k + 1);
          }
          set_cell(m, c++, 1, ids, pts);
        } else {
          // split along the (i,j)-(i+1,j+1) diagonal
          const int tri[2][3] = {{0, 1, 2}, {0, 2, 3}};
          for (int t = 0; t < 2; ++t) {
            int64_t ids[6];
            V3 pts[6];
            for (int a = 0; a < 3; ++a) {
              int qa = tri[t][a];
              ids[a] = nid(q[qa][0], q[qa][1], k);
              pts[a] = node(q[qa][0], q[qa][1], k);
              ids[a + 3] = nid(q[qa][0], q[qa][1], k + 1);
              pts[a + 3] = node(q[qa][0], q[qa][1], k + 1);
            }
            set_cell(m, c++, 4, ids, pts);
          }
        }
      }
  return m;
}

ucp_mesh* ucp_mixed_box(int32_t n, double L, uint64_t seed) {
  if (n < 6 || (n % 2)) {
    set_err("mixed box needs an even n >= 6");
    return nullptr;
  }
  Lattice lat;
  lat.nx = lat.ny = lat.nz = n;
  lat.per[0] = lat.per[1] = lat.per[2] = 1;
  lat.h[0] = lat.h[1] = lat.h[2] = L / n;
  lat.o[0] = lat.o[1] = lat.o[2] = 0.0;
  // layer kinds: 0 hex, 1 transition up (pyramid base down), 2 Kuhn tets,
  // 3 prisms about z, 4 transition down (pyramid base up)
  std::vector<int> kind(n, 0);
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  kind[n / 2] = 1;
  for (int k = n / 2 + 1; k < n - 1; ++k) kind[k] = U(rng) < 0.5 ? 2 : 3;
  kind[n - 1] = 4;
  int64_t per_layer[5] = {1, 5, 6, 2, 5};
  int64_t nc = 0;
  for (int k = 0; k < n; ++k) nc += per_layer[kind[k]] * (int64_t)n * n;
  ucp_mesh* m = new_mesh(nc);
  for (int k = 0; k < 3; ++k) {
    m->L[k] = L;
    m->per[k] = 1;
    m->box_lo[k] = 0;
    m->box_hi[k] = L;
  }
  const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  int64_t c = 0;
  for (int kk = 0; kk < n; ++kk)
    for (int jj = 0; jj < n; ++jj)
      for (int ii = 0; ii < n; ++ii) {
        int64_t ids[8];
        V3 pts[8];
        for (int b = 0; b < 8; ++b) {
          int bx = b & 1, by = (b >> 1) & 1, bz = (b >> 2) & 1;
          int hn = kBitToHex[b];
          ids[hn] = lat.id(ii + bx, jj + by, kk + bz);
          pts[hn] = lat.pos(ii + bx, jj + by, kk + bz);
        }
        auto put = [&](int type, std::initializer_list<int> nodes) {
          int64_t id2[8];
          V3 p2[8];
          int j = 0;
          for (int v : nodes) {
            id2[j] = ids[v];
            p2[j] = pts[v];
            ++j;
          }
          if (type == 2 && tet_signed_vol(p2[0], p2[1], p2[2], p2[3]) < 0) {
            std::swap(id2[2], id2[3]);
            std::swap(p2[2], p2[3]);
          }
          set_cell(m, c++, type, id2, p2);
        };
        switch (kind[kk]) {
          case 0: put(1, {0, 1, 2, 3, 4, 5, 6, 7}); break;
          case 1:  // pyramid on the bottom face with apex at node 4, and 4 tets
            put(3, {0, 1, 2, 3, 4});
            put(2, {2, 4, 5, 6});
            put(2, {2, 4, 6, 7});
            put(2, {2, 4, 3, 7});
            put(2, {2, 4, 1, 5});
            break;
          case 2:
            for (int t = 0; t < 6; ++t) {
              int bits[4] = {0, 0, 0, 0}, cur = 0;
              for (int s = 0; s < 3; ++s) {
                cur |= (1 << perm[t][s]);
                bits[s + 1] = cur;
              }
              put(2, {kBitToHex[bits[0]], kBitToHex[bits[1]], kBitToHex[bits[2]], kBitToHex[bits[3]]});
            }
            break;
          case 3:
            put(4, {0, 1, 2, 4, 5, 6});
            put(4, {0, 2, 3, 4, 6, 7});
            break;
          case 4:  // mirror of case 1 in z: pyramid on the top face, apex node 0
            put(3, {4, 5, 6, 7, 0});
            put(2, {6, 0, 1, 2});
            put(2, {6, 0, 2, 3});
            put(2, {6, 0, 7, 3});
            put(2, {6, 0, 5, 1});
            break;
        }
      }
  return m;
}

// ------------------------------------------------------------ GRID files
// UCNS3D's ASCII grid (OPEN_ARBITRARY, io.f90:4157-4304; FIND_SHAPE,
// grid_p.f90:1652-1743; READ_BOUND, bc_p.f90:36-130): GRID.vrt "id x y z",
// GRID.cel "id n1 .. n8" with the shape told by repeated nodes (hexahedron:
// all distinct; tetrahedron n3 = n4, n5 = n6 = n7 = n8; pyramid n5 = .. = n8;
// prism n3 = n4, n7 = n8), GRID.bnd "id n1 n2 n3 n4 code" (a triangle has
// n3 = n4).  Ids are 1-based.
ucp_mesh* ucp_read_grid(const char* prefix) {
  const std::string pre = prefix ? prefix : "";
  FILE* fv = std::fopen((pre + "GRID.vrt").c_str(), "r");
  FILE* fc = std::fopen((pre + "GRID.cel").c_str(), "r");
  FILE* fb = std::fopen((pre + "GRID.bnd").c_str(), "r");
  auto close_all = [&]() {
    if (fv) std::fclose(fv);
    if (fc) std::fclose(fc);
    if (fb) std::fclose(fb);
  };
  if (!fv || !fc || !fb) {
    close_all();
    set_err("cannot open " + pre + "GRID.vrt, GRID.cel or GRID.bnd");
    return nullptr;
  }
  std::vector<V3> node;
  long long id;
  double x, y, z;
  while (std::fscanf(fv, "%lld %lf %lf %lf", &id, &x, &y, &z) == 4) {
    if (id < 1) {
      close_all();
      set_err("GRID.vrt: node ids start at 1");
      return nullptr;
    }
    if ((size_t)id > node.size()) node.resize(id, {std::nan(""), 0, 0});
    node[id - 1] = {x, y, z};
  }
  std::vector<std::array<long long, 8>> cells;
  std::array<long long, 8> n8;
  while (std::fscanf(fc, "%lld %lld %lld %lld %lld %lld %lld %lld %lld", &id, &n8[0], &n8[1], &n8[2], &n8[3], &n8[4],
                     &n8[5], &n8[6], &n8[7]) == 9)
    cells.push_back(n8);
  ucp_mesh* m = new_mesh((int64_t)cells.size());
  bool ok = !cells.empty();
  if (!ok) set_err("GRID.cel holds no cells");
  for (int64_t c = 0; ok && c < (int64_t)cells.size(); ++c) {
    const auto& a = cells[c];
    int type;
    int slot[8];
    int nv;
    if (a[4] != a[5] && a[5] != a[6] && a[6] != a[7] && a[2] != a[3]) {
      type = 1, nv = 8;
      for (int k = 0; k < 8; ++k) slot[k] = k;
    } else if (a[2] == a[3] && a[4] == a[5] && a[5] == a[6] && a[6] == a[7]) {
      type = 2, nv = 4;
      slot[0] = 0, slot[1] = 1, slot[2] = 2, slot[3] = 4;
    } else if (a[2] != a[3] && a[4] == a[5] && a[5] == a[6] && a[6] == a[7]) {
      type = 3, nv = 5;
      for (int k = 0; k < 5; ++k) slot[k] = k;
    } else if (a[2] == a[3] && a[4] != a[5] && a[6] == a[7]) {
      type = 4, nv = 6;
      slot[0] = 0, slot[1] = 1, slot[2] = 2, slot[3] = 4, slot[4] = 5, slot[5] = 6;
    } else {
      set_err("GRID.cel: cell " + std::to_string(c + 1) + " is none of hexahedron, tetrahedron, pyramid, prism");
      ok = false;
      break;
    }
    int64_t ids[8];
    V3 pts[8];
    for (int k = 0; k < nv; ++k) {
      const long long g = a[slot[k]];
      if (g < 1 || (size_t)g > node.size() || std::isnan(node[g - 1].x)) {
        set_err("GRID.cel: cell " + std::to_string(c + 1) + " names a node missing from GRID.vrt");
        ok = false;
        break;
      }
      ids[k] = g - 1;
      pts[k] = node[g - 1];
    }
    if (ok) set_cell(m, c, type, ids, pts);
  }
  struct BndFace {
    std::array<int64_t, 4> k;  // 0-based node ids in file order, -1 for a triangle's fourth
    int nv, code;
  };
  std::vector<BndFace> bnd;
  long long b[4];
  int code;
  while (ok && std::fscanf(fb, "%lld %lld %lld %lld %lld %d", &id, &b[0], &b[1], &b[2], &b[3], &code) == 6) {
    const int nv = b[2] == b[3] ? 3 : 4;
    BndFace r{{b[0] - 1, b[1] - 1, b[2] - 1, nv == 3 ? -1 : b[3] - 1}, nv, code};
    for (int k = 0; k < nv; ++k)
      if (r.k[k] < 0 || (size_t)r.k[k] >= node.size() || std::isnan(node[r.k[k]].x)) {
        set_err("GRID.bnd: face " + std::to_string(id) + " names a node missing from GRID.vrt");
        ok = false;
      }
    bnd.push_back(r);
  }
  close_all();
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (const V3& p : node)
    if (!std::isnan(p.x)) {
      lo[0] = std::min(lo[0], p.x), hi[0] = std::max(hi[0], p.x);
      lo[1] = std::min(lo[1], p.y), hi[1] = std::max(hi[1], p.y);
      lo[2] = std::min(lo[2], p.z), hi[2] = std::max(hi[2], p.z);
    }
  for (int k = 0; k < 3; ++k) {
    m->box_lo[k] = lo[k];
    m->box_hi[k] = hi[k];
    m->L[k] = hi[k] - lo[k];  // XPER, YPER, ZPER of READ_INPUT (io.f90:4977-4979)
  }
  // Periodic faces (codes 5 and 50; APPLY_BOUNDARY, bc_p.f90:499-620): a
  // face whose centroid lies on the low side of the bounding box in one
  // axis pairs with the face of the same shape on the high side whose
  // centroid has the same other two coordinates.  The pair's nodes are
  // then one node each (matched by those two coordinates), so the faces
  // meet like interior faces and the axis is periodic with the box's
  // extent as the period.
  std::vector<int64_t> rep(node.size());
  std::iota(rep.begin(), rep.end(), 0);
  auto find = [&](int64_t a) {
    while (rep[a] != a) a = rep[a] = rep[rep[a]];
    return a;
  };
  auto coord = [](const V3& p, int k) { return k == 0 ? p.x : k == 1 ? p.y : p.z; };
  const double ext = std::max({1.0, std::fabs(lo[0]), std::fabs(lo[1]), std::fabs(lo[2]), std::fabs(hi[0]),
                               std::fabs(hi[1]), std::fabs(hi[2])});
  const double tol = 1e-13 * ext;  // TOLSMALL of the reference, relative to the coordinates' size
  struct PerFace {
    V3 c;
    size_t i;
  };
  std::vector<PerFace> side[3][2];
  for (size_t i = 0; ok && i < bnd.size(); ++i) {
    if (bnd[i].code != 5 && bnd[i].code != 50) continue;
    V3 c = {0, 0, 0};
    for (int k = 0; k < bnd[i].nv; ++k) c = c + node[bnd[i].k[k]];
    c = (1.0 / bnd[i].nv) * c;
    int axis = -1, hiside = 0;
    for (int a = 0; a < 3 && axis < 0; ++a) {
      if (std::fabs(coord(c, a) - lo[a]) < tol) axis = a, hiside = 0;
      else if (std::fabs(coord(c, a) - hi[a]) < tol) axis = a, hiside = 1;
    }
    if (axis < 0) {
      set_err("GRID.bnd: periodic face " + std::to_string(i + 1) + " does not lie on a side of the bounding box");
      ok = false;
      break;
    }
    side[axis][hiside].push_back({c, i});
  }
  for (int a = 0; ok && a < 3; ++a) {
    if (side[a][0].empty() && side[a][1].empty()) continue;
    const int a1 = (a + 1) % 3, a2 = (a + 2) % 3;
    auto& H = side[a][1];
    std::sort(H.begin(), H.end(), [&](const PerFace& u, const PerFace& v) { return coord(u.c, a1) < coord(v.c, a1); });
    std::vector<char> used(H.size(), 0);
    size_t paired = 0;
    for (const PerFace& f : side[a][0]) {
      const BndFace& A = bnd[f.i];
      size_t j = std::lower_bound(H.begin(), H.end(), coord(f.c, a1) - tol,
                                  [&](const PerFace& u, double x) { return coord(u.c, a1) < x; }) -
                 H.begin();
      for (; j < H.size() && coord(H[j].c, a1) <= coord(f.c, a1) + tol; ++j)
        if (!used[j] && bnd[H[j].i].nv == A.nv && std::fabs(coord(H[j].c, a2) - coord(f.c, a2)) < tol) break;
      if (j >= H.size() || coord(H[j].c, a1) > coord(f.c, a1) + tol) {
        set_err("GRID.bnd: periodic face " + std::to_string(f.i + 1) + " has no partner on the opposite side");
        ok = false;
        break;
      }
      used[j] = 1;
      ++paired;
      const BndFace& B = bnd[H[j].i];
      for (int u = 0; u < B.nv && ok; ++u) {
        const V3& q = node[B.k[u]];
        int match = -1;
        for (int v = 0; v < A.nv; ++v) {
          const V3& pa = node[A.k[v]];
          if (std::fabs(coord(pa, a1) - coord(q, a1)) < tol && std::fabs(coord(pa, a2) - coord(q, a2)) < tol) match = v;
        }
        if (match < 0) {
          set_err("GRID.bnd: the nodes of periodic faces " + std::to_string(f.i + 1) + " and " +
                  std::to_string(H[j].i + 1) + " do not match");
          ok = false;
          break;
        }
        const int64_t x = find(A.k[match]), y = find(B.k[u]);
        if (x != y) rep[std::max(x, y)] = std::min(x, y);
      }
    }
    if (ok && paired != H.size()) {
      set_err("GRID.bnd: a periodic face on the high side of axis " + std::to_string(a) + " has no partner");
      ok = false;
    }
    if (ok) m->per[a] = 1;
  }
  if (ok && (m->per[0] || m->per[1] || m->per[2]))
    for (int64_t c = 0; c < m->nc && ok; ++c) {
      const int nv = topo(m->type[c]).nv;
      for (int k = 0; k < nv; ++k) m->gnode[c * 8 + k] = find(m->gnode[c * 8 + k]);
      for (int k = 0; k < nv && ok; ++k)
        for (int l = k + 1; l < nv; ++l)
          if (m->gnode[c * 8 + k] == m->gnode[c * 8 + l]) {
            set_err("GRID: cell " + std::to_string(c + 1) + " meets its own periodic image");
            ok = false;
            break;
          }
    }
  for (const BndFace& r : bnd) {
    if (!ok) break;
    if (r.code == 5 || r.code == 50) continue;
    std::array<int64_t, 4> k = r.k;
    for (int v = 0; v < r.nv; ++v) k[v] = find(k[v]);
    std::sort(k.begin(), k.begin() + r.nv);
    m->bnd_code[k] = r.code;
  }
  if (!ok) {
    delete m;
    return nullptr;
  }
  m->has_bnd = true;
  return m;
}

int32_t ucp_write_grid(const ucp_mesh* m, const char* prefix) {
  if (!m || !m->prepared) {
    set_err("write_grid needs a prepared mesh (its boundary faces and codes)");
    return UCG_ESTATE;
  }
  const bool periodic = m->per[0] || m->per[1] || m->per[2];
  // nodes by global id (each node's position as its first cell sees it);
  // on a periodic mesh a node seen by a cell across a periodic side (shifted
  // by a whole period) is written again as its own image node
  int64_t nn = 0;
  for (int64_t c = 0; c < m->nc; ++c)
    for (int k = 0; k < topo(m->type[c]).nv; ++k) nn = std::max(nn, m->gnode[c * 8 + k] + 1);
  std::vector<V3> pos(nn);
  std::vector<char> seen(nn, 0);
  std::map<std::array<int64_t, 4>, int64_t> image;  // (global id, shift in x, y, z) -> 0-based output id
  std::vector<V3> ipos;
  std::vector<int64_t> cid((size_t)m->nc * 8, -1);  // output node id of each cell vertex
  for (int64_t c = 0; c < m->nc; ++c)
    for (int k = 0; k < topo(m->type[c]).nv; ++k) {
      const int64_t g = m->gnode[c * 8 + k];
      const V3 p = vtx(*m, c, k);
      if (!seen[g]) {
        seen[g] = 1;
        pos[g] = p;
      }
      const V3 d = p - pos[g];
      const std::array<int64_t, 4> key = {g, m->per[0] ? std::llround(d.x / m->L[0]) : 0,
                                          m->per[1] ? std::llround(d.y / m->L[1]) : 0,
                                          m->per[2] ? std::llround(d.z / m->L[2]) : 0};
      if (key[1] == 0 && key[2] == 0 && key[3] == 0) {
        cid[c * 8 + k] = g;
        continue;
      }
      auto it = image.find(key);
      if (it == image.end()) {
        it = image.emplace(key, nn + (int64_t)ipos.size()).first;
        ipos.push_back(p);
      }
      cid[c * 8 + k] = it->second;
    }
  // faces across a periodic side: the neighbour sees them shifted by a period
  auto face_centre = [&](int64_t c, int f) {
    const int nv = m->face_type[c * 6 + f] == 5 ? 4 : 3;
    V3 s = {0, 0, 0};
    for (int k = 0; k < nv; ++k) s = s + vtx(*m, c, m->fnode[c * 24 + f * 4 + k]);
    return (1.0 / nv) * s;
  };
  auto across = [&](int64_t c, int f) {
    const int64_t nb = m->neigh[c * 6 + f];
    if (!periodic || nb < 0) return false;
    const V3 d = face_centre(c, f) - face_centre(nb, m->neigh_face[c * 6 + f]);
    return norm(d) > 1e-9 * std::max({m->L[0], m->L[1], m->L[2]});
  };
  if (periodic) {
    const double tol = 1e-13 * std::max({1.0, std::fabs(m->box_lo[0]), std::fabs(m->box_lo[1]),
                                         std::fabs(m->box_lo[2]), std::fabs(m->box_hi[0]), std::fabs(m->box_hi[1]),
                                         std::fabs(m->box_hi[2])});
    for (int64_t c = 0; c < m->nc; ++c)
      for (int f = 0; f < m->nfaces[c]; ++f) {
        if (!across(c, f)) continue;
        const V3 fc = face_centre(c, f);
        const double x[3] = {fc.x, fc.y, fc.z};
        bool side = false;
        for (int a = 0; a < 3; ++a)
          side = side || (m->per[a] && (std::fabs(x[a] - m->box_lo[a]) < tol || std::fabs(x[a] - m->box_hi[a]) < tol));
        if (!side) {
          set_err("write_grid: a periodic face of cell " + std::to_string(c + 1) +
                  " is off the sides of the box, where the GRID format's periodic pairing looks for it");
          return UCG_EINVAL;
        }
      }
  }
  const std::string pre = prefix ? prefix : "";
  FILE* fv = std::fopen((pre + "GRID.vrt").c_str(), "w");
  FILE* fc = std::fopen((pre + "GRID.cel").c_str(), "w");
  FILE* fb = std::fopen((pre + "GRID.bnd").c_str(), "w");
  if (!fv || !fc || !fb) {
    if (fv) std::fclose(fv);
    if (fc) std::fclose(fc);
    if (fb) std::fclose(fb);
    set_err("cannot create " + pre + "GRID.vrt, GRID.cel or GRID.bnd");
    return UCG_EINVAL;
  }
  for (int64_t g = 0; g < nn; ++g)
    if (seen[g]) std::fprintf(fv, "%lld %.17g %.17g %.17g\n", (long long)(g + 1), pos[g].x, pos[g].y, pos[g].z);
  for (size_t i = 0; i < ipos.size(); ++i)
    std::fprintf(fv, "%lld %.17g %.17g %.17g\n", (long long)(nn + i + 1), ipos[i].x, ipos[i].y, ipos[i].z);
  for (int64_t c = 0; c < m->nc; ++c) {
    const int64_t* gn = &cid[c * 8];
    long long s[8];
    switch (m->type[c]) {
      case 1: for (int k = 0; k < 8; ++k) s[k] = gn[k]; break;
      case 2: s[0] = gn[0], s[1] = gn[1], s[2] = s[3] = gn[2], s[4] = s[5] = s[6] = s[7] = gn[3]; break;
      case 3: for (int k = 0; k < 5; ++k) s[k] = gn[k]; s[5] = s[6] = s[7] = gn[4]; break;
      default: s[0] = gn[0], s[1] = gn[1], s[2] = s[3] = gn[2], s[4] = gn[3], s[5] = gn[4], s[6] = s[7] = gn[5];
    }
    std::fprintf(fc, "%lld %lld %lld %lld %lld %lld %lld %lld %lld\n", (long long)(c + 1), s[0] + 1, s[1] + 1, s[2] + 1,
                 s[3] + 1, s[4] + 1, s[5] + 1, s[6] + 1, s[7] + 1);
  }
  long long ib = 0;
  for (int64_t c = 0; c < m->nc; ++c)
    for (int f = 0; f < m->nfaces[c]; ++f) {
      const bool per_face = across(c, f);
      if (m->neigh[c * 6 + f] >= 0 && !per_face) continue;
      const int nv = m->face_type[c * 6 + f] == 5 ? 4 : 3;
      long long g[4];
      for (int k = 0; k < nv; ++k) g[k] = cid[c * 8 + m->fnode[c * 24 + f * 4 + k]] + 1;
      if (nv == 3) g[3] = g[2];
      std::fprintf(fb, "%lld %lld %lld %lld %lld %d\n", ++ib, g[0], g[1], g[2], g[3], per_face ? 5 : m->bc[c * 6 + f]);
    }
  const bool bad = std::ferror(fv) || std::ferror(fc) || std::ferror(fb);
  std::fclose(fv);
  std::fclose(fc);
  std::fclose(fb);
  if (bad) {
    set_err("write error in the GRID files");
    return UCG_EINVAL;
  }
  return UCG_OK;
}

static int32_t prepare(ucp_mesh* m, const ucp_scheme* s, bool tables) {
  if (!m || !s) {
    set_err("null argument");
    return UCG_EINVAL;
  }
  if (s->iorder < 1 || s->iorder > 4 || (s->scheme != 2 && s->scheme != 3) || (s->ees != 0 && s->ees != 5)) {
    set_err("unsupported scheme (scheme 2|3, iorder 1..4, ees 0|5)");
    return UCG_EINVAL;
  }
#ifdef _OPENMP
  if (s->nthreads > 0) omp_set_num_threads(s->nthreads);
#endif
  m->sz = SchemeSizes();
  m->sz.scheme = s->scheme;
  m->sz.iorder = s->iorder;
  m->sz.ees = s->scheme == 3 ? s->ees : 0;
  stencil_sizes(m->sz);
  if (!build_connectivity(*m)) return UCG_EINVAL;
  if (!build_geometry(*m)) return UCG_EINVAL;
  if (!build_stencils(*m)) return UCG_EINVAL;
  m->tables = false;
  m->basis_mean.clear();
  m->invmat.clear();
  m->invmat2.clear();
  m->indicator.clear();
  m->indicator2.clear();
  m->table_id.clear();
  m->ntab = 0;
  if (tables) {
    if (!build_tables(*m)) return UCG_EINVAL;
  } else {
    std::vector<int64_t> rep;
    assign_tables(*m, rep);
  }
  m->tables = tables;
  m->shape32.assign(m->type.begin(), m->type.end());
  m->prepared = true;
  return UCG_OK;
}

int32_t ucp_prepare(ucp_mesh* m, const ucp_scheme* s) { return prepare(m, s, true); }
int32_t ucp_prepare_geometry(ucp_mesh* m, const ucp_scheme* s) { return prepare(m, s, false); }

int32_t ucp_shapes(const ucp_mesh* m, ucg_shapes* out) {
  if (!m || !out || !m->prepared) {
    set_err("mesh not prepared");
    return UCG_ESTATE;
  }
  out->ncells = m->nc;
  out->shape = m->shape32.data();
  out->vertices = m->vx.data();
  out->centre = m->centre.data();
  out->volume = m->volume.data();
  out->frame = m->invccjac.data();
  out->frame_origin = m->jac_a.data();
  out->frame_det = m->jac_det.data();
  for (int k = 0; k < 3; ++k) out->period[k] = m->per[k] ? m->L[k] : 0.0;
  return UCG_OK;
}

int64_t ucp_ncells(const ucp_mesh* m) { return m ? m->nc : 0; }
int64_t ucp_ntables(const ucp_mesh* m) { return m ? m->ntab : 0; }

int32_t ucp_fill_config(const ucp_mesh* m, ucg_config* cfg) {
  if (!m || !cfg || !m->prepared) {
    set_err("mesh not prepared");
    return UCG_ESTATE;
  }
  const SchemeSizes& s = m->sz;
  cfg->scheme = s.scheme;
  cfg->iorder = s.iorder;
  cfg->ees = s.ees;
  cfg->ideg = s.ideg;
  cfg->imax = s.imax;
  cfg->admis_max = s.admis_max;
  cfg->ideg2 = s.ideg2;
  cfg->imax2 = s.imax2;
  cfg->nq_quad = s.qrule.nq;
  cfg->nq_tri = s.trule.nq;
  for (int q = 0; q < UCG_MAX_QP; ++q) {
    cfg->quad_w[q] = q < s.qrule.nq ? s.qrule.w[q] : 0.0;
    cfg->tri_w[q] = q < s.trule.nq ? s.trule.w[q] : 0.0;
  }
  return UCG_OK;
}

int32_t ucp_geometry(const ucp_mesh* m, ucg_geometry* g) {
  if (!m || !g || !m->prepared) {
    set_err("mesh not prepared");
    return UCG_ESTATE;
  }
  g->ncells = m->nc;
  g->nfaces = m->nfaces.data();
  g->face_type = m->face_type.data();
  g->neigh = m->neigh.data();
  g->neigh_face = m->neigh_face.data();
  g->bc = m->bc.data();
  g->qperm = m->qperm.data();
  g->face_angle = m->face_angle.data();
  g->face_area = m->face_area.data();
  g->dih = m->dih.data();
  g->qpoints = m->qpoints.data();
  g->volume = m->volume.data();
  g->minedge = m->minedge.data();
  g->invccjac = m->invccjac.data();
  g->basis_mean = m->tables ? m->basis_mean.data() : nullptr;
  g->admis = m->admis.data();
  g->full = m->full.data();
  return UCG_OK;
}

int32_t ucp_recon(const ucp_mesh* m, ucg_recon* r) {
  if (!m || !r || !m->prepared) {
    set_err("mesh not prepared");
    return UCG_ESTATE;
  }
  r->first = 0;
  r->count = m->nc;
  r->stencil = m->stencil.data();
  r->ntables = m->ntab;
  r->table_id = m->table_id.data();
  r->invmat = m->tables ? m->invmat.data() : nullptr;
  r->invmat2 = m->invmat2.empty() ? nullptr : m->invmat2.data();
  r->indicator = m->indicator.empty() ? nullptr : m->indicator.data();
  r->indicator2 = m->indicator2.empty() ? nullptr : m->indicator2.data();
  return UCG_OK;
}

int32_t ucp_cell_centres(const ucp_mesh* m, double* xyz) {
  if (!m || !xyz) return UCG_EINVAL;
  if (m->centre.size() == (size_t)m->nc * 3) {
    std::memcpy(xyz, m->centre.data(), sizeof(double) * m->nc * 3);
    return UCG_OK;
  }
  for (int64_t c = 0; c < m->nc; ++c) {
    const Topo& t = topo(m->type[c]);
    V3 cen = {0, 0, 0};
    for (int k = 0; k < t.nv; ++k) cen = cen + vtx(*m, c, k);
    xyz[c * 3] = cen.x / t.nv;
    xyz[c * 3 + 1] = cen.y / t.nv;
    xyz[c * 3 + 2] = cen.z / t.nv;
  }
  return UCG_OK;
}

int32_t ucp_initial_condition(const ucp_mesh* m, int32_t kind, const double* params, int32_t nparams, double* u) {
  if (!m || !params || !u || nparams < 1) {
    set_err("bad initial condition arguments");
    return UCG_EINVAL;
  }
  if (kind != UCP_IC_TGV && kind != UCP_IC_VORTEX && kind != UCP_IC_UNIFORM) {
    set_err("unknown initial condition");
    return UCG_EINVAL;
  }
  if ((kind == UCP_IC_VORTEX && nparams < 11) || (kind == UCP_IC_UNIFORM && nparams < 6)) {
    set_err("too few initial condition parameters");
    return UCG_EINVAL;
  }
  TetRule R = tet_rule(4);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < m->nc; ++c) {
    const Topo& t = topo(m->type[c]);
    double acc[5] = {0, 0, 0, 0, 0}, vol = 0.0;
    for (int k = 0; k < t.ntet; ++k) {
      V3 p[4];
      for (int j = 0; j < 4; ++j) p[j] = vtx(*m, c, t.tet[k][j]);
      double v = std::fabs(tet_signed_vol(p[0], p[1], p[2], p[3]));
      for (size_t q = 0; q < R.w.size(); ++q) {
        V3 x = p[0] + R.p[q][0] * (p[1] - p[0]) + R.p[q][1] * (p[2] - p[0]) + R.p[q][2] * (p[3] - p[0]);
        double xx[3] = {x.x, x.y, x.z}, uq[5];
        ic_point(kind, params, nparams, xx, uq);
        for (int j = 0; j < 5; ++j) acc[j] += R.w[q] * v * uq[j];
      }
      vol += v;
    }
    for (int j = 0; j < 5; ++j) u[c * 5 + j] = acc[j] / vol;
  }
  return UCG_OK;
}

void ucp_free(ucp_mesh* m) { delete m; }

}  // extern "C"
