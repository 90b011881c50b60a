// ORACLE - test infrastructure only.
//
// A plain FP64 CPU restatement of UCNS3D's explicit residual and SSP-RK3
// step, used by tests/ as the checker of the CUDA engine and by bench.py as
// the timed CPU baseline ("port": the Fortran reference cannot be built
// here - no Fortran compiler, no MPI).  It is never linked into, loaded by or
// called from the engine.  Parity is UNPINNED at the reference-test level:
// the reference ships no golden vectors or known-answer tests (its only test
// mesh is missing), so this restatement is pinned by the property tests in
// tests/ (free-stream preservation, exactness, conservation, consistency).
//
// It follows the reference's operation order, per cell:
//   LEAST_SQUARES -> COMPUTE_GRADIENTS_MEAN_LSQ      src/gradients.f90:253-497
//   COMPUTE_GRADIENTS_INNER_MEAN_LSQ_VISCOUS         src/gradients.f90:502-706
//   WENOWEIGHTS / CP_RECONSTRUCTION / EXTRAPOLATE_BOUND
//                                                    src/reconstruct_p.f90:407-1250, 1556
//   CHARACTERISTIC_RECONSTRUCTION (WENWRT = 2) + WENO_NEIGHBOUR +
//   compute_gradcharv_smoothindicator + diag_At_B_A  src/reconstruct_p.f90:497-917, 1608-1818
//   COMPUTE_EIGENVECTORS                             src/flow_operations.f90:3934-3995
//   CHECKSOL                                         src/reconstruct_p.f90:3126-3242
//   MUSCL / FIND_BOUNDS / COMPUTE_MUSCL_RECONSTRUCTION / SLOPE_LIMITERS(1-9)
//                                                    src/reconstruct_p.f90:2286, 1821, 2044, 3421
//   CHECKSOLX                                        src/reconstruct_p.f90:3245-3406
//   SOLUTIONTRIAV2                                   src/reconstruct_p.f90:2358
//   CALCULATE_FLUXESHI_CONVECTIVE + HLLC / RUSANOV / HLL_RIEMANN_SOLVER + ROTATEF/ROTATEB
//                                                    src/flux_p.f90:478, riemann.f90:221, 1236, 28,
//                                                    grid_t.f90:4217
//   CALCULATE_FLUXESHI_DIFFUSIVE + SUTHERLAND        src/flux_p.f90:1520, flow_operations.f90:2609
//   CALCULATE_BOUNDED_VISCOUS (walls, boundaries)    src/dg_functions.f90:1179
//   BOUNDARYS (inflow/outflow/symmetry/wall/far field, BOUNDTYPE 0|1)
//                                                    src/flow_operations.f90:2860-3375
//   RUNGE_KUTTA3, CALCULATE_CFL                      src/time_p.f90:885-1027, 27-191
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "ucns3d_gpu.h"

namespace {

const int F = UCG_MAX_FACES, Q = UCG_MAX_QP, NV = 5;
const double TOLSMALL = 1.0e-13, TOLBIG = 1.0e13;  // grid_p.f90:18-19

struct Mono {
  int e[3];
};
std::vector<Mono> monos(int order) {
  std::vector<Mono> m;
  for (int n = 1; n <= order; ++n)
    for (int c = 0; c <= n; ++c)
      for (int b = 0; b <= n - c; ++b) m.push_back({{n - c - b, b, c}});
  return m;
}
double pw(double x, int e) {
  double r = 1.0;
  for (int i = 0; i < e; ++i) r *= x;
  return r;
}

struct Ctx {
  const ucg_config* cfg;
  const ucg_geometry* g;
  const ucg_recon* r;
  int64_t n;
  std::vector<Mono> mono;
};

void cons2prim(const Ctx& x, const double* u, double* p) {
  double oo = 1.0 / u[0];
  p[0] = u[0];
  p[1] = u[1] * oo;
  p[2] = u[2] * oo;
  p[3] = u[3] * oo;
  p[4] = (x.cfg->gamma - 1.0) * (u[4] - 0.5 * u[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]));
}

// basis at a local point: monomial minus its cell mean (BASIS_REC, icompwrt 0/1)
void basis(const Ctx& x, int64_t c, const double* xi, int nd, double* b) {
  for (int d = 0; d < nd; ++d) {
    const Mono& m = x.mono[d];
    b[d] = pw(xi[0], m.e[0]) * pw(xi[1], m.e[1]) * pw(xi[2], m.e[2]) - x.g->basis_mean[c * x.cfg->ideg + d];
  }
}
// d/dxi_k of the monomials (DFX, DFY, DFZ)
void dbasis(const Ctx& x, const double* xi, int nd, double* dx, double* dy, double* dz) {
  for (int d = 0; d < nd; ++d) {
    const Mono& m = x.mono[d];
    double X = xi[0], Y = xi[1], Z = xi[2];
    dx[d] = m.e[0] ? m.e[0] * pw(X, m.e[0] - 1) * pw(Y, m.e[1]) * pw(Z, m.e[2]) : 0.0;
    dy[d] = m.e[1] ? m.e[1] * pw(X, m.e[0]) * pw(Y, m.e[1] - 1) * pw(Z, m.e[2]) : 0.0;
    dz[d] = m.e[2] ? m.e[2] * pw(X, m.e[0]) * pw(Y, m.e[1]) * pw(Z, m.e[2] - 1) : 0.0;
  }
}

inline int nq_of(const Ctx& x, int64_t c, int f) {
  return x.g->face_type[c * F + f] == 5 ? x.cfg->nq_quad : x.cfg->nq_tri;
}
inline double wq_of(const Ctx& x, int64_t c, int f, int q) {
  return x.g->face_type[c * F + f] == 5 ? x.cfg->quad_w[q] : x.cfg->tri_w[q];
}
inline int tab(const Ctx& x, int64_t c) { return x.r->table_id ? x.r->table_id[c] : (int)c; }

// Venkatakrishnan limiter (SLOPE_LIMITERS case 7)
double venkat(double usol, double u0, double umin, double umax, double minedge, double kappa) {
  double d2 = usol - u0;
  if (std::fabs(d2) <= 0.0) return 1.0;
  double dmin = d2;
  dmin = std::copysign(1.0, dmin) * (std::fabs(dmin) + TOLSMALL);
  double dplus = (d2 > 0.0) ? umax - u0 : umin - u0;
  double epsi2 = std::pow(kappa * minedge, 3);
  return (1.0 / dmin) * ((((dplus * dplus) + epsi2) * dmin + (2.0 * (dmin * dmin) * dplus)) /
                         ((dplus * dplus) + (2.0 * dmin * dmin) + (dmin * dplus) + epsi2));
}

// SLOPE_LIMITERS (reconstruct_p.f90:3421-3945) for limiter codes 1-9
double slope_limiter(int kind, double usol, double u0, double umin, double umax, double minedge, double kappa) {
  if (kind == 7) return venkat(usol, u0, umin, umax, minedge, kappa);
  const double d2 = usol - u0;
  if (std::fabs(d2) <= 0.0) return 1.0;
  double psi;
  if (kind == 4 || kind == 8) {
    psi = venkat(usol, u0, umin, umax, minedge, kappa);
  } else {
    const double sfd = ((d2 > 0.0) ? (umax - u0) : (umin - u0)) / d2;
    if (kind == 1) psi = std::min(1.0, sfd);
    else if (kind == 5) psi = (sfd * sfd + sfd) / (sfd * sfd + 1.0);
    else if (kind == 6) psi = 2.0 * sfd / (sfd + 1.0);
    else psi = (sfd < 1.5) ? -((4.0 / 27.0) * std::pow(sfd, 3)) + sfd : 1.0;
  }
  if (kind == 2 || kind == 3 || kind == 9 || kind == 4 || kind == 8) {
    const double delu = umax - umin, e3 = std::pow(kappa * minedge, 3);
    double sig;
    if (delu * delu <= e3) {
      sig = 1.0;
    } else if (delu * delu < 2.0 * e3) {
      const double y = (delu * delu - e3) / e3;
      sig = (2.0 * std::pow(y, 3)) - (3.0 * std::pow(y, 2)) + 1.0;
    } else {
      sig = 0.0;
    }
    psi = sig + (1.0 - sig) * psi;
  }
  return psi;
}

// MUSCL on one cell: ULEFT from the central-stencil polynomial G0 [ideg][5]
void muscl_cell(const Ctx& x, int64_t c, const double* U, const double* G0, double* ul /*[F][Q][5]*/) {
  const ucg_geometry* g = x.g;
  const int ideg = x.cfg->ideg;
  const double* u0 = U + c * NV;
  double umin[NV], umax[NV];
  for (int v = 0; v < NV; ++v) umin[v] = umax[v] = u0[v];
  for (int f = 0; f < g->nfaces[c]; ++f) {
    int64_t nb = g->neigh[c * F + f];
    if (nb < 0) continue;  // physical boundary faces add no bound (FIND_BOUNDS)
    for (int v = 0; v < NV; ++v) {
      umin[v] = std::min(umin[v], U[nb * NV + v]);
      umax[v] = std::max(umax[v], U[nb * NV + v]);
    }
  }
  double usol[F][Q][NV], slope[NV];
  for (int v = 0; v < NV; ++v) slope[v] = TOLBIG;
  std::vector<double> b(ideg);
  for (int f = 0; f < g->nfaces[c]; ++f)
    for (int q = 0; q < nq_of(x, c, f); ++q) {
      basis(x, c, &g->qpoints[((c * F + f) * Q + q) * 3], ideg, b.data());
      for (int v = 0; v < NV; ++v) {
        double res = 0.0;
        for (int d = 0; d < ideg; ++d) res += b[d] * G0[d * NV + v];
        usol[f][q][v] = u0[v] + res;
        double psi = slope_limiter(x.cfg->limiter, usol[f][q][v], u0[v], umin[v], umax[v], g->minedge[c],
                                   x.cfg->kappa_ven);
        slope[v] = std::min(slope[v], psi);
      }
    }
  for (int f = 0; f < g->nfaces[c]; ++f)
    for (int q = 0; q < nq_of(x, c, f); ++q)
      for (int v = 0; v < NV; ++v) {
        double du = usol[f][q][v] - u0[v];
        ul[(f * Q + q) * NV + v] = u0[v] + du * slope[v];
      }
}

// CHECKSOL / CHECKSOLX test of one cell's face values against its mean
bool jump_check(const Ctx& x, int64_t c, const double* u0, const double* ul, double jump) {
  double pr[NV], pl[NV];
  cons2prim(x, u0, pr);
  for (int f = 0; f < x.g->nfaces[c]; ++f)
    for (int q = 0; q < nq_of(x, c, f); ++q) {
      cons2prim(x, &ul[(f * Q + q) * NV], pl);
      if (std::fabs(pl[0] - pr[0]) >= jump * pr[0]) return true;
      if (std::fabs(pl[4] - pr[4]) >= jump * pr[4]) return true;
      if (pl[4] < 0.0 || pl[0] < 0.0) return true;
    }
  return false;
}

// reconstruction of one cell: face values ul [F][Q][5] and, for
// Navier-Stokes, face gradients ulv [F][Q][4][3] of (T, u, v, w)
void char_faces(const Ctx& x, int64_t c, const double* U, const double* G, double* ul);

// MOOD (recalc != nullptr, RUNGE_KUTTA3_MOOD): every cell gets its WENO
// values; a reduced cell (CHECKSOL or not FULL) takes the MUSCL fall-back only
// if recalc[c] (RECALC of the last MOOD pass: MUSCL, reconstruct_p.f90:2306-
// 2315, with RECALC from FIX_LIST, mood.f90:440-518), then CHECKSOLX as
// always.  reduced (optional): the cell's REDUCE; G0 (optional, [ideg][5]):
// the central stencil polynomial.
void reconstruct_cell(const Ctx& x, int64_t c, const double* U, double* ul, double* ulv,
                      const int8_t* recalc = nullptr, int8_t* reduced = nullptr, double* G0 = nullptr) {
  const ucg_config* cfg = x.cfg;
  const ucg_geometry* g = x.g;
  const ucg_recon* r = x.r;
  const int ideg = cfg->ideg, imax = cfg->imax, A = cfg->admis_max, W = imax + 1;
  const int ideg2 = cfg->ideg2, imax2 = cfg->imax2;
  const int t = tab(x, c);
  const int32_t* st = &r->stencil[c * A * W];
  const double* u0 = U + c * NV;
  const int admis = g->admis[c];
  // ---- least squares, every admissible stencil
  std::vector<double> G((size_t)A * ideg * NV, 0.0);  // [ll][d][v]
  for (int ll = 0; ll < admis; ++ll) {
    bool low = (cfg->ees == 5 && ll > 0);
    int nk = low ? imax2 : imax, nd = low ? ideg2 : ideg;
    const double* M = low ? &r->invmat2[((int64_t)t * A + ll) * imax2 * ideg2] : &r->invmat[((int64_t)t * A + ll) * imax * ideg];
    for (int d = 0; d < nd; ++d)
      for (int v = 0; v < NV; ++v) {
        double s = 0.0;
        for (int k = 0; k < nk; ++k) {
          int64_t y = st[ll * W + k + 1];
          s += M[k * nd + d] * (U[y * NV + v] - u0[v]);
        }
        G[((size_t)ll * ideg + d) * NV + v] = s;
      }
  }
  bool reduce = false;
  if (cfg->scheme == 3 && cfg->wenwrt == 2) {
    // ---- CHARACTERISTIC_RECONSTRUCTION, then CHECKSOL
    char_faces(x, c, U, G.data(), ul);
    if (!g->full[c]) reduce = true;
    else reduce = jump_check(x, c, u0, ul, 0.85);
  } else if (cfg->scheme == 3) {
    // ---- CP_RECONSTRUCTION
    std::vector<double> w((size_t)A * NV);
    std::vector<double> g1((size_t)ideg * NV, 0.0);  // central polynomial (CWENO)
    for (int v = 0; v < NV; ++v) {
      std::vector<double> is(admis), lam(admis), wt(admis);
      if (cfg->ees == 5) {
        double lc1 = 1.0 - 1.0 / cfg->lwci;
        lam[0] = lc1;
        for (int ll = 1; ll < admis; ++ll) lam[ll] = (1.0 - lc1) / (admis - 1);
        std::vector<double> g3(ideg, 0.0);
        for (int ll = 1; ll < admis; ++ll)
          for (int d = 0; d < ideg2; ++d) g3[d] = g3[d] + lam[ll] * G[((size_t)ll * ideg + d) * NV + v];
        std::vector<double> gg(ideg);
        for (int d = 0; d < ideg; ++d) {
          gg[d] = (1.0 / lam[0]) * (G[(size_t)d * NV + v] - g3[d]);
          g1[d * NV + v] = gg[d];
        }
        const double* S = &r->indicator[(int64_t)t * ideg * ideg];
        double acc = 0.0;
        for (int d = 0; d < ideg; ++d) {
          double sg = 0.0;
          for (int e = 0; e < ideg; ++e) sg += S[d * ideg + e] * gg[e];
          acc += gg[d] * sg;
        }
        is[0] = acc;
        const double* S2 = &r->indicator2[(int64_t)t * ideg2 * ideg2];
        for (int ll = 1; ll < admis; ++ll) {
          double a2 = 0.0;
          for (int d = 0; d < ideg2; ++d) {
            double sg = 0.0;
            for (int e = 0; e < ideg2; ++e) sg += S2[d * ideg2 + e] * G[((size_t)ll * ideg + e) * NV + v];
            a2 += G[((size_t)ll * ideg + d) * NV + v] * sg;
          }
          is[ll] = a2;
        }
      } else {
        const double* S = &r->indicator[(int64_t)t * ideg * ideg];
        for (int ll = 0; ll < admis; ++ll) {
          double acc = 0.0;
          for (int d = 0; d < ideg; ++d) {
            double sg = 0.0;
            for (int e = 0; e < ideg; ++e) sg += S[d * ideg + e] * G[((size_t)ll * ideg + e) * NV + v];
            acc += G[((size_t)ll * ideg + d) * NV + v] * sg;
          }
          is[ll] = acc;
        }
        for (int ll = 0; ll < admis; ++ll) lam[ll] = 1.0;
        lam[0] = cfg->lwci;
      }
      const double eps = cfg->weno_eps;
      if (cfg->ees == 5 && cfg->wenoz) {
        double tau = 0.0;
        for (int ll = 0; ll < admis; ++ll) tau = tau + std::fabs(is[0] - is[ll]);
        tau = tau / (admis - 1);
        for (int ll = 0; ll < admis; ++ll) wt[ll] = lam[ll] * (1.0 + std::pow(tau / (eps + is[ll]), 4));
      } else {
        for (int ll = 0; ll < admis; ++ll) wt[ll] = lam[ll] / std::pow(eps + is[ll], 4);
      }
      double sum = 0.0;
      for (int ll = 0; ll < admis; ++ll) sum = sum + wt[ll];
      for (int ll = 0; ll < admis; ++ll) w[(size_t)ll * NV + v] = wt[ll] / sum;
    }
    // face values: sum over stencils of weight * (U + basis . g)
    for (int i = 0; i < F * Q * NV; ++i) ul[i] = 0.0;
    std::vector<double> b(ideg);
    for (int ll = 0; ll < admis; ++ll) {
      bool low = (cfg->ees == 5 && ll > 0);
      int nd = low ? ideg2 : ideg;
      for (int f = 0; f < g->nfaces[c]; ++f)
        for (int q = 0; q < nq_of(x, c, f); ++q) {
          basis(x, c, &g->qpoints[((c * F + f) * Q + q) * 3], ideg, b.data());
          for (int v = 0; v < NV; ++v) {
            double res = 0.0;
            for (int d = 0; d < nd; ++d) {
              double gv = (cfg->ees == 5 && ll == 0) ? g1[d * NV + v] : G[((size_t)ll * ideg + d) * NV + v];
              res += b[d] * gv;
            }
            double* o = &ul[(f * Q + q) * NV + v];
            *o = *o + (u0[v] + res) * w[(size_t)ll * NV + v];
          }
        }
    }
    // CHECKSOL
    if (!g->full[c]) reduce = true;
    else reduce = jump_check(x, c, u0, ul, 0.85);
  }
  if (!g->full[c]) reduce = true;
  if (reduced) *reduced = reduce ? 1 : 0;
  if (G0)
    for (int i = 0; i < ideg * NV; ++i) G0[i] = G[i];
  // MUSCL (all cells for scheme 2; flagged cells for WENO; under MOOD only
  // the flagged cells of the last RECALC)
  if (recalc ? (reduce && recalc[c]) : (cfg->scheme == 2 || reduce)) muscl_cell(x, c, U, G.data(), ul);
  // CHECKSOLX: first order where the face values jump too far
  if (jump_check(x, c, u0, ul, 0.95)) {
    for (int f = 0; f < F; ++f)
      for (int q = 0; q < Q; ++q)
        for (int v = 0; v < NV; ++v) ul[(f * Q + q) * NV + v] = u0[v];
  }
  // ---- SOLUTIONTRIAV2: face gradients of (T, u, v, w) from stencil 1
  if (cfg->governing == 1) {
    double p0[NV];
    cons2prim(x, u0, p0);
    double s1[4] = {p0[4] / (p0[0] * cfg->r_gas), p0[1], p0[2], p0[3]};
    std::vector<double> Gv((size_t)ideg * 4, 0.0);
    const double* M = &r->invmat[((int64_t)t * A + 0) * imax * ideg];
    for (int d = 0; d < ideg; ++d)
      for (int v = 0; v < 4; ++v) {
        double s = 0.0;
        for (int k = 0; k < imax; ++k) {
          int64_t y = st[k + 1];
          double py[NV];
          cons2prim(x, &U[y * NV], py);
          double s2[4] = {py[4] / (py[0] * cfg->r_gas), py[1], py[2], py[3]};
          s += M[k * ideg + d] * (s2[v] - s1[v]);
        }
        Gv[d * 4 + v] = s;
      }
    const double* J = &g->invccjac[c * 9];
    std::vector<double> bx(ideg), by(ideg), bz(ideg);
    for (int f = 0; f < g->nfaces[c]; ++f)
      for (int q = 0; q < nq_of(x, c, f); ++q) {
        dbasis(x, &g->qpoints[((c * F + f) * Q + q) * 3], ideg, bx.data(), by.data(), bz.data());
        for (int v = 0; v < 4; ++v) {
          double gl[3] = {0.0, 0.0, 0.0};
          for (int d = 0; d < ideg; ++d) gl[0] += Gv[d * 4 + v] * bx[d];
          for (int d = 0; d < ideg; ++d) gl[1] += Gv[d * 4 + v] * by[d];
          for (int d = 0; d < ideg; ++d) gl[2] += Gv[d * 4 + v] * bz[d];
          // AINVJT = INVCCJAC^T
          for (int k = 0; k < 3; ++k)
            ulv[((f * Q + q) * 4 + v) * 3 + k] = J[0 * 3 + k] * gl[0] + J[1 * 3 + k] * gl[1] + J[2 * 3 + k] * gl[2];
        }
      }
  }
}

void rotf(const double* a, const double* v, double* o) {
  // ROTATEF; a = (cos a1, sin a1, cos a2, sin a2)
  double ca1 = a[0], sa1 = a[1], ca2 = a[2], sa2 = a[3];
  o[0] = v[0];
  o[1] = ca1 * sa2 * v[1] + sa1 * sa2 * v[2] + ca2 * v[3];
  o[2] = ca1 * ca2 * v[1] + sa1 * ca2 * v[2] - sa2 * v[3];
  o[3] = -sa1 * v[1] + ca1 * v[2];
  o[4] = v[4];
}
void rotb(const double* a, const double* v, double* o) {
  double ca1 = a[0], sa1 = a[1], ca2 = a[2], sa2 = a[3];
  o[0] = v[0];
  o[1] = ca1 * sa2 * v[1] + ca1 * ca2 * v[2] - sa1 * v[3];
  o[2] = sa1 * sa2 * v[1] + sa1 * ca2 * v[2] + ca1 * v[3];
  o[3] = ca2 * v[1] - sa2 * v[2];
  o[4] = v[4];
}

void hllc(double gamma, const double* cl, const double* cr, double* flux) {
  double rl = cl[0], ul = cl[1] / rl, vl = cl[2] / rl, wl = cl[3] / rl;
  double pl = (gamma - 1.0) * (cl[4] - 0.5 * rl * (ul * ul + vl * vl + wl * wl));
  double rr = cr[0], ur = cr[1] / rr, vr = cr[2] / rr, wr = cr[3] / rr;
  double pr = (gamma - 1.0) * (cr[4] - 0.5 * rr * (ur * ur + vr * vr + wr * wr));
  double el = cl[4], er = cr[4];
  double ccl = std::sqrt(gamma * pl / rl), ccr = std::sqrt(gamma * pr / rr);
  double srl = std::sqrt(rl), srr = std::sqrt(rr);
  double cc2 = std::sqrt((((ccl * ccl) * srl) + ((ccr * ccr) * srr)) / (srl + srr) +
                         0.5 * ((srl * srr) / ((srl + srr) * (srl + srr))) * ((ur - ul) * (ur - ul)));
  double uu2 = ((ul * srl) + (ur * srr)) / (srl + srr);
  double sl = std::min(ul - ccl, uu2 - cc2), sr = std::max(ur + ccr, uu2 + cc2);
  sl = std::min(sl, 0.0);
  sr = std::max(sr, 0.0);
  double sm = (pr - pl + (rl * ul * (sl - ul)) - (rr * ur * (sr - ur))) / ((rl * (sl - ul)) - (rr * (sr - ur)));
  double fl[5] = {rl * ul, rl * ul * ul + pl, rl * ul * vl, rl * ul * wl, ul * (el + pl)};
  double fr[5] = {rr * ur, rr * ur * ur + pr, rr * ur * vr, rr * ur * wr, ur * (er + pr)};
  double mul = rl * ((sl - ul) / (sl - sm)), mur = rr * ((sr - ur) / (sr - sm));
  double lastl = (el / rl) + ((sm - ul) * (sm + (pl / (rl * (sl - ul)))));
  double lastr = (er / rr) + ((sm - ur) * (sm + (pr / (rr * (sr - ur)))));
  double ls[5] = {mul, mul * sm, mul * vl, mul * wl, mul * lastl};
  double rs[5] = {mur, mur * sm, mur * vr, mur * wr, mur * lastr};
  double sg = std::copysign(1.0, sm);
  for (int k = 0; k < 5; ++k)
    flux[k] = (((1.0 + sg) / 2.0) * (fl[k] + sl * (ls[k] - cl[k]))) + (((1.0 - sg) / 2.0) * (fr[k] + sr * (rs[k] - cr[k])));
}

// RUSANOV_RIEMANN_SOLVER (riemann.f90:1236-1403) and HLL_RIEMANN_SOLVER
// (riemann.f90:28-217, Davis wave speeds) in the face frame
void xflux(double gamma, const double* c, double* f, double& u, double& p) {
  const double r = c[0];
  u = c[1] / r;
  const double v = c[2] / r, w = c[3] / r;
  p = (gamma - 1.0) * (c[4] - 0.5 * r * (u * u + v * v + w * w));
  f[0] = r * u;
  f[1] = (r * (u * u)) + p;
  f[2] = r * u * v;
  f[3] = r * u * w;
  f[4] = u * (c[4] + p);
}
void rusanov(double gamma, const double* cl, const double* cr, double* flux) {
  double fl[5], fr[5], ul, ur, pl, pr;
  xflux(gamma, cl, fl, ul, pl);
  xflux(gamma, cr, fr, ur, pr);
  const double sl = std::fabs(ul) + std::sqrt(gamma * pl / cl[0]);
  const double sr = std::fabs(ur) + std::sqrt(gamma * pr / cr[0]);
  const double smax = std::max(std::fabs(sl), std::fabs(sr));
  for (int k = 0; k < 5; ++k) flux[k] = 0.5 * (fl[k] + fr[k]) - 0.5 * smax * (cr[k] - cl[k]);
}
void hll(double gamma, const double* cl, const double* cr, double* flux) {
  double fl[5], fr[5], ul, ur, pl, pr;
  xflux(gamma, cl, fl, ul, pl);
  xflux(gamma, cr, fr, ur, pr);
  const double ccl = std::sqrt(gamma * pl / cl[0]), ccr = std::sqrt(gamma * pr / cr[0]);
  const double sl = std::min(ul - ccl, ur - ccr), sr = std::max(ul + ccl, ur + ccr);
  for (int k = 0; k < 5; ++k) {
    const double fhll = (sr * fl[k] - sl * fr[k] + (sl * sr * (cr[k] - cl[k]))) / (sr - sl);
    double f = 0.0;
    if (sl >= 0.0) f = fl[k];
    if (sr <= 0.0) f = fr[k];
    if (sl <= 0.0 && sr >= 0.0) f = fhll;
    flux[k] = f;
  }
}
// ROE_RIEMANN_SOLVER (riemann.f90:433-632): global frame, face normal n,
// entropy fix of the acoustic waves (width 0.2)
void roe(double gamma, const double* cl, const double* cr, const double* n, double* flux) {
  const double nx = n[0], ny = n[1], nz = n[2];
  const double rhoL = cl[0], uL = cl[1] / rhoL, vL = cl[2] / rhoL, wL = cl[3] / rhoL;
  const double pL = (gamma - 1.0) * (cl[4] - 0.5 * rhoL * (uL * uL + vL * vL + wL * wL));
  const double rhoR = cr[0], uR = cr[1] / rhoR, vR = cr[2] / rhoR, wR = cr[3] / rhoR;
  const double pR = (gamma - 1.0) * (cr[4] - 0.5 * rhoR * (uR * uR + vR * vR + wR * wR));
  const double qnL = uL * nx + vL * ny + wL * nz, qnR = uR * nx + vR * ny + wR * nz;
  const double aL = std::sqrt(gamma * pL / rhoL), aR = std::sqrt(gamma * pR / rhoR);
  const double HL = aL * aL / (gamma - 1.0) + 0.5 * (uL * uL + vL * vL + wL * wL);
  const double HR = aR * aR / (gamma - 1.0) + 0.5 * (uR * uR + vR * vR + wR * wR);
  const double RT = std::sqrt(rhoR / rhoL);
  const double rho = RT * rhoL, u = (uL + RT * uR) / (1.0 + RT), v = (vL + RT * vR) / (1.0 + RT),
               w = (wL + RT * wR) / (1.0 + RT), H = (HL + RT * HR) / (1.0 + RT);
  const double a = std::sqrt((gamma - 1.0) * (H - 0.5 * (u * u + v * v + w * w)));
  const double qn = u * nx + v * ny + w * nz;
  const double drho = rhoR - rhoL, dp = pR - pL, dqn = qnR - qnL;
  const double LdU[4] = {(dp - rho * a * dqn) / (2.0 * a * a), drho - dp / (a * a), (dp + rho * a * dqn) / (2.0 * a * a), rho};
  double ws[4] = {std::fabs(qn - a), std::fabs(qn), std::fabs(qn + a), std::fabs(qn)};
  if (ws[0] < 0.2) ws[0] = 0.5 * (ws[0] * ws[0] / 0.2 + 0.2);
  if (ws[2] < 0.2) ws[2] = 0.5 * (ws[2] * ws[2] / 0.2 + 0.2);
  const double du = uR - uL, dv = vR - vL, dw = wR - wL;
  const double R[5][4] = {{1.0, 1.0, 1.0, 0.0},
                          {u - a * nx, u, u + a * nx, du - dqn * nx},
                          {v - a * ny, v, v + a * ny, dv - dqn * ny},
                          {w - a * nz, w, w + a * nz, dw - dqn * nz},
                          {H - a * qn, 0.5 * (u * u + v * v + w * w), H + a * qn, u * du + v * dv + w * dw - qn * dqn}};
  const double fL[5] = {rhoL * qnL, rhoL * qnL * uL + pL * nx, rhoL * qnL * vL + pL * ny, rhoL * qnL * wL + pL * nz,
                        rhoL * qnL * HL};
  const double fR[5] = {rhoR * qnR, rhoR * qnR * uR + pR * nx, rhoR * qnR * vR + pR * ny, rhoR * qnR * wR + pR * nz,
                        rhoR * qnR * HR};
  for (int k = 0; k < 5; ++k) {
    const double diss = ws[0] * LdU[0] * R[k][0] + ws[1] * LdU[1] * R[k][1] + ws[2] * LdU[2] * R[k][2] +
                        ws[3] * LdU[3] * R[k][3];
    flux[k] = 0.5 * (fL[k] + fR[k] - diss);
  }
}

// unit vector normal to n with the largest 2D projection (the tangent choice
// of rROE/tROE_RIEMANN_SOLVER, riemann.f90:1000-1030 and 700-725)
static void face_tangent(const double* n, double* l) {
  const double tx = n[1] * n[1] + n[2] * n[2], ty = n[2] * n[2] + n[0] * n[0], tz = n[0] * n[0] + n[1] * n[1];
  if (tx >= ty && tx >= tz) {
    l[0] = 0.0, l[1] = -n[2], l[2] = n[1];
  } else if (ty >= tx && ty >= tz) {
    l[0] = -n[2], l[1] = 0.0, l[2] = n[0];
  } else {
    l[0] = -n[1], l[1] = n[0], l[2] = 0.0;
  }
  const double t = std::sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2]);
  for (int d = 0; d < 3; ++d) l[d] /= t;
}

static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// primitive state, physical flux along n, sound speed and total enthalpy
struct RoeSide {
  double rho, vel[3], p, a, H, f[5];
};
static RoeSide roe_side(double gamma, const double* c, const double* n) {
  RoeSide s;
  s.rho = c[0];
  for (int d = 0; d < 3; ++d) s.vel[d] = c[1 + d] / c[0];
  const double q2 = dot3(s.vel, s.vel);
  s.p = (gamma - 1.0) * (c[4] - 0.5 * s.rho * q2);
  s.a = std::sqrt(gamma * s.p / s.rho);
  s.H = s.a * s.a / (gamma - 1.0) + 0.5 * q2;
  const double qn = dot3(s.vel, n);
  s.f[0] = s.rho * qn;
  for (int d = 0; d < 3; ++d) s.f[1 + d] = s.rho * qn * s.vel[d] + s.p * n[d];
  s.f[4] = s.rho * qn * s.H;
  return s;
}

// Roe-averaged density, velocity, enthalpy and sound speed
struct RoeAvg {
  double rho, vel[3], H, a;
};
static RoeAvg roe_avg(double gamma, const RoeSide& L, const RoeSide& R) {
  RoeAvg m;
  const double RT = std::sqrt(R.rho / L.rho);
  m.rho = RT * L.rho;
  for (int d = 0; d < 3; ++d) m.vel[d] = (L.vel[d] + RT * R.vel[d]) / (1.0 + RT);
  m.H = (L.H + RT * R.H) / (1.0 + RT);
  m.a = std::sqrt((gamma - 1.0) * (m.H - 0.5 * dot3(m.vel, m.vel)));
  return m;
}

static double entropy_fix(double ws) { return ws < 0.2 ? 0.5 * (ws * ws / 0.2 + 0.2) : ws; }

// rROE_RIEMANN_SOLVER (riemann.f90:892-1234): HLL along the velocity-jump
// direction n1, Roe along n2 (in the plane of n and n1, normal to n1), with
// the wave speeds blended by alpha1 = n.n1, alpha2 = n.n2
void rhll(double gamma, const double* cl, const double* cr, const double* n, double* flux) {
  const RoeSide L = roe_side(gamma, cl, n), R = roe_side(gamma, cr, n);
  const double dvel[3] = {R.vel[0] - L.vel[0], R.vel[1] - L.vel[1], R.vel[2] - L.vel[2]};
  const double adq = std::sqrt(dot3(dvel, dvel));
  double n1[3], n2[3];
  if (adq > 1.0e-13) {
    for (int d = 0; d < 3; ++d) n1[d] = dvel[d] / adq;
  } else {
    face_tangent(n, n1);
  }
  double alpha1 = dot3(n, n1);
  if (alpha1 < 0.0 || (alpha1 == 0.0 && std::signbit(alpha1))) {
    for (int d = 0; d < 3; ++d) n1[d] = -n1[d];
    alpha1 = -alpha1;
  }
  const double t[3] = {n1[1] * n[2] - n1[2] * n[1], n1[2] * n[0] - n1[0] * n[2], n1[0] * n[1] - n1[1] * n[0]};
  n2[0] = t[1] * n1[2] - t[2] * n1[1];
  n2[1] = t[2] * n1[0] - t[0] * n1[2];
  n2[2] = t[0] * n1[1] - t[1] * n1[0];
  const double ln2 = std::sqrt(dot3(n2, n2));
  if (ln2 > 0.0) {
    for (int d = 0; d < 3; ++d) n2[d] /= ln2;
  } else {  // n1 parallel to n (alpha2 = 0): the flux does not depend on n2
    face_tangent(n, n2);
  }
  double alpha2 = dot3(n, n2);
  if (alpha2 < 0.0 || (alpha2 == 0.0 && std::signbit(alpha2))) {
    for (int d = 0; d < 3; ++d) n2[d] = -n2[d];
    alpha2 = -alpha2;
  }
  const RoeAvg m = roe_avg(gamma, L, R);
  const double q1 = dot3(m.vel, n1);
  const double SLm = std::min(std::min(0.0, q1 - m.a), dot3(L.vel, n1) - L.a);
  const double SRp = std::max(std::max(0.0, q1 + m.a), dot3(R.vel, n1) + R.a);
  const double qn = dot3(m.vel, n2), dqn = dot3(R.vel, n2) - dot3(L.vel, n2);
  const double drho = R.rho - L.rho, dp = R.p - L.p, a = m.a;
  const double LdU[4] = {(dp - m.rho * a * dqn) / (2.0 * a * a), drho - dp / (a * a),
                         (dp + m.rho * a * dqn) / (2.0 * a * a), m.rho};
  const double eig[4] = {qn - a, qn, qn + a, qn};
  double ws[4] = {entropy_fix(std::fabs(qn - a)), std::fabs(qn), entropy_fix(std::fabs(qn + a)), std::fabs(qn)};
  for (int k = 0; k < 4; ++k)
    ws[k] = alpha2 * ws[k] - (alpha1 * 2.0 * SRp * SLm + alpha2 * (SRp + SLm) * eig[k]) / (SRp - SLm);
  const double u = m.vel[0], v = m.vel[1], w = m.vel[2];
  const double R4[5] = {0.0, dvel[0] - dqn * n2[0], dvel[1] - dqn * n2[1], dvel[2] - dqn * n2[2],
                        dot3(m.vel, dvel) - qn * dqn};
  const double Rv[5][4] = {{1.0, 1.0, 1.0, R4[0]},
                           {u - a * n2[0], u, u + a * n2[0], R4[1]},
                           {v - a * n2[1], v, v + a * n2[1], R4[2]},
                           {w - a * n2[2], w, w + a * n2[2], R4[3]},
                           {m.H - a * qn, 0.5 * dot3(m.vel, m.vel), m.H + a * qn, R4[4]}};
  for (int k = 0; k < 5; ++k) {
    double diss = 0.0;
    for (int j = 0; j < 4; ++j) diss += ws[j] * LdU[j] * Rv[k][j];
    flux[k] = (SRp * L.f[k] - SLm * R.f[k]) / (SRp - SLm) - 0.5 * diss;
  }
}

// tROE_RIEMANN_SOLVER (riemann.f90:634-890): Roe with the shear waves along
// the face tangents l (face_tangent) and m = n x l
void troe(double gamma, const double* cl, const double* cr, const double* n, double* flux) {
  double l[3], mt[3];
  face_tangent(n, l);
  mt[0] = n[1] * l[2] - n[2] * l[1];
  mt[1] = n[2] * l[0] - n[0] * l[2];
  mt[2] = n[0] * l[1] - n[1] * l[0];
  const double lm = std::sqrt(dot3(mt, mt));
  for (int d = 0; d < 3; ++d) mt[d] /= lm;
  const RoeSide L = roe_side(gamma, cl, n), R = roe_side(gamma, cr, n);
  const RoeAvg m = roe_avg(gamma, L, R);
  const double a = m.a, qn = dot3(m.vel, n), ql = dot3(m.vel, l), qm = dot3(m.vel, mt);
  const double dvel[3] = {R.vel[0] - L.vel[0], R.vel[1] - L.vel[1], R.vel[2] - L.vel[2]};
  const double drho = R.rho - L.rho, dp = R.p - L.p, dqn = dot3(dvel, n);
  const double LdU[5] = {(dp - m.rho * a * dqn) / (2.0 * a * a), drho - dp / (a * a),
                         (dp + m.rho * a * dqn) / (2.0 * a * a), m.rho * dot3(dvel, l), m.rho * dot3(dvel, mt)};
  const double ws[5] = {entropy_fix(std::fabs(qn - a)), std::fabs(qn), entropy_fix(std::fabs(qn + a)), std::fabs(qn),
                        std::fabs(qn)};
  const double u = m.vel[0], v = m.vel[1], w = m.vel[2];
  const double Rv[5][5] = {{1.0, 1.0, 1.0, 0.0, 0.0},
                           {u - a * n[0], u, u + a * n[0], l[0], mt[0]},
                           {v - a * n[1], v, v + a * n[1], l[1], mt[1]},
                           {w - a * n[2], w, w + a * n[2], l[2], mt[2]},
                           {m.H - a * qn, 0.5 * dot3(m.vel, m.vel), m.H + a * qn, ql, qm}};
  for (int k = 0; k < 5; ++k) {
    double diss = 0.0;
    for (int j = 0; j < 5; ++j) diss += ws[j] * LdU[j] * Rv[k][j];
    flux[k] = 0.5 * (L.f[k] + R.f[k] - diss);
  }
}

void riemann(const ucg_config* cfg, const double* cl, const double* cr, double* flux) {
  if (cfg->riemann == 2) rusanov(cfg->gamma, cl, cr, flux);
  else if (cfg->riemann == 9) hll(cfg->gamma, cl, cr, flux);
  else hllc(cfg->gamma, cl, cr, flux);
}

// ghost state of a physical boundary face (BOUNDARYS,
// src/flow_operations.f90:2860-3375).  cfg->bc_state holds the free-stream
// primitive state (rho, u, v, w, p) that INFLOW/OUTFLOW return
// (flow_operations.f90:1161, 1526: RRES, uvel, vvel, wvel, PRES).
void prim2cons(double gm, const double* p, double* u) {
  double skin = 0.5 * ((p[1] * p[1]) + (p[2] * p[2]) + (p[3] * p[3]));
  double ie = p[4] / ((gm - 1.0) * p[0]);
  u[0] = p[0];
  u[1] = p[1] * p[0];
  u[2] = p[2] * p[0];
  u[3] = p[3] * p[0];
  u[4] = (p[0] * ie) + (p[0] * skin);
}
// subsonic inflow state of CASE(1) (:2911-2928) and of the CASE(6) inflow
void subsonic_inflow(double gm, const double* s1, const double* s2, double sps, double nx, double ny, double nz,
                     double* cr) {
  double s3[NV];
  s3[4] = 0.5 * ((s1[4]) + (s2[4]) - (s2[0] * sps * ((nx * (s1[1] - s2[1])) + (ny * (s1[2] - s2[2])) + (nz * (s1[3] - s2[3])))));
  s3[0] = s1[0] + (s3[4] - s1[4]) / (sps * sps);
  s3[1] = s1[1] - (nx * (s1[4] - s3[4])) / (sps * s2[0]);
  s3[2] = s1[2] - (ny * (s1[4] - s3[4])) / (sps * s2[0]);
  s3[3] = s1[3] - (nz * (s1[4] - s3[4])) / (sps * s2[0]);
  prim2cons(gm, s3, cr);
}
// subsonic outflow state of CASE(2) (:2997-3010) and of the CASE(6) outflow
void subsonic_outflow(double gm, const double* s1, const double* s2, double sps, double nx, double ny, double nz,
                      double* cr) {
  double s3[NV];
  s3[4] = s1[4];
  s3[0] = s2[0] + (s3[4] - s2[4]) / (sps * sps);
  s3[1] = s2[1] + (nx * (s2[4] - s3[4])) / (sps * s2[0]);
  s3[2] = s2[2] + (ny * (s2[4] - s3[4])) / (sps * s2[0]);
  s3[3] = s2[3] + (nz * (s2[4] - s3[4])) / (sps * s2[0]);
  prim2cons(gm, s3, cr);
}
void boundary_state(const Ctx& x, int code, const double* ang, const double* cl, double* cr) {
  const ucg_config* cfg = x.cfg;
  const double gm = cfg->gamma;
  double nx = ang[0] * ang[3], ny = ang[1] * ang[3], nz = ang[2];
  double s1[NV], s2[NV];
  for (int k = 0; k < NV; ++k) s1[k] = cfg->bc_state[k];
  switch (code) {
    case 1: {  // INFLOW (:2883)
      if (cfg->boundtype == 0) {  // supersonic: the free stream
        prim2cons(gm, s1, cr);
        return;
      }
      cons2prim(x, cl, s2);
      double sps = std::sqrt((gm * s2[4]) / (s2[0]));
      double vel = std::sqrt(s2[1] * s2[1] + s2[2] * s2[2] + s2[3] * s2[3]);
      if (vel / (sps + TOLSMALL) > 1.0) prim2cons(gm, s1, cr);
      else subsonic_inflow(gm, s1, s2, sps, nx, ny, nz, cr);
      return;
    }
    case 2: {  // OUTFLOW (:2972)
      if (cfg->boundtype == 0) {  // supersonic: the cell's own state
        for (int k = 0; k < NV; ++k) cr[k] = cl[k];
        return;
      }
      cons2prim(x, cl, s2);
      double sps = std::sqrt((gm * s2[4]) / (s2[0]));
      double vel = std::sqrt(s2[1] * s2[1] + s2[2] * s2[2] + s2[3] * s2[3]);
      if (vel / (sps + TOLSMALL) > 1.0) {
        for (int k = 0; k < NV; ++k) cr[k] = cl[k];
      } else {
        subsonic_outflow(gm, s1, s2, sps, nx, ny, nz, cr);
      }
      return;
    }
    case 4:  // WALL (:3140)
      if (cfg->governing == 1) {  // ITESTCASE 4 (:3172-3186): no slip, the whole momentum mirrored
        cr[0] = cl[0];
        cr[1] = -cl[1];
        cr[2] = -cl[2];
        cr[3] = -cl[3];
        cr[4] = cl[4];
        return;
      }
      [[fallthrough]];
    case 3: {  // SYMMETRY (:3102), and the ITESTCASE 3 wall: the face-frame normal momentum mirrored
      double rl[NV], rr[NV];
      rotf(ang, cl, rl);
      rr[0] = rl[0];
      rr[1] = -rl[1];
      rr[2] = rl[2];
      rr[3] = rl[3];
      rr[4] = rl[4];
      rotb(ang, rr, cr);
      return;
    }
    case 6: {  // FARFIELD (:3230): direction from vnb = the rotated conserved
               // normal momentum, supersonic when |vnb| >= the sound speed
      double rl[NV];
      rotf(ang, cl, rl);
      const double vnb = rl[1];
      cons2prim(x, cl, s2);
      double sps = std::sqrt((gm * s2[4]) / (s2[0]));
      if (vnb <= 0.0) {
        if (std::fabs(vnb) >= sps) prim2cons(gm, s1, cr);
        else subsonic_inflow(gm, s1, s2, sps, nx, ny, nz, cr);
      } else {
        if (std::fabs(vnb) >= sps) {
          for (int k = 0; k < NV; ++k) cr[k] = cl[k];
        } else {
          subsonic_outflow(gm, s1, s2, sps, nx, ny, nz, cr);
        }
      }
      return;
    }
    default: {  // no other code reaches the residual (the engine rejects them)
      const double nan = std::nan("");
      for (int k = 0; k < NV; ++k) cr[k] = nan;
      return;
    }
  }
}

// COMPUTE_EIGENVECTORS (flow_operations.f90:3934-3995): left (EL) and right
// (ER) eigenvectors of the x-direction Euler flux Jacobian at the arithmetic
// average of two face-frame states (density, velocity, total energy).
void eigenvectors(double gamma, const double* rl, const double* rr, double EL[5][5], double ER[5][5]) {
  const double gm1 = gamma - 1.0, oo2 = 0.5;
  const double oor1 = 1.0 / rl[0], oor2 = 1.0 / rr[0];
  const double rs = oo2 * (rl[0] + rr[0]);
  const double us = oo2 * ((rl[1] * oor1) + (rr[1] * oor2));
  const double vs = oo2 * ((rl[2] * oor1) + (rr[2] * oor2));
  const double ws = oo2 * ((rl[3] * oor1) + (rr[3] * oor2));
  const double es = oo2 * (rl[4] + rr[4]);
  const double vvs = us * us + vs * vs + ws * ws;
  const double vsd = oo2 * vvs;
  const double ps = gm1 * (es - oo2 * rs * vvs);
  const double as = std::sqrt(gamma * ps / rs);
  const double hs = (oo2 * vvs) + ((as * as) / gm1);
  const double R[5][5] = {{1.0, 1.0, 0.0, 0.0, 1.0},
                          {us - as, us, 0.0, 0.0, us + as},
                          {vs, vs, 1.0, 0.0, vs},
                          {ws, ws, 0.0, 1.0, ws},
                          {hs - us * as, oo2 * vvs, vs, ws, hs + us * as}};
  const double den = 2.0 * as * hs - 2.0 * as * vsd;
  const double us2 = us * us, vs2 = vs * vs, ws2 = ws * ws;
  double L[5][5];
  L[0][0] = (hs * us + as * us2 + as * vs2 - as * vsd - us * vsd + as * ws2) / den;
  L[0][1] = (-hs - as * us + vsd) / den;
  L[0][2] = -((as * vs) / den);
  L[0][3] = -((as * ws) / den);
  L[0][4] = as / den;
  L[1][0] = (2.0 * as * hs - 2.0 * as * us2 - 2.0 * as * vs2 - 2.0 * as * ws2) / den;
  L[1][1] = (2.0 * as * us) / den;
  L[1][2] = (2.0 * as * vs) / den;
  L[1][3] = (2.0 * as * ws) / den;
  L[1][4] = (-2.0 * as) / den;
  L[2][0] = (-2.0 * as * hs * vs + 2.0 * as * vs * vsd) / den;
  L[2][1] = 0.0;
  L[2][2] = 1.0;
  L[2][3] = 0.0;
  L[2][4] = 0.0;
  L[3][0] = (-2.0 * as * hs * ws + 2.0 * as * vsd * ws) / den;
  L[3][1] = 0.0;
  L[3][2] = 0.0;
  L[3][3] = 1.0;
  L[3][4] = 0.0;
  L[4][0] = (-(hs * us) + as * us2 + as * vs2 - as * vsd + us * vsd + as * ws2) / den;
  L[4][1] = (hs - as * us - vsd) / den;
  L[4][2] = -((as * vs) / den);
  L[4][3] = -((as * ws) / den);
  L[4][4] = as / den;
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) {
      EL[i][j] = L[i][j];
      ER[i][j] = R[i][j];
    }
}

// CHARACTERISTIC_RECONSTRUCTION (reconstruct_p.f90:497-758), per face L of
// cell c: eigenvectors from the cell mean and the face neighbour's mean (or
// the boundary ghost of the cell mean, WENO_NEIGHBOUR :761-917), both rotated
// into the face frame; the stencil polynomials (with the mean as row 0)
// projected on the left eigenvectors, W = gradients * EL^T (the projected
// quantities are the global-frame conserved variables, as in the
// reference); smoothness indicators diag(W^T S W) (diag_At_B_A); weights per
// characteristic variable; LIMITEDDW = sum_ll W_ll * w_ll; back-projection
// FINDW = ER * LIMITEDDW; face values FINDW(:,0) + basis . FINDW(:,1:).
// CWENO (EES 5): the central polynomial has the lower-order stencils
// removed, and the lower-order stencils use INDICATORC over IDEGFREE2
// (compute_gradcharv_smoothindicator :1723-1760).
void char_faces(const Ctx& x, int64_t c, const double* U, const double* G, double* ul) {
  const ucg_config* cfg = x.cfg;
  const ucg_geometry* g = x.g;
  const ucg_recon* r = x.r;
  const int ideg = cfg->ideg, ideg2 = cfg->ideg2;
  const int t = tab(x, c);
  const int admis = g->admis[c];
  const bool cw = cfg->ees == 5;
  const double* u0 = U + c * NV;
  // gradients[ll][d][v], d = 0 the cell mean
  std::vector<double> gr((size_t)admis * (ideg + 1) * NV, 0.0);
  auto GR = [&](int ll, int d, int v) -> double& { return gr[((size_t)ll * (ideg + 1) + d) * NV + v]; };
  std::vector<double> lam(admis, 1.0);
  for (int ll = 0; ll < admis; ++ll)
    for (int v = 0; v < NV; ++v) GR(ll, 0, v) = u0[v];
  if (cw) {
    lam[0] = 1.0 - 1.0 / cfg->lwci;
    for (int ll = 1; ll < admis; ++ll) lam[ll] = (1.0 - lam[0]) / (admis - 1);
    std::vector<double> g5((size_t)ideg * NV, 0.0);
    for (int ll = 1; ll < admis; ++ll)
      for (int d = 0; d < ideg2; ++d)
        for (int v = 0; v < NV; ++v) {
          g5[d * NV + v] = g5[d * NV + v] + lam[ll] * G[((size_t)ll * ideg + d) * NV + v];
          GR(ll, d + 1, v) = G[((size_t)ll * ideg + d) * NV + v];
        }
    for (int d = 0; d < ideg; ++d)
      for (int v = 0; v < NV; ++v) GR(0, d + 1, v) = (1.0 / lam[0]) * (G[(size_t)d * NV + v] - g5[d * NV + v]);
  } else {
    lam[0] = cfg->lwci;
    for (int ll = 0; ll < admis; ++ll)
      for (int d = 0; d < ideg; ++d)
        for (int v = 0; v < NV; ++v) GR(ll, d + 1, v) = G[((size_t)ll * ideg + d) * NV + v];
  }
  const double* S = &r->indicator[(int64_t)t * ideg * ideg];
  const double* S2 = cw ? &r->indicator2[(int64_t)t * ideg2 * ideg2] : nullptr;
  std::vector<double> W((size_t)admis * (ideg + 1) * NV), b(ideg);
  for (int f = 0; f < g->nfaces[c]; ++f) {
    const double a1 = g->face_angle[(c * F + f) * 2], a2 = g->face_angle[(c * F + f) * 2 + 1];
    const double ang[4] = {std::cos(a1), std::sin(a1), std::cos(a2), std::sin(a2)};
    double ur[NV], rvl[NV], rvr[NV];
    const int64_t nb = g->neigh[c * F + f];
    if (nb >= 0) {
      for (int v = 0; v < NV; ++v) ur[v] = U[nb * NV + v];
    } else {
      boundary_state(x, g->bc[c * F + f], ang, u0, ur);
    }
    rotf(ang, u0, rvl);
    rotf(ang, ur, rvr);
    double EL[5][5], ER[5][5];
    eigenvectors(cfg->gamma, rvl, rvr, EL, ER);
    // W[ll][d][k] = sum_v gradients[ll][d][v] * EL[k][v]
    for (int ll = 0; ll < admis; ++ll) {
      const int nd = (cw && ll > 0) ? ideg2 : ideg;
      for (int d = 0; d <= nd; ++d)
        for (int k = 0; k < NV; ++k) {
          double s = 0.0;
          for (int v = 0; v < NV; ++v) s += GR(ll, d, v) * EL[k][v];
          W[((size_t)ll * (ideg + 1) + d) * NV + k] = s;
        }
    }
    auto Wv = [&](int ll, int d, int k) { return W[((size_t)ll * (ideg + 1) + d) * NV + k]; };
    // smoothness indicators and weights per characteristic variable
    std::vector<double> w((size_t)admis * NV);
    for (int k = 0; k < NV; ++k) {
      std::vector<double> is(admis), wt(admis);
      for (int ll = 0; ll < admis; ++ll) {
        const bool low = cw && ll > 0;
        const int nd = low ? ideg2 : ideg;
        const double* B = low ? S2 : S;
        double acc = 0.0;
        for (int i = 0; i < nd; ++i) {
          double ba = 0.0;
          for (int j = 0; j < nd; ++j) ba += B[i * nd + j] * Wv(ll, j + 1, k);
          acc += Wv(ll, i + 1, k) * ba;
        }
        is[ll] = acc;
      }
      const double eps = cfg->weno_eps;
      if (cw && cfg->wenoz) {
        double tau = 0.0;
        for (int ll = 0; ll < admis; ++ll) tau = tau + std::fabs(is[0] - is[ll]);
        tau = tau / (admis - 1);
        for (int ll = 0; ll < admis; ++ll) wt[ll] = lam[ll] * (1.0 + std::pow(tau / (eps + is[ll]), 4));
      } else {
        for (int ll = 0; ll < admis; ++ll) wt[ll] = lam[ll] / std::pow(eps + is[ll], 4);
      }
      double sum = 0.0;
      for (int ll = 0; ll < admis; ++ll) sum = sum + wt[ll];
      for (int ll = 0; ll < admis; ++ll) w[(size_t)ll * NV + k] = wt[ll] / sum;
    }
    // LIMITEDDW and its back-projection FINDW[d][v]
    std::vector<double> fw((size_t)(ideg + 1) * NV);
    for (int d = 0; d <= ideg; ++d) {
      double lim[NV] = {0, 0, 0, 0, 0};
      for (int ll = 0; ll < admis; ++ll) {
        const int nd = (cw && ll > 0) ? ideg2 : ideg;
        if (d > nd) continue;
        for (int k = 0; k < NV; ++k) lim[k] = lim[k] + Wv(ll, d, k) * w[(size_t)ll * NV + k];
      }
      for (int v = 0; v < NV; ++v) {
        double s = 0.0;
        for (int k = 0; k < NV; ++k) s += ER[v][k] * lim[k];
        fw[(size_t)d * NV + v] = s;
      }
    }
    for (int q = 0; q < nq_of(x, c, f); ++q) {
      basis(x, c, &g->qpoints[((c * F + f) * Q + q) * 3], ideg, b.data());
      for (int v = 0; v < NV; ++v) {
        double res = 0.0;
        for (int d = 0; d < ideg; ++d) res += b[d] * fw[(size_t)(d + 1) * NV + v];
        ul[(f * Q + q) * NV + v] = fw[v] + res;
      }
    }
  }
}

void sutherland(const ucg_config* cfg, double rho, double p, double* mu, double* lam) {
  double t1 = p / (rho * cfg->r_gas);
  double t0 = cfg->pres / (cfg->rres * cfg->r_gas);
  const double betaas = 1.5, suther = 0.412158681;  // parameters.f90:1220-1221
  *mu = cfg->visc * std::pow(t1 / t0, betaas) * ((t0 + (suther * t0)) / (t1 + (suther * t0)));
  *lam = (*mu) * cfg->r_gas * cfg->gamma / (cfg->prandtl * (cfg->gamma - 1.0));
}

// CALL_FLUX_SUBROUTINES_3D: rhs [n][5]
// RHS(I) of one cell from the face values UL (and ULV for Navier-Stokes):
// CALCULATE_FLUXESHI_CONVECTIVE, flux_p.f90:478-1030, and the diffusive
// fluxes of CALCULATE_FLUXESHI_DIFFUSIVE, flux_p.f90:1520-2107
void cell_rhs(const Ctx& x, int64_t c, const std::vector<double>& UL, const std::vector<double>& ULV, double* out) {
  const bool ns = x.cfg->governing == 1;
  const ucg_geometry* g = x.g;
  {
    double R[NV] = {0, 0, 0, 0, 0};
    // convective
    for (int f = 0; f < g->nfaces[c]; ++f) {
      double a1 = g->face_angle[(c * F + f) * 2], a2 = g->face_angle[(c * F + f) * 2 + 1];
      double ang[4] = {std::cos(a1), std::sin(a1), std::cos(a2), std::sin(a2)};
      double god[NV] = {0, 0, 0, 0, 0};
      int64_t nb = g->neigh[c * F + f];
      int nf = g->neigh_face[c * F + f];
      for (int q = 0; q < nq_of(x, c, f); ++q) {
        const double* cl = &UL[(((size_t)c * F + f) * Q + q) * NV];
        double crb[NV];
        const double* cr;
        if (nb >= 0) {
          int qq = g->qperm[(c * F + f) * Q + q];
          cr = &UL[(((size_t)nb * F + nf) * Q + qq) * NV];
        } else {
          boundary_state(x, g->bc[c * F + f], ang, cl, crb);
          cr = crb;
        }
        double clr[NV], crr[NV], hf[NV], fl[NV];
        if (x.cfg->riemann >= 3 && x.cfg->riemann <= 5) {  // Roe family: global frame, face normal
          const double nrm[3] = {ang[0] * ang[3], ang[1] * ang[3], ang[2]};
          if (x.cfg->riemann == 3) roe(x.cfg->gamma, cl, cr, nrm, fl);
          else if (x.cfg->riemann == 4) rhll(x.cfg->gamma, cl, cr, nrm, fl);
          else troe(x.cfg->gamma, cl, cr, nrm, fl);
        } else {
          rotf(ang, cr, crr);
          rotf(ang, cl, clr);
          riemann(x.cfg, clr, crr, hf);
          rotb(ang, hf, fl);
        }
        double ws = wq_of(x, c, f, q) * g->face_area[c * F + f];
        for (int v = 0; v < NV; ++v) god[v] = god[v] + (fl[v] * ws);
      }
      for (int v = 0; v < NV; ++v) R[v] = R[v] + god[v];
    }
    // diffusive
    if (ns) {
      const ucg_config* cfg = x.cfg;
      for (int f = 0; f < g->nfaces[c]; ++f) {
        double a1 = g->face_angle[(c * F + f) * 2], a2 = g->face_angle[(c * F + f) * 2 + 1];
        double nx = std::cos(a1) * std::sin(a2), ny = std::sin(a1) * std::sin(a2), nz = std::cos(a2);
        double nn[3] = {nx, ny, nz};
        double god[NV] = {0, 0, 0, 0, 0};
        int64_t nb = g->neigh[c * F + f];
        int nf = g->neigh_face[c * F + f];
        for (int q = 0; q < nq_of(x, c, f); ++q) {
          const double* cl = &UL[(((size_t)c * F + f) * Q + q) * NV];
          const double* gl = &ULV[(((size_t)c * F + f) * Q + q) * 12];
          const double* cr;
          const double* gr;
          double crb[NV];
          double damp = cfg->lamx, vdamp = 4.0 / 3.0;
          if (nb >= 0) {
            int qq = g->qperm[(c * F + f) * Q + q];
            cr = &UL[(((size_t)nb * F + nf) * Q + qq) * NV];
            gr = &ULV[(((size_t)nb * F + nf) * Q + qq) * 12];
          } else {
            // CALCULATE_BOUNDED_VISCOUS (dg_functions.f90:1179-1300): the
            // ghost state of BOUNDARYS and the cell's own gradients on the
            // ghost side; codes 1-4 drop the jump term (flux_p.f90:1872-1874)
            const double ang[4] = {std::cos(a1), std::sin(a1), std::cos(a2), std::sin(a2)};
            const int code = g->bc[c * F + f];
            boundary_state(x, code, ang, cl, crb);
            cr = crb;
            gr = gl;
            if (code > 0 && code < 5) damp = 0.0;
          }
          double lv[NV], rv[NV];
          cons2prim(x, cl, lv);
          cons2prim(x, cr, rv);
          double mul, mur, laml, lamr;
          sutherland(cfg, lv[0], lv[4], &mul, &laml);
          sutherland(cfg, rv[0], rv[4], &mur, &lamr);
          // LCVGRAD rows: u, v, w, T (ULEFTV components 2,3,4,1)
          double lg[4][3], rg[4][3];
          for (int k = 0; k < 3; ++k) {
            lg[0][k] = gl[1 * 3 + k]; lg[1][k] = gl[2 * 3 + k]; lg[2][k] = gl[3 * 3 + k]; lg[3][k] = gl[0 * 3 + k];
            rg[0][k] = gr[1 * 3 + k]; rg[1][k] = gr[2 * 3 + k]; rg[2][k] = gr[3 * 3 + k]; rg[3][k] = gr[0 * 3 + k];
          }
          double dih = std::fabs(g->dih[c * F + f]);
          double jump[4] = {rv[1] - lv[1], rv[2] - lv[2], rv[3] - lv[3],
                            (rv[4] / (rv[0] * cfg->r_gas)) - (lv[4] / (lv[0] * cfg->r_gas))};
          double gg[4][3];
          for (int a = 0; a < 4; ++a)
            for (int k = 0; k < 3; ++k) gg[a][k] = ((lg[a][k] + rg[a][k]) / 2.0) + damp * ((vdamp / dih) * nn[k] * jump[a]);
          double fxv[5] = {0, 0, 0, 0, 0}, fyv[5] = {0, 0, 0, 0, 0}, fzv[5] = {0, 0, 0, 0, 0};
          double qh[3];
          for (int k = 0; k < 3; ++k) qh[k] = -0.5 * ((laml + lamr) * gg[3][k]);
          fxv[4] = fxv[4] - qh[0];
          fyv[4] = fyv[4] - qh[1];
          fzv[4] = fzv[4] - qh[2];
          double ux = gg[0][0], uy = gg[0][1], uz = gg[0][2];
          double vx = gg[1][0], vy = gg[1][1], vz = gg[1][2];
          double wx = gg[2][0], wy = gg[2][1], wz = gg[2][2];
          double tl[3][3];
          tl[0][0] = (4.0 / 3.0) * ux - (2.0 / 3.0) * vy - (2.0 / 3.0) * wz;
          tl[1][1] = (4.0 / 3.0) * vy - (2.0 / 3.0) * ux - (2.0 / 3.0) * wz;
          tl[2][2] = (4.0 / 3.0) * wz - (2.0 / 3.0) * ux - (2.0 / 3.0) * vy;
          tl[0][1] = tl[1][0] = (uy + vx);
          tl[0][2] = tl[2][0] = (wx + uz);
          tl[1][2] = tl[2][1] = (vz + wy);
          double mu2 = 0.5 * (mul + mur);
          double tau[3][3];
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) tau[a][b] = mu2 * tl[a][b];
          for (int k = 1; k <= 3; ++k) {
            fxv[k] = fxv[k] + tau[0][k - 1];
            fyv[k] = fyv[k] + tau[1][k - 1];
            fzv[k] = fzv[k] + tau[2][k - 1];
          }
          double rho12 = 0.5 * (cl[0] + cr[0]);
          double u12 = 0.5 * (cl[1] + cr[1]) / rho12, v12 = 0.5 * (cl[2] + cr[2]) / rho12, w12 = 0.5 * (cl[3] + cr[3]) / rho12;
          fxv[4] = fxv[4] + u12 * tau[0][0] + v12 * tau[0][1] + w12 * tau[0][2];
          fyv[4] = fyv[4] + u12 * tau[1][0] + v12 * tau[1][1] + w12 * tau[1][2];
          fzv[4] = fzv[4] + u12 * tau[2][0] + v12 * tau[2][1] + w12 * tau[2][2];
          double ws = wq_of(x, c, f, q) * g->face_area[c * F + f];
          for (int v = 0; v < NV; ++v) god[v] = god[v] + ((nx * fxv[v] + ny * fyv[v] + nz * fzv[v]) * ws);
        }
        for (int v = 0; v < NV; ++v) R[v] = R[v] - god[v];
      }
    }
    for (int v = 0; v < NV; ++v) out[v] = R[v];
  }
}

void residual(const Ctx& x, const double* U, double* rhs, std::vector<double>& UL, std::vector<double>& ULV) {
  const int64_t n = x.n;
  const bool ns = x.cfg->governing == 1;
  UL.assign((size_t)n * F * Q * NV, 0.0);
  if (ns) ULV.assign((size_t)n * F * Q * 12, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t c = 0; c < n; ++c) reconstruct_cell(x, c, U, &UL[(size_t)c * F * Q * NV], ns ? &ULV[(size_t)c * F * Q * 12] : nullptr);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t c = 0; c < n; ++c) cell_rhs(x, c, UL, ULV, &rhs[c * NV]);
}

// PAD_NAD (mood.f90:35-330): PAD if the candidate Uk's density or pressure is
// not positive (or NaN); else NAD if its density or total energy (variables 1
// and 5) leaves [min, max] of the stage input Uc over the cell and its face
// neighbours through interior and periodic faces, widened in the relaxed
// mode (MOOD_MODE > 0) by NAD_DELTA = max(d1, d2 * (max - min)).
void pad_nad(const Ctx& x, const double* Uc, const double* Uk, double d1, double d2, std::vector<int8_t>& mood) {
  const ucg_geometry* g = x.g;
  mood.assign(x.n, 0);
  for (int64_t c = 0; c < x.n; ++c) {
    double pr[NV];
    cons2prim(x, &Uk[c * NV], pr);
    bool pad = !(pr[0] > 0.0) || !(pr[4] > 0.0);
    bool nad = false;
    if (!pad) {
      double umin[NV], umax[NV];
      for (int v = 0; v < NV; ++v) umin[v] = umax[v] = Uc[c * NV + v];
      for (int f = 0; f < g->nfaces[c]; ++f) {
        const int64_t nb = g->neigh[c * F + f];
        if (nb < 0) continue;
        for (int v = 0; v < NV; ++v) {
          umin[v] = std::min(umin[v], Uc[nb * NV + v]);
          umax[v] = std::max(umax[v], Uc[nb * NV + v]);
        }
      }
      for (int v : {0, NV - 1}) {
        const double u = Uk[c * NV + v];
        if (x.cfg->mood_mode > 0) {
          const double delta = std::max(d1, d2 * (umax[v] - umin[v]));
          if (u < umin[v] - delta || u > umax[v] + delta) nad = true;
        } else {
          if (u < umin[v] || u > umax[v]) nad = true;
        }
      }
    }
    mood[c] = (pad || nad) ? 1 : 0;
  }
}

// FIX_LIST (mood.f90:440-518): the flagged cells and their face neighbours
void fix_list(const Ctx& x, const std::vector<int8_t>& mood, std::vector<int8_t>& recalc) {
  const ucg_geometry* g = x.g;
  recalc.assign(x.n, 0);
  for (int64_t c = 0; c < x.n; ++c) {
    bool s = mood[c] != 0;
    for (int f = 0; f < g->nfaces[c]; ++f) {
      const int64_t nb = g->neigh[c * F + f];
      if (nb >= 0 && mood[nb]) s = true;
    }
    recalc[c] = s ? 1 : 0;
  }
}

// One stage of RUNGE_KUTTA3_MOOD (time_p.f90:582-880), Euler: stage s (1-3)
// from the stage input Uc and the step base Un into Uo, RECALC in/out.
// The candidate from the reconstruction under the last RECALC; then
// MOOD_OPERATOR_2 (MOOD_VAR1/2): PAD_NAD, FIX_LIST, MUSCL (no CHECKSOLX) on
// the selected reduced cells, their residual and stage redone; then
// MOOD_OPERATOR_1 (MOOD_VAR3/4): PAD_NAD, FIX_LIST, the flagged cells' face
// values their stage-input mean (CASCADE 2 of
// CALCULATE_FLUXESHI_CONVECTIVE_MOOD, flux_p.f90:2722-2733), the selected
// cells' residual and stage redone.  order: MOOD_O.
void mood_stage(const Ctx& x, int s, double dt, const double* Uc, const double* Un, double* Uo,
                std::vector<int8_t>& recalc, int32_t* order) {
  const int64_t n = x.n;
  const ucg_geometry* g = x.g;
  const int ideg = x.cfg->ideg;
  std::vector<double> UL((size_t)n * F * Q * NV, 0.0), ULV, G0((size_t)n * ideg * NV), R((size_t)n * NV),
      Uk((size_t)n * NV);
  std::vector<int8_t> red(n);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t c = 0; c < n; ++c)
    reconstruct_cell(x, c, Uc, &UL[(size_t)c * F * Q * NV], nullptr, recalc.data(), &red[c], &G0[(size_t)c * ideg * NV]);
  const double a[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0}, b[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0}, k[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
  const int si = s - 1;
  auto stage = [&](int64_t c, double* out) {
    double rr[NV];
    cell_rhs(x, c, UL, ULV, rr);
    const double oov = 1.0 / g->volume[c];
    for (int v = 0; v < NV; ++v) {
      const double d = dt * (rr[v] * oov);
      out[v] = si == 0 ? Un[c * NV + v] - d : (a[si] * Un[c * NV + v]) + (b[si] * Uc[c * NV + v]) - (k[si] * d);
    }
  };
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t c = 0; c < n; ++c) stage(c, &Uk[c * NV]);
  // first cascade
  std::vector<int8_t> m1, s1, m2, s2;
  pad_nad(x, Uc, Uk.data(), x.cfg->mood_var[0], x.cfg->mood_var[1], m1);
  fix_list(x, m1, s1);
  for (int64_t c = 0; c < n; ++c)
    if (s1[c] && red[c]) muscl_cell(x, c, Uc, &G0[(size_t)c * ideg * NV], &UL[(size_t)c * F * Q * NV]);
  std::vector<double> Uk2(Uk);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t c = 0; c < n; ++c)
    if (s1[c]) stage(c, &Uk2[c * NV]);
  // second cascade
  pad_nad(x, Uc, Uk2.data(), x.cfg->mood_var[2], x.cfg->mood_var[3], m2);
  fix_list(x, m2, s2);
  for (int64_t c = 0; c < n; ++c)
    if (m2[c])
      for (int i = 0; i < F * Q; ++i)
        for (int v = 0; v < NV; ++v) UL[((size_t)c * F * Q + i) * NV + v] = Uc[c * NV + v];
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t c = 0; c < n; ++c) {
    if (s2[c]) stage(c, &Uo[c * NV]);
    else
      for (int v = 0; v < NV; ++v) Uo[c * NV + v] = Uk2[c * NV + v];
    if (order) order[c] = s2[c] ? 1 : s1[c] ? 2 : x.cfg->iorder + 1;
  }
  recalc = s2;
}

bool check_ctx(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r) {
  if (!cfg || !g || !r) return false;
  if (r->first != 0 || r->count != g->ncells) return false;
  return true;
}

}  // namespace

extern "C" {

// One CALL_FLUX_SUBROUTINES_3D: RHS(I)%VAL for every cell.
int orc_residual(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r, const double* U, double* rhs) {
  if (!check_ctx(cfg, g, r) || !U || !rhs) return UCG_EINVAL;
  Ctx x{cfg, g, r, g->ncells, monos(cfg->iorder)};
  std::vector<double> UL, ULV;
  residual(x, U, rhs, UL, ULV);
  return UCG_OK;
}

// Face values ULEFT [n][F][Q][5] after reconstruction (for kernel-level tests).
int orc_face_values(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r, const double* U, double* ul) {
  if (!check_ctx(cfg, g, r) || !U || !ul) return UCG_EINVAL;
  Ctx x{cfg, g, r, g->ncells, monos(cfg->iorder)};
  const bool ns = cfg->governing == 1;
  std::vector<double> tmp;
#pragma omp parallel for schedule(dynamic, 64) private(tmp)
  for (int64_t c = 0; c < g->ncells; ++c) {
    tmp.assign(ns ? F * Q * 12 : 1, 0.0);
    for (int i = 0; i < F * Q * NV; ++i) ul[(size_t)c * F * Q * NV + i] = 0.0;
    reconstruct_cell(x, c, U, &ul[(size_t)c * F * Q * NV], ns ? tmp.data() : nullptr);
  }
  return UCG_OK;
}

// CALCULATE_CFL (time_p.f90:27-191), CCFL = CFL/3.
int orc_compute_dt(const ucg_config* cfg, const ucg_geometry* g, const double* U, double cfl, double* dt) {
  if (!cfg || !g || !U || !dt) return UCG_EINVAL;
  double ccfl = cfl / 3.0, best = TOLBIG;
  Ctx x{cfg, g, nullptr, g->ncells, {}};
  for (int64_t c = 0; c < g->ncells; ++c) {
    double p[NV];
    cons2prim(x, &U[c * NV], p);
    double agrt = std::sqrt(p[4] * cfg->gamma / p[0]);
    double veln = std::max(std::max(std::fabs(p[1]), std::fabs(p[2])), std::fabs(p[3])) + agrt;
    double me = g->minedge[c];
    double d;
    if (cfg->governing == 1) {
      double mu, lam;
      sutherland(cfg, p[0], p[4], &mu, &lam);
      d = ccfl * (1.0 / ((std::fabs(veln) / me) + (0.5 * (lam + mu) / (me * me))));
    } else {
      d = ccfl * (me / std::fabs(veln));
    }
    best = std::min(best, d);
  }
  *dt = best;
  return UCG_OK;
}

// RUNGE_KUTTA3 (time_p.f90:885-1027) in place on U [n][5].
int orc_rk3_step(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r, double dt, double* U) {
  if (!check_ctx(cfg, g, r) || !U) return UCG_EINVAL;
  Ctx x{cfg, g, r, g->ncells, monos(cfg->iorder)};
  const int64_t n = g->ncells;
  std::vector<double> U0(U, U + n * NV), U1, rhs(n * NV), UL, ULV;
  const double to4 = 3.0 / 4.0, oo4 = 1.0 / 4.0, to3 = 2.0 / 3.0, oo3 = 1.0 / 3.0;
  residual(x, U, rhs.data(), UL, ULV);
  for (int64_t c = 0; c < n; ++c) {
    double oov = 1.0 / g->volume[c];
    for (int v = 0; v < NV; ++v) U[c * NV + v] = U0[c * NV + v] - (dt * (rhs[c * NV + v] * oov));
  }
  residual(x, U, rhs.data(), UL, ULV);
  for (int64_t c = 0; c < n; ++c) {
    double oov = 1.0 / g->volume[c];
    for (int v = 0; v < NV; ++v) {
      double u3 = U[c * NV + v];
      U[c * NV + v] = (to4 * U0[c * NV + v]) + (oo4 * u3) - ((oo4) * ((dt) * ((rhs[c * NV + v]) * (oov))));
    }
  }
  residual(x, U, rhs.data(), UL, ULV);
  for (int64_t c = 0; c < n; ++c) {
    double oov = 1.0 / g->volume[c];
    for (int v = 0; v < NV; ++v)
      U[c * NV + v] = ((oo3)*U0[c * NV + v]) + ((to3)*U[c * NV + v]) - (((to3)) * ((dt) * ((rhs[c * NV + v]) * (oov))));
  }
  return UCG_OK;
}

// One stage of RUNGE_KUTTA3 (src/time_p.f90:885-1027): stage 1 U = Un -
// dt R(Un)/V (U holds Un on entry), stage 2 U = 3/4 Un + 1/4 U - 1/4 dt R(U)/V,
// stage 3 U = 1/3 Un + 2/3 U - 2/3 dt R(U)/V, in place on U.
int orc_rk3_stage(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r, double dt, int stage,
                  const double* Un, double* U) {
  if (!check_ctx(cfg, g, r) || !U || !Un || stage < 1 || stage > 3) return UCG_EINVAL;
  Ctx x{cfg, g, r, g->ncells, monos(cfg->iorder)};
  const int64_t n = g->ncells;
  std::vector<double> rhs(n * NV), UL, ULV;
  residual(x, U, rhs.data(), UL, ULV);
  const double a[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0}, b[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0}, k[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
  const int s = stage - 1;
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    double oov = 1.0 / g->volume[c];
    for (int v = 0; v < NV; ++v) {
      const double u = U[c * NV + v], rr = dt * (rhs[c * NV + v] * oov);
      U[c * NV + v] = s == 0 ? Un[c * NV + v] - rr : (a[s] * Un[c * NV + v]) + (b[s] * u) - (k[s] * rr);
    }
  }
  return UCG_OK;
}

}  // extern "C"

namespace {
// CALCULATE_CFLL (time_p.f90:193-333): the local time step of every cell
void local_dt(const Ctx& x, const double* U, double ccfl, std::vector<double>& dtl) {
  const ucg_config* cfg = x.cfg;
  const ucg_geometry* g = x.g;
  const int64_t n = x.n;
  const bool ns = cfg->governing == 1;
  const double gm = cfg->gamma;
  dtl.assign(n, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    double p[NV];
    cons2prim(x, &U[c * NV], p);
    const double agrt = std::sqrt(p[4] * gm / p[0]);
    const double veln = std::max(std::max(std::fabs(p[1]), std::fabs(p[2])), std::fabs(p[3])) + agrt;
    const double me = g->minedge[c];
    if (ns) {
      double mu, lam;
      sutherland(cfg, p[0], p[4], &mu, &lam);
      dtl[c] = ccfl * (1.0 / ((std::fabs(veln) / me) + (0.5 * (lam + mu) / (me * me))));
    } else {
      dtl[c] = ccfl * (me / std::fabs(veln));
    }
  }
}

// One implicit correction du of U: RHS, the Jacobian and `nsweeps` sweeps
// from du = 0, with the local time steps dtl.  Dual time (dt > 0): the
// diagonal V (1/DTL + 1.5/dt) + ..., and with U2 (U^n) and U3 (U^{n-1})
// given (ISCOUN 2) the right-hand side -(RHS + V (1.5 U - 2 U^n + 0.5
// U^{n-1}) / dt).
void implicit_du(const Ctx& x, const double* U, const std::vector<double>& dtl, int nsweeps, double dt,
                 const double* U2, const double* U3, std::vector<double>& du) {
  const ucg_config* cfg = x.cfg;
  const ucg_geometry* g = x.g;
  const int64_t n = x.n;
  const bool ns = cfg->governing == 1;
  const double gm = cfg->gamma;
  std::vector<double> rhs(n * NV), UL, ULV, dinv(n), off((size_t)n * F * 25), dn(n * NV);
  du.assign(n * NV, 0.0);
  {
    residual(x, U, rhs.data(), UL, ULV);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
      // Jacobian
      const double* cl = &U[c * NV];
      double lv[NV];
      cons2prim(x, cl, lv);
      double diag = 0.0;
      for (int f = 0; f < g->nfaces[c]; ++f) {
        const double a1 = g->face_angle[(c * F + f) * 2], a2 = g->face_angle[(c * F + f) * 2 + 1];
        const double ang[4] = {std::cos(a1), std::sin(a1), std::cos(a2), std::sin(a2)};
        const double nx = ang[0] * ang[3], ny = ang[1] * ang[3], nz = ang[2];
        const double area = g->face_area[c * F + f];
        const int64_t nb = g->neigh[c * F + f];
        double cr[NV], rv[NV], clr[NV], crr[NV];
        if (nb >= 0)
          for (int v = 0; v < NV; ++v) cr[v] = U[nb * NV + v];
        else
          boundary_state(x, g->bc[c * F + f], ang, cl, cr);
        rotf(ang, cr, crr);
        rotf(ang, cl, clr);
        cons2prim(x, cr, rv);
        const double as1 = std::sqrt(lv[4] * gm / lv[0]) + std::fabs(clr[1] / clr[0]);
        const double as2 = std::sqrt(rv[4] * gm / rv[0]) + std::fabs(crr[1] / crr[0]);
        double vpp = std::max(as1, as2);
        if (ns) {
          double mul, laml, mur, lamr;
          sutherland(cfg, lv[0], lv[4], &mul, &laml);
          sutherland(cfg, rv[0], rv[4], &mur, &lamr);
          double vis = (mul + mur) * 0.5;
          const double rh = 0.5 * (cl[0] + cr[0]), dih = g->dih[c * F + f];
          vis = std::max((4.0 / (3.0 * rh)) * vis * area / dih, (gm / rh) * vis * area / (dih * cfg->prandtl));
          vpp = vpp + vis;
        }
        diag = diag + (0.5 * (vpp * 1.0)) * area;
        // COMPUTE_JACOBIANSE of the right state
        const double A2 = gm - 1.0, A3 = gm - 2.0, oors = 1.0 / cr[0];
        const double us = cr[1] * oors, vs = cr[2] * oors, ws = cr[3] * oors, es = cr[4] * oors;
        const double phi = 0.5 * A2 * ((us * us) + (vs * vs) + (ws * ws));
        const double A1 = gm * es - phi, vvs = nx * us + ny * vs + nz * ws;
        const double J[25] = {0.0, nx, ny, nz, 0.0,
                              nx * phi - us * vvs, vvs - A3 * nx * us, ny * us - A2 * nx * vs, nz * us - A2 * nx * ws, A2 * nx,
                              ny * phi - vs * vvs, nx * vs - A2 * ny * us, vvs - A3 * ny * vs, nz * vs - A2 * ny * ws, A2 * ny,
                              nz * phi - ws * vvs, nx * ws - A2 * nz * us, ny * ws - A2 * nz * vs, vvs - A3 * nz * ws, A2 * nz,
                              vvs * (phi - A1), nx * A1 - A2 * us * vvs, ny * A1 - A3 * vs * vvs, nz * A1 - A2 * ws * vvs,
                              gm * vvs};
        for (int i = 0; i < NV; ++i)
          for (int j = 0; j < NV; ++j)
            off[((size_t)c * F + f) * 25 + i * NV + j] = ((0.5 * J[i * NV + j]) - ((0.5 * vpp) * (i == j ? 1.0 : 0.0))) * area;
      }
      if (dt > 0.0) diag = g->volume[c] * ((1.0 / dtl[c]) + (1.5 / dt)) + diag;
      else diag = diag + (g->volume[c] / dtl[c]);
      dinv[c] = 1.0 / diag;
    }
    for (int sw = 0; sw < nsweeps; ++sw) {
#pragma omp parallel for schedule(static)
      for (int64_t c = 0; c < n; ++c) {
        double b[NV];
        const double* d0 = &du[c * NV];
        for (int v = 0; v < NV; ++v) {
          const int64_t i = c * NV + v;
          b[v] = U2 ? -(rhs[i] + ((((1.5 * U[i]) - (2.0 * U2[i]) + (0.5 * U3[i])) / dt) * g->volume[c])) : -rhs[i];
        }
        for (int f = 0; f < g->nfaces[c]; ++f) {
          const int64_t nb = g->neigh[c * F + f];
          double d1[NV];
          if (nb >= 0) {
            for (int v = 0; v < NV; ++v) d1[v] = du[nb * NV + v];
          } else {
            const int code = g->bc[c * F + f];
            if (code == 1) {
              for (int v = 0; v < NV; ++v) d1[v] = 0.0;
            } else if (code == 3 || code == 4) {
              const double a1 = g->face_angle[(c * F + f) * 2], a2 = g->face_angle[(c * F + f) * 2 + 1];
              const double ang[4] = {std::cos(a1), std::sin(a1), std::cos(a2), std::sin(a2)};
              boundary_state(x, code, ang, d0, d1);
            } else {
              for (int v = 0; v < NV; ++v) d1[v] = d0[v];
            }
          }
          const double* o = &off[((size_t)c * F + f) * 25];
          for (int i = 0; i < NV; ++i) {
            double t = 0.0;
            for (int j = 0; j < NV; ++j) t = t + o[i * NV + j] * d1[j];
            b[i] = b[i] - t;
          }
        }
        for (int v = 0; v < NV; ++v) dn[c * NV + v] = dinv[c] * b[v];
      }
      du.swap(dn);
    }
  }
}
}  // namespace

extern "C" {

// IMPLICIT_TIMEs (time_p.f90:2783-2905, RUNGEKUTTA = 10, ISCOUN = 1) in
// place on U, `nsteps` times: RHS, the local time steps of CALCULATE_CFLL
// (time_p.f90:193-333), the first-order Jacobian of CALCULATE_JACOBIAN
// (implicit_fluxes.f90:12-594) with COMPUTE_JACOBIANSE
// (flow_operations.f90:4004-4049; its entry (5,3) takes gamma - 2), then
// RELAXATION (implicit_time.f90:1-778, RELAX = 1): `nsweeps` sweeps of
// du = D^-1 (-RHS - sum_f O_f du_f) from du = 0, each reading the previous
// sweep's du (the reference updates in place, in an order set by its
// OpenMP schedule); du_f on physical faces: 0 on inflow, the cell's du on
// outflow and far field, BOUNDARYS of du on symmetry and walls.
int orc_implicit_step(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r, double cfl, int nsteps,
                      int nsweeps, double* U) {
  if (!check_ctx(cfg, g, r) || !U || !(cfl > 0.0) || nsteps < 0 || nsweeps < 1) return UCG_EINVAL;
  Ctx x{cfg, g, r, g->ncells, monos(cfg->iorder)};
  std::vector<double> du, dtl;
  for (int step = 0; step < nsteps; ++step) {
    local_dt(x, U, cfl / 3.0, dtl);  // CALCULATE_CFLL before each IMPLICIT_TIMEs call
    implicit_du(x, U, dtl, nsweeps, 0.0, nullptr, nullptr, du);
    for (int64_t c = 0; c < g->ncells * NV; ++c) U[c] = U[c] + du[c];
  }
  return UCG_OK;
}

// DUAL_TIME (time_p.f90:3035-3243, RUNGEKUTTA = 11): one physical step dt
// in place on U with U^n in U2 and U^{n-1} in U3 (both U before the first
// step, IT = RESTART), rotated on return; the local time steps once, from
// the state at the start of the step (CALCULATE_CFLL in the time loop,
// :4104); inner implicit iterations, the first without the time term
// (ISCOUN 1), until sum_c |du_c| V_c / TOTALVOLUME over its largest value
// in the step is <= tol or maxit are done (*iters).
int orc_dual_time_step(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r, double dt, double cfl,
                       int maxit, double tol, int nsweeps, double* U, double* U2, double* U3, int* iters) {
  if (!check_ctx(cfg, g, r) || !U || !U2 || !U3 || !(dt > 0.0) || !(cfl > 0.0) || maxit < 1 || nsweeps < 1)
    return UCG_EINVAL;
  Ctx x{cfg, g, r, g->ncells, monos(cfg->iorder)};
  const int64_t n = g->ncells;
  double tot = 0.0;
  for (int64_t c = 0; c < n; ++c) tot += g->volume[c];
  std::vector<double> du, dtl;
  local_dt(x, U, cfl / 3.0, dtl);
  double firsti = 0.0;
  int jj;
  for (jj = 1; jj <= maxit; ++jj) {
    implicit_du(x, U, dtl, nsweeps, dt, jj == 1 ? nullptr : U2, U3, du);
    double res = 0.0;
    for (int64_t c = 0; c < n; ++c) {
      const double* d = &du[c * NV];
      res += std::sqrt((d[0] * d[0]) + (d[1] * d[1]) + (d[2] * d[2]) + (d[3] * d[3]) + (d[4] * d[4])) * g->volume[c];
    }
    for (int64_t i = 0; i < n * NV; ++i) U[i] = U[i] + du[i];
    res = res / tot;
    if (res > firsti) firsti = res;
    res = res / firsti;
    if (res <= tol) break;
  }
  if (iters) *iters = jj > maxit ? maxit : jj;
  for (int64_t i = 0; i < n * NV; ++i) {
    U3[i] = U2[i];
    U2[i] = U[i];
  }
  return UCG_OK;
}

// DUAL_TIME_EX (time_p.f90:3244-3436, RUNGEKUTTA = 12) with RELAXATION_EX
// (:3844-3888): one physical step dt in place on U (U^n in U2, U^{n-1} in
// U3, both U before the first step), the local time steps once from the
// state at the start of the step; explicit pseudo-time iterations
//   du = -(V/dt (1.5 U - 2 U^n + 0.5 U^{n-1}) + RHS(U)) dtau,
//   dtau = (DTL / V) / (1 + 1.5 DTL/dt),  U += du,
// until sum_c |du_c| V_c / TOTALVOLUME over its largest value in the step is
// <= tol or maxit are done (*iters); then U^{n-1} <- U^n <- U and U <- 2 U^n
// - U^{n-1}, the next step's first iterate.
int orc_dual_time_step_explicit(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r, double dt,
                                double cfl, int maxit, double tol, double* U, double* U2, double* U3, int* iters) {
  if (!check_ctx(cfg, g, r) || !U || !U2 || !U3 || !(dt > 0.0) || !(cfl > 0.0) || maxit < 1) return UCG_EINVAL;
  Ctx x{cfg, g, r, g->ncells, monos(cfg->iorder)};
  const int64_t n = g->ncells;
  double tot = 0.0;
  for (int64_t c = 0; c < n; ++c) tot += g->volume[c];
  std::vector<double> dtl, rhs(n * NV), du(n * NV), UL, ULV;
  local_dt(x, U, cfl / 3.0, dtl);
  double firsti = 0.0;
  int jj;
  for (jj = 1; jj <= maxit; ++jj) {
    residual(x, U, rhs.data(), UL, ULV);
    double res = 0.0;
    for (int64_t c = 0; c < n; ++c) {
      const double dt1 = g->volume[c] / dt;
      const double dtau = (dtl[c] / g->volume[c]) * (1.0 / (1.0 + (1.5 * (dtl[c] / dt))));
      double* d = &du[c * NV];
      for (int v = 0; v < NV; ++v) {
        const int64_t i = c * NV + v;
        const double imp = (dt1 * (((1.5 * U[i]) - (2.0 * U2[i])) + (0.5 * U3[i]))) + rhs[i];
        d[v] = (-imp) * dtau;
      }
      res += std::sqrt((d[0] * d[0]) + (d[1] * d[1]) + (d[2] * d[2]) + (d[3] * d[3]) + (d[4] * d[4])) * g->volume[c];
    }
    for (int64_t i = 0; i < n * NV; ++i) U[i] = U[i] + du[i];
    res = res / tot;
    if (res > firsti) firsti = res;
    res = res / firsti;
    if (res <= tol) break;
  }
  if (iters) *iters = jj > maxit ? maxit : jj;
  for (int64_t i = 0; i < n * NV; ++i) {
    U3[i] = U2[i];
    U2[i] = U[i];
    U[i] = (2.0 * U2[i]) - U3[i];
  }
  return UCG_OK;
}

// RUNGE_KUTTA3_MOOD (time_p.f90:582-880) in place on U [n][5], Euler with
// WENO; recalc [n] is RECALC, carried between calls (zero before the first
// step, memory.f90:1002-1005); order (optional, [n]) MOOD_O after the step.
int orc_rk3_step_mood(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r, double dt, double* U,
                      int8_t* recalc, int32_t* order) {
  if (!check_ctx(cfg, g, r) || !U || !recalc || !cfg->mood || cfg->governing != 2 || cfg->scheme != 3)
    return UCG_EINVAL;
  Ctx x{cfg, g, r, g->ncells, monos(cfg->iorder)};
  const int64_t n = g->ncells;
  std::vector<int8_t> rc(recalc, recalc + n);
  std::vector<double> Un(U, U + n * NV), Ua(n * NV), Ub(n * NV);
  mood_stage(x, 1, dt, Un.data(), Un.data(), Ua.data(), rc, nullptr);
  mood_stage(x, 2, dt, Ua.data(), Un.data(), Ub.data(), rc, nullptr);
  mood_stage(x, 3, dt, Ub.data(), Un.data(), U, rc, order);
  for (int64_t c = 0; c < n; ++c) recalc[c] = rc[c];
  return UCG_OK;
}

// Wall force in x (COMPUTEFORCE, src/io.f90:18752-18915, inviscid part):
// over faces with boundary code 4, SSP = sum_q p(ULEFT_q) * w_q - PRES, then
// FORCEX += SSP * SURF * NX with NX = cos(angle1) * sin(angle2).
int orc_force(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r, const double* U, double* fx) {
  if (!check_ctx(cfg, g, r) || !U || !fx) return UCG_EINVAL;
  const int64_t n = g->ncells;
  std::vector<double> ul((size_t)n * F * Q * NV);
  int rc = orc_face_values(cfg, g, r, U, ul.data());
  if (rc) return rc;
  Ctx x{cfg, g, r, n, monos(cfg->iorder)};
  double force = 0.0;
  for (int64_t c = 0; c < n; ++c)
    for (int f = 0; f < g->nfaces[c]; ++f) {
      if (g->neigh[c * F + f] >= 0 || g->bc[c * F + f] != 4) continue;
      const bool quad = g->face_type[c * F + f] == 5;
      const int nq = quad ? cfg->nq_quad : cfg->nq_tri;
      const double* w = quad ? cfg->quad_w : cfg->tri_w;
      double ssp = 0.0;
      for (int q = 0; q < nq; ++q) {
        double pm[NV];
        cons2prim(x, &ul[(((size_t)c * F + f) * Q + q) * NV], pm);
        ssp = ssp + (pm[4] * w[q]);
      }
      ssp = ssp - cfg->pres;
      const double a1 = g->face_angle[(c * F + f) * 2], a2 = g->face_angle[(c * F + f) * 2 + 1];
      const double nx = std::cos(a1) * std::sin(a2);
      force = force + ((ssp * g->face_area[c * F + f]) * nx);
    }
  *fx = force;
  return UCG_OK;
}

// COMPUTEFORCE (io.f90:18752-19000) in full: out = FX, FY, FZ, MX, MY, MZ.
// Per wall face (code 4): SSP = sum_q w_q p_q - PRES and, Navier-Stokes,
// SS = -sum_q mu_q (n . tau_q) w_q with tau from the cell's own face-point
// velocity gradients (ULEFTV rows u, v, w) and mu from SUTHERLAND at the
// face state; F += SSP * S * n + SS * S; the moments take the pressure
// part about the cell centre (IELEM%XXC, YYC, ZZC), centre NULL = none.
int orc_wall_loads(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r, const double* U,
                   const double* centre, double* out) {
  if (!check_ctx(cfg, g, r) || !U || !out) return UCG_EINVAL;
  const int64_t n = g->ncells;
  const bool ns = cfg->governing == 1;
  Ctx x{cfg, g, r, n, monos(cfg->iorder)};
  std::vector<double> ul((size_t)n * F * Q * NV, 0.0), ulv(ns ? (size_t)n * F * Q * 12 : 1, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t c = 0; c < n; ++c)
    reconstruct_cell(x, c, U, &ul[(size_t)c * F * Q * NV], ns ? &ulv[(size_t)c * F * Q * 12] : nullptr);
  double fx = 0.0, fy = 0.0, fz = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  for (int64_t c = 0; c < n; ++c)
    for (int f = 0; f < g->nfaces[c]; ++f) {
      if (g->neigh[c * F + f] >= 0 || g->bc[c * F + f] != 4) continue;
      const bool quad = g->face_type[c * F + f] == 5;
      const int nq = quad ? cfg->nq_quad : cfg->nq_tri;
      const double* w = quad ? cfg->quad_w : cfg->tri_w;
      const double a1 = g->face_angle[(c * F + f) * 2], a2 = g->face_angle[(c * F + f) * 2 + 1];
      const double nx = std::cos(a1) * std::sin(a2), ny = std::sin(a1) * std::sin(a2), nz = std::cos(a2);
      const double S = g->face_area[c * F + f];
      double ssp = 0.0, ssx = 0.0, ssy = 0.0, ssz = 0.0;
      for (int q = 0; q < nq; ++q) {
        const size_t k = (((size_t)c * F + f) * Q + q);
        double pm[NV];
        cons2prim(x, &ul[k * NV], pm);
        ssp = ssp + (pm[4] * w[q]);
        if (ns) {
          const double* gv = &ulv[k * 12];  // rows T, u, v, w; columns x, y, z
          const double ux = gv[3], uy = gv[4], uz = gv[5], vx = gv[6], vy = gv[7], vz = gv[8];
          const double wx = gv[9], wy = gv[10], wz = gv[11];
          double mu, lam;
          sutherland(cfg, pm[0], pm[4], &mu, &lam);
          const double txx = (4.0 / 3.0) * ux - (2.0 / 3.0) * vy - (2.0 / 3.0) * wz;
          const double tyy = (4.0 / 3.0) * vy - (2.0 / 3.0) * ux - (2.0 / 3.0) * wz;
          const double tzz = (4.0 / 3.0) * wz - (2.0 / 3.0) * ux - (2.0 / 3.0) * vy;
          const double tyx = uy + vx, tzx = wx + uz, tzy = vz + wy;
          ssx = ssx - ((mu * ((nx * txx) + (ny * tyx) + (nz * tzx))) * w[q]);
          ssy = ssy - ((mu * ((nx * tyx) + (ny * tyy) + (nz * tzy))) * w[q]);
          ssz = ssz - ((mu * ((nx * tzx) + (ny * tzy) + (nz * tzz))) * w[q]);
        }
      }
      ssp = ssp - cfg->pres;
      fx = fx + ((ssp * S * nx)) + (ssx * S);
      fy = fy + ((ssp * S * ny)) + (ssy * S);
      fz = fz + ((ssp * S * nz)) + (ssz * S);
      if (centre) {
        const double xc = centre[c * 3], yc = centre[c * 3 + 1], zc = centre[c * 3 + 2];
        mx = mx + ((ssp * S * nz)) * yc - ((ssp * S * ny)) * zc;
        my = my + ((ssp * S * nx)) * zc - ((ssp * S * nz)) * xc;
        mz = mz + ((ssp * S * ny)) * xc - ((ssp * S * nx)) * yc;
      }
    }
  out[0] = fx, out[1] = fy, out[2] = fz, out[3] = mx, out[4] = my, out[5] = mz;
  return UCG_OK;
}

// HLLC flux of two conserved states in the face frame (known-answer tests).
int orc_hllc(double gamma, const double* cl, const double* cr, double* flux) {
  hllc(gamma, cl, cr, flux);
  return UCG_OK;
}

// one ghost state of BOUNDARYS for boundary code `code` on a face of angles
// (ANGLE1, ANGLE2); gamma, boundtype and the free stream come from cfg
int orc_boundary(const ucg_config* cfg, int code, const double* angles, const double* cl, double* cr) {
  Ctx x{};
  x.cfg = cfg;
  const double ang[4] = {std::cos(angles[0]), std::sin(angles[0]), std::cos(angles[1]), std::sin(angles[1])};
  boundary_state(x, code, ang, cl, cr);
  return (code == 1 || code == 2 || code == 3 || code == 4 || code == 6) ? UCG_OK : UCG_EINVAL;
}

// one global-frame flux of the Roe family (iRiemann 3 Roe, 4 rotated
// Roe-HLL, 5 t-Roe) through a face of unit normal n
int orc_riemann(int kind, double gamma, const double* cl, const double* cr, const double* n, double* flux) {
  if (kind == 3) roe(gamma, cl, cr, n, flux);
  else if (kind == 4) rhll(gamma, cl, cr, n, flux);
  else if (kind == 5) troe(gamma, cl, cr, n, flux);
  else return UCG_EINVAL;
  return UCG_OK;
}

// Domain sums (time_p.f90:4145-4198): 1 = kinetic energy, 2 = mass, 3 = energy.
// ENSTROPHY_CALC (flow_operations.f90:2718-2815, BOUNDTYPE 1) summed as
// TOTENS (time_p.f90:4311-4320): sum V * rho * 0.5 * (0.5 * ONORM * rho),
// ONORM = |G - G^T|_F^2 with G the cell-centre velocity gradients
// (SOLUTIONTRIAV2's GRADS, reconstruct_p.f90:2590-2660), which for IORDER 1
// equal the face gradients of the linear viscous polynomial.
int orc_enstrophy(const ucg_config* cfg, const ucg_geometry* g, const ucg_recon* r, const double* U, double* out) {
  if (!check_ctx(cfg, g, r) || !U || !out || cfg->governing != 1 || cfg->scheme != 2 || cfg->iorder != 1)
    return UCG_EINVAL;
  Ctx x{cfg, g, r, g->ncells, monos(cfg->iorder)};
  std::vector<double> UL, ULV;
  std::vector<double> rhs((size_t)x.n * NV);
  residual(x, U, rhs.data(), UL, ULV);
  double s = 0.0;
  for (int64_t c = 0; c < x.n; ++c) {
    const double* G = &ULV[(size_t)c * F * Q * 12 + 3];
    double on = 0.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const double d = G[i * 3 + j] - G[j * 3 + i];
        on += d * d;
      }
    const double rho = U[c * NV];
    s += g->volume[c] * (rho * 0.5 * (0.5 * (on * rho)));
  }
  *out = s;
  return UCG_OK;
}

int orc_reduce(const ucg_geometry* g, const double* U, int what, double* out) {
  if (!g || !U || !out) return UCG_EINVAL;
  double s = 0.0;
  for (int64_t c = 0; c < g->ncells; ++c) {
    const double* u = &U[c * NV];
    double v;
    if (what == UCG_REDUCE_KE) v = 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0];
    else if (what == UCG_REDUCE_MASS) v = u[0];
    else v = u[4];
    s += g->volume[c] * v;
  }
  *out = s;
  return UCG_OK;
}

}  // extern "C"
