// Device-side building blocks shared by the engine kernels: problem
// descriptor, basis evaluation, gas relations, face rotation, HLLC.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ucns3d_gpu.h"

namespace ucg {

constexpr int NV = UCG_NV;
constexpr int MF = UCG_MAX_FACES;
constexpr int MQ = UCG_MAX_QP;
constexpr double TOLSMALL = 1.0e-13;  // grid_p.f90:18
constexpr double TOLBIG = 1.0e13;     // grid_p.f90:19

// Health word bits set by kernels (read by ucg_check_health).
enum : unsigned { HEALTH_NONPHYS = 1u };

// Problem description passed by value to every kernel.  Arrays are device
// pointers; "[c]" means one entry per cell, cell index fastest where noted.
struct Problem {
  int64_t n;
  int iorder, ideg, imax, admis_max, ideg2, imax2, ees, scheme, governing, wenoz;
  int nq_quad, nq_tri;
  double gamma, prandtl, visc, r_gas, pres, rres, lwci, weno_eps, kappa_ven, lamx;
  double quad_w[MQ], tri_w[MQ];
  double bc_state[NV];
  // geometry, per cell contiguous (AoS) unless noted
  const int8_t* nfaces;     // [n]
  const int8_t* ftype;      // [n][MF]  5 quad, 6 tri
  const int32_t* neigh;     // [n][MF]
  const int8_t* nface;      // [n][MF]  neighbour's face
  const int8_t* bc;         // [n][MF]
  const uint8_t* qperm;     // [n][MF][MQ]
  const double* rot;        // [n][MF][4]  cos a1, sin a1, cos a2, sin a2
  const double* area;       // [n][MF]
  const double* dih;        // [n][MF]
  const double* vol;        // [n]
  const double* minedge;    // [n]
  const double* jinv;       // [n][9]
  const int8_t* admis;      // [n]
  const int8_t* full;       // [n]
  // reconstruction tables, per cell contiguous, precision T
  const void* qpts;         // [n][MF][MQ][3]
  const void* bmean;        // [n][ideg]
  const int32_t* sten;      // [n][A][imax+1]
  const void* invmat;       // [n][A][imax][ideg]
  const void* invmat2;      // [n][A][imax2][ideg2]
  const void* ind;          // [n][ideg][ideg]
  const void* ind2;         // [n][ideg2][ideg2]
  // scratch
  void* dul;                // [n][MF][MQ][NV]  face value minus cell mean (T)
  double* ulv;              // [n][MF][MQ][4][3] face gradients of T,u,v,w
  double* gv;               // [n][ideg][4]  viscous LSQ coefficients
  double* rhs;              // [n][NV] residual output (residual-only mode)
  unsigned* health;
  double* dt_dev;           // device dt (ucg_step)
};

// ------------------------------------------------------------- basis
// Exponents of the reconstruction basis in the order of BASIS_REC
// (src/basis.f90:24-100): degree by degree, z powers then y powers ascending.
__constant__ __device__ static const int8_t kExp[34][3] = {
    {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
    {2, 0, 0}, {1, 1, 0}, {0, 2, 0}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2},
    {3, 0, 0}, {2, 1, 0}, {1, 2, 0}, {0, 3, 0}, {2, 0, 1}, {1, 1, 1}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {0, 0, 3},
    {4, 0, 0}, {3, 1, 0}, {2, 2, 0}, {1, 3, 0}, {0, 4, 0}, {3, 0, 1}, {2, 1, 1}, {1, 2, 1}, {0, 3, 1},
    {2, 0, 2}, {1, 1, 2}, {0, 2, 2}, {1, 0, 3}, {0, 1, 3}, {0, 0, 4}};

template <int P>
struct Deg {
  static constexpr int ideg = (P + 1) * (P + 2) * (P + 3) / 6 - 1;
};

// monomials of degree 1..P at (x,y,z), in basis order
template <int P, typename R>
__device__ __forceinline__ void monomials(R x, R y, R z, R* m) {
  R px[P + 1], py[P + 1], pz[P + 1];
  px[0] = py[0] = pz[0] = R(1);
#pragma unroll
  for (int k = 1; k <= P; ++k) {
    px[k] = px[k - 1] * x;
    py[k] = py[k - 1] * y;
    pz[k] = pz[k - 1] * z;
  }
  int d = 0;
#pragma unroll
  for (int n = 1; n <= P; ++n)
#pragma unroll
    for (int c = 0; c <= n; ++c)
#pragma unroll
      for (int b = 0; b <= n - c; ++b) m[d++] = px[n - c - b] * py[b] * pz[c];
}

// first derivatives d/dx, d/dy, d/dz of the monomials (DFX/DFY/DFZ)
template <int P>
__device__ __forceinline__ void dmonomials(double x, double y, double z, double* dx, double* dy, double* dz) {
  double px[P + 1], py[P + 1], pz[P + 1];
  px[0] = py[0] = pz[0] = 1.0;
#pragma unroll
  for (int k = 1; k <= P; ++k) {
    px[k] = px[k - 1] * x;
    py[k] = py[k - 1] * y;
    pz[k] = pz[k - 1] * z;
  }
  int d = 0;
#pragma unroll
  for (int n = 1; n <= P; ++n)
#pragma unroll
    for (int c = 0; c <= n; ++c)
#pragma unroll
      for (int b = 0; b <= n - c; ++b) {
        int a = n - c - b;
        dx[d] = a ? a * px[a - 1] * py[b] * pz[c] : 0.0;
        dy[d] = b ? b * px[a] * py[b - 1] * pz[c] : 0.0;
        dz[d] = c ? c * px[a] * py[b] * pz[c - 1] : 0.0;
        ++d;
      }
}

// ------------------------------------------------------------- gas
__device__ __forceinline__ void cons2prim(double gamma, const double* u, double* p) {
  double oo = 1.0 / u[0];
  p[0] = u[0];
  p[1] = u[1] * oo;
  p[2] = u[2] * oo;
  p[3] = u[3] * oo;
  p[4] = (gamma - 1.0) * (u[4] - 0.5 * u[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]));
}

__device__ __forceinline__ void prim2cons(double gamma, const double* p, double* u) {
  double skin = 0.5 * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
  double ie = p[4] / ((gamma - 1.0) * p[0]);
  u[0] = p[0];
  u[1] = p[1] * p[0];
  u[2] = p[2] * p[0];
  u[3] = p[3] * p[0];
  u[4] = p[0] * ie + p[0] * skin;
}

// ROTATEF / ROTATEB (src/grid_t.f90:4217-4305); r = cos a1, sin a1, cos a2, sin a2
__device__ __forceinline__ void rot_f(const double* r, const double* v, double* o) {
  o[0] = v[0];
  o[1] = r[0] * r[3] * v[1] + r[1] * r[3] * v[2] + r[2] * v[3];
  o[2] = r[0] * r[2] * v[1] + r[1] * r[2] * v[2] - r[3] * v[3];
  o[3] = -r[1] * v[1] + r[0] * v[2];
  o[4] = v[4];
}
__device__ __forceinline__ void rot_b(const double* r, const double* v, double* o) {
  o[0] = v[0];
  o[1] = r[0] * r[3] * v[1] + r[0] * r[2] * v[2] - r[1] * v[3];
  o[2] = r[1] * r[3] * v[1] + r[1] * r[2] * v[2] + r[0] * v[3];
  o[3] = r[2] * v[1] - r[3] * v[2];
  o[4] = v[4];
}

// HLLC in the face frame (HLLC_RIEMANN_SOLVER, src/riemann.f90:221-426):
// Einfeldt-type wave speeds from Roe averages, SL <= 0 <= SR, and the final
// flux is the sign(SM) blend of the two star fluxes.
__device__ __forceinline__ void hllc(double gamma, const double* cl, const double* cr, double* flux) {
  double rl = cl[0], ul = cl[1] / rl, vl = cl[2] / rl, wl = cl[3] / rl;
  double pl = (gamma - 1.0) * (cl[4] - 0.5 * rl * (ul * ul + vl * vl + wl * wl));
  double rr = cr[0], ur = cr[1] / rr, vr = cr[2] / rr, wr = cr[3] / rr;
  double pr = (gamma - 1.0) * (cr[4] - 0.5 * rr * (ur * ur + vr * vr + wr * wr));
  double el = cl[4], er = cr[4];
  double ccl = sqrt(gamma * pl / rl), ccr = sqrt(gamma * pr / rr);
  double srl = sqrt(rl), srr = sqrt(rr), ssum = srl + srr;
  double cc2 = sqrt((ccl * ccl * srl + ccr * ccr * srr) / ssum +
                    0.5 * ((srl * srr) / (ssum * ssum)) * ((ur - ul) * (ur - ul)));
  double uu2 = (ul * srl + ur * srr) / ssum;
  double sl = fmin(fmin(ul - ccl, uu2 - cc2), 0.0);
  double sr = fmax(fmax(ur + ccr, uu2 + cc2), 0.0);
  double sm = (pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur)) / (rl * (sl - ul) - rr * (sr - ur));
  double mul = rl * ((sl - ul) / (sl - sm)), mur = rr * ((sr - ur) / (sr - sm));
  double lastl = el / rl + (sm - ul) * (sm + pl / (rl * (sl - ul)));
  double lastr = er / rr + (sm - ur) * (sm + pr / (rr * (sr - ur)));
  double sg = copysign(1.0, sm);
  double al = 0.5 * (1.0 + sg), ar = 0.5 * (1.0 - sg);
  double fl0 = rl * ul, fr0 = rr * ur;
  flux[0] = al * (fl0 + sl * (mul - cl[0])) + ar * (fr0 + sr * (mur - cr[0]));
  flux[1] = al * (fl0 * ul + pl + sl * (mul * sm - cl[1])) + ar * (fr0 * ur + pr + sr * (mur * sm - cr[1]));
  flux[2] = al * (fl0 * vl + sl * (mul * vl - cl[2])) + ar * (fr0 * vr + sr * (mur * vr - cr[2]));
  flux[3] = al * (fl0 * wl + sl * (mul * wl - cl[3])) + ar * (fr0 * wr + sr * (mur * wr - cr[3]));
  flux[4] = al * (ul * (el + pl) + sl * (mul * lastl - cl[4])) + ar * (ur * (er + pr) + sr * (mur * lastr - cr[4]));
}

// Venkatakrishnan limiter, SLOPE_LIMITERS case 7 (src/reconstruct_p.f90:3647-3652)
__device__ __forceinline__ double venkat(double d2, double umin0, double umax0, double epsi2) {
  if (fabs(d2) <= 0.0) return 1.0;
  double dmin = copysign(1.0, d2) * (fabs(d2) + TOLSMALL);
  double dplus = d2 > 0.0 ? umax0 : umin0;
  return (1.0 / dmin) * (((dplus * dplus + epsi2) * dmin + 2.0 * (dmin * dmin) * dplus) /
                         (dplus * dplus + 2.0 * dmin * dmin + dmin * dplus + epsi2));
}

// CHECKSOL / CHECKSOLX jump test of one face value against the cell mean
__device__ __forceinline__ bool jump_bad(double gamma, const double* pm, const double* uf, double jump) {
  double pf[NV];
  cons2prim(gamma, uf, pf);
  return (fabs(pf[0] - pm[0]) >= jump * pm[0]) || (fabs(pf[4] - pm[4]) >= jump * pm[4]) || (pf[4] < 0.0) ||
         (pf[0] < 0.0);
}

__device__ __forceinline__ double face_weight(const Problem& p, int ft, int q) {
  return ft == 5 ? p.quad_w[q] : p.tri_w[q];
}
__device__ __forceinline__ int face_nq(const Problem& p, int ft) { return ft == 5 ? p.nq_quad : p.nq_tri; }

// Sutherland's law (SUTHERLAND, src/flow_operations.f90:2609-2640);
// (t1/t0)^1.5 written as r*sqrt(r).
__device__ __forceinline__ void sutherland(const Problem& p, double rho, double pr, double* mu, double* lam) {
  const double suther = 0.412158681;
  double t1 = pr / (rho * p.r_gas);
  double t0 = p.pres / (p.rres * p.r_gas);
  double r = t1 / t0;
  *mu = p.visc * (r * sqrt(r)) * ((t0 + suther * t0) / (t1 + suther * t0));
  *lam = (*mu) * p.r_gas * p.gamma / (p.prandtl * (p.gamma - 1.0));
}

}  // namespace ucg
