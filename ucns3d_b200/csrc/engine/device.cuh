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
enum : unsigned { HEALTH_NONPHYS = 1u };  // HEALTH_TIMEOUT = 2 below

// Problem description passed by value to every kernel.  Arrays are device
// pointers; "[c]" means one entry per cell, cell index fastest where noted.
struct Problem {
  int64_t n;     // cells the kernels of a launch cover
  int64_t nall;  // cells of the engine (more than n for a partition's reconstruction: ucg_set_cell_roles)
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
  // reconstruction tables in precision T, interleaved over 32-cell groups
  // (element j of cell c at ((c / 32) * len + j) * 32 + c % 32)
  const void* qpts;         // len = MF*QS*3: [f][q][xyz], QS = max(nq_quad, nq_tri)
  const void* bmean;        // len = ideg
  // stencils and pseudo-inverses are interleaved over groups of 32 cells:
  // element j of cell c is at ((c / 32) * len + j) * 32 + c % 32, with
  // len = A*(imax+1) for the stencils and `tstride` for the pseudo-inverses.
  // Slice ll of a cell's pseudo-inverse block ([nk][nd], nk = imax or imax2,
  // nd = ideg or ideg2) starts at element soff[ll].
  const int32_t* sten;
  const void* invmat;
  int64_t tstride;
  int soff[8];
  // smoothness matrices, vector-interleaved (see Vec) with len = `istride`:
  // packed upper triangle of S [ideg][ideg] at element 0 and of the CWENO
  // S2 [ideg2][ideg2] at i2off, rows padded to whole vectors, off-diagonal
  // entries S_de + S_ed
  const void* ind;
  int64_t istride;
  int i2off;
  // scratch
  void* gbuf;               // stencil polynomials G[ll][d][v], interleaved like the stencils
  double* qbuf;             // characteristic WENO: G_l^T S G_l per stencil, 15 values, interleaved
  double* isb;              // conserved WENO: smoothness indicators [A][NV] per cell, interleaved (k_wis)
  bool wface;               // IORDER 4 conserved WENO through k_wis + k_wface
  int8_t* wflag;            // cells whose reconstruction was reduced (CHECKSOL or not FULL) [n];
                            // k_wface writes it for k_wpost's fall-back pass, k_wpost under MOOD
  // MOOD (RUNGE_KUTTA3_MOOD): all nullptr without it
  int8_t* mprev;            // RECALC of the last MOOD pass: the fall-back cells of the next reconstruction
  int8_t* mood;             // MOOD flag of the current cascade (PAD_NAD)
  int8_t* msel;             // cells whose residual the current cascade recomputes (FIX_LIST); also
                            // selects the faces k_face recomputes (nullptr: every face)
  int8_t* mmus;             // first cascade: msel and reduced, MUSCL recomputed
  int8_t* mord;             // MOOD_O per cell
  void* dul;                // [n][MF][MQ][NV]  face value minus cell mean (T)
  double* ulv;              // [n][MF][MQ][4][3] face gradients of T,u,v,w (MUSCL IORDER 1)
  double* fgrad;            // [nown][QS][4][3] face-point average of both sides' gradients of T,u,v,w (WENO)
  void* gv;                 // [n][ideg][4]  viscous LSQ coefficients, in the table precision
  double* prim;             // [n][4] T, u, v, w of each cell (viscous LSQ, formed once per stage)
  double* upad;             // [n][6] conserved state in 48-byte records (k_lsq gathers, formed once per stage)
  double* rhs;              // [n][NV] residual output (residual-only mode)
  const int32_t* own;       // owned faces, code cell*8 + face
  int64_t nown;
  double* fflux;            // [n][MF][NV] convective face sums (owner and negated copy)
  double* vflux;            // [n][MF][NV] viscous face sums
  unsigned* health;
  int lsq_bulk;  // stencil least squares through the shared-memory bulk-copy ring (k_lsq_tma)
  long lsq_wait; // polls of a k_lsq_tma stage wait before it gives up (< 0: the default)
  int wenwrt;    // 1 conserved-variable WENO, 2 characteristic-variable WENO
  int riemann;   // 1 HLLC, 2 Rusanov, 3 Roe, 4 rotated Roe-HLL, 5 t-Roe, 9 HLL
  int limiter;   // SLOPE_LIMITERS code (7 Venkatakrishnan)
  int boundtype; // BOUNDTYPE: 0 supersonic inflow/outflow, 1 characteristic treatment
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

// 16-byte vectors of the table precision: VEC elements per lane and load.
// "Vector-interleaved" arrays store element j of cell c at
// (((c/32)*len/VEC + j/VEC)*32 + c%32)*VEC + j%VEC (len a multiple of VEC),
// so a warp reads VEC consecutive elements of 32 cells with one 512-byte load.
template <typename T>
struct Vec {
  static constexpr int N = 16 / (int)sizeof(T);
};
__device__ __forceinline__ void ldv(const float* p, float (&o)[4]) {
  const float4 x = *(const float4*)p;
  o[0] = x.x;
  o[1] = x.y;
  o[2] = x.z;
  o[3] = x.w;
}
__device__ __forceinline__ void ldv(const double* p, double (&o)[2]) {
  const double2 x = *(const double2*)p;
  o[0] = x.x;
  o[1] = x.y;
}

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

// first derivatives d/dx, d/dy, d/dz of the monomials (DFX/DFY/DFZ), in R
template <int P, typename R = double>
__device__ __forceinline__ void dmonomials(R x, R y, R z, R* dx, R* dy, R* dz) {
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
      for (int b = 0; b <= n - c; ++b) {
        int a = n - c - b;
        dx[d] = a ? R(a) * px[a - 1] * py[b] * pz[c] : R(0);
        dy[d] = b ? R(b) * px[a] * py[b - 1] * pz[c] : R(0);
        dz[d] = c ? R(c) * px[a] * py[b] * pz[c - 1] : R(0);
        ++d;
      }
}

// ------------------------------------------------------------- gas
// The gas relations, rotations, HLLC, the limiter and the boundary states
// are templates over the scalar type S: the engine uses S = double, the
// discrete adjoint and tangent (adjoint.cu) forward-mode dual numbers.
__host__ __device__ __forceinline__ double value(double x) { return x; }

template <typename S>
__host__ __device__ __forceinline__ void cons2prim(double gamma, const S* u, S* p) {
  S oo = 1.0 / u[0];
  p[0] = u[0];
  p[1] = u[1] * oo;
  p[2] = u[2] * oo;
  p[3] = u[3] * oo;
  p[4] = (gamma - 1.0) * (u[4] - 0.5 * u[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]));
}

template <typename S>
__host__ __device__ __forceinline__ void prim2cons(double gamma, const S* p, S* u) {
  S skin = 0.5 * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
  S ie = p[4] / ((gamma - 1.0) * p[0]);
  u[0] = p[0];
  u[1] = p[1] * p[0];
  u[2] = p[2] * p[0];
  u[3] = p[3] * p[0];
  u[4] = p[0] * ie + p[0] * skin;
}

// ROTATEF / ROTATEB (src/grid_t.f90:4217-4305); r = cos a1, sin a1, cos a2, sin a2
template <typename S>
__host__ __device__ __forceinline__ void rot_f(const double* r, const S* v, S* o) {
  o[0] = v[0];
  o[1] = r[0] * r[3] * v[1] + r[1] * r[3] * v[2] + r[2] * v[3];
  o[2] = r[0] * r[2] * v[1] + r[1] * r[2] * v[2] - r[3] * v[3];
  o[3] = -r[1] * v[1] + r[0] * v[2];
  o[4] = v[4];
}
template <typename S>
__host__ __device__ __forceinline__ void rot_b(const double* r, const S* v, S* o) {
  o[0] = v[0];
  o[1] = r[0] * r[3] * v[1] + r[0] * r[2] * v[2] - r[1] * v[3];
  o[2] = r[1] * r[3] * v[1] + r[1] * r[2] * v[2] + r[0] * v[3];
  o[3] = r[2] * v[1] - r[3] * v[2];
  o[4] = v[4];
}

// HLLC in the face frame (HLLC_RIEMANN_SOLVER, src/riemann.f90:221-426):
// Einfeldt-type wave speeds from Roe averages, SL <= 0 <= SR, and the final
// flux is the sign(SM) blend of the two star fluxes.  The reciprocals of the
// two densities and of sqrt(rl) + sqrt(rr) are formed once and multiplied
// (8 divisions instead of 18; the FP64 face kernel is bound by the divide
// and square-root sequences): values differ from the all-division form by
// rounding only.
template <typename S>
__host__ __device__ __forceinline__ void hllc(double gamma, const S* cl, const S* cr, S* flux) {
  // reciprocals of the densities and of sqrt(rl) + sqrt(rr) formed once
  S rl = cl[0], irl = 1.0 / rl, ul = cl[1] * irl, vl = cl[2] * irl, wl = cl[3] * irl;
  S pl = (gamma - 1.0) * (cl[4] - 0.5 * rl * (ul * ul + vl * vl + wl * wl));
  S rr = cr[0], irr = 1.0 / rr, ur = cr[1] * irr, vr = cr[2] * irr, wr = cr[3] * irr;
  S pr = (gamma - 1.0) * (cr[4] - 0.5 * rr * (ur * ur + vr * vr + wr * wr));
  S el = cl[4], er = cr[4];
  S ccl = sqrt(gamma * pl * irl), ccr = sqrt(gamma * pr * irr);
  S srl = sqrt(rl), srr = sqrt(rr), ssum = srl + srr, iss = 1.0 / ssum;
  S cc2 = sqrt((ccl * ccl * srl + ccr * ccr * srr) * iss + 0.5 * ((srl * srr) * (iss * iss)) * ((ur - ul) * (ur - ul)));
  S uu2 = (ul * srl + ur * srr) * iss;
  S sl = fmin(fmin(ul - ccl, uu2 - cc2), 0.0);
  S sr = fmax(fmax(ur + ccr, uu2 + cc2), 0.0);
  S sm = (pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur)) / (rl * (sl - ul) - rr * (sr - ur));
  S mul = rl * ((sl - ul) / (sl - sm)), mur = rr * ((sr - ur) / (sr - sm));
  S lastl = el * irl + (sm - ul) * (sm + pl / (rl * (sl - ul)));
  S lastr = er * irr + (sm - ur) * (sm + pr / (rr * (sr - ur)));
  double sg = copysign(1.0, value(sm));
  double al = 0.5 * (1.0 + sg), ar = 0.5 * (1.0 - sg);
  S fl0 = rl * ul, fr0 = rr * ur;
  flux[0] = al * (fl0 + sl * (mul - cl[0])) + ar * (fr0 + sr * (mur - cr[0]));
  flux[1] = al * (fl0 * ul + pl + sl * (mul * sm - cl[1])) + ar * (fr0 * ur + pr + sr * (mur * sm - cr[1]));
  flux[2] = al * (fl0 * vl + sl * (mul * vl - cl[2])) + ar * (fr0 * vr + sr * (mur * vr - cr[2]));
  flux[3] = al * (fl0 * wl + sl * (mul * wl - cl[3])) + ar * (fr0 * wr + sr * (mur * wr - cr[3]));
  flux[4] = al * (ul * (el + pl) + sl * (mul * lastl - cl[4])) + ar * (ur * (er + pr) + sr * (mur * lastr - cr[4]));
}

// COMPUTE_EIGENVECTORS (src/flow_operations.f90:3934-3995): left (EL) and
// right (ER) eigenvectors of the x-direction Euler flux Jacobian at the
// arithmetic average of two face-frame states, written with stride `st`:
// EL[(k * 5 + v) * st] (row k), ER[(v * 5 + k) * st] (column k).
__device__ __forceinline__ void char_eigenvectors(double gamma, const double* rl, const double* rr, double* EL,
                                                  double* ER, int st) {
  const double gm1 = gamma - 1.0;
  const double oor1 = 1.0 / rl[0], oor2 = 1.0 / rr[0];
  const double rs = 0.5 * (rl[0] + rr[0]);
  const double us = 0.5 * ((rl[1] * oor1) + (rr[1] * oor2));
  const double vs = 0.5 * ((rl[2] * oor1) + (rr[2] * oor2));
  const double ws = 0.5 * ((rl[3] * oor1) + (rr[3] * oor2));
  const double es = 0.5 * (rl[4] + rr[4]);
  const double vvs = us * us + vs * vs + ws * ws;
  const double vsd = 0.5 * vvs;
  const double ps = gm1 * (es - 0.5 * rs * vvs);
  const double as = sqrt(gamma * ps / rs);
  const double hs = (0.5 * vvs) + ((as * as) / gm1);
  const double R[5][5] = {{1.0, 1.0, 0.0, 0.0, 1.0},
                          {us - as, us, 0.0, 0.0, us + as},
                          {vs, vs, 1.0, 0.0, vs},
                          {ws, ws, 0.0, 1.0, ws},
                          {hs - us * as, 0.5 * vvs, vs, ws, hs + us * as}};
  const double iden = 1.0 / (2.0 * as * hs - 2.0 * as * vsd);
  const double us2 = us * us, vs2 = vs * vs, ws2 = ws * ws;
  const double L[5][5] = {
      {(hs * us + as * us2 + as * vs2 - as * vsd - us * vsd + as * ws2) * iden, (-hs - as * us + vsd) * iden,
       -(as * vs) * iden, -(as * ws) * iden, as * iden},
      {(2.0 * as * hs - 2.0 * as * us2 - 2.0 * as * vs2 - 2.0 * as * ws2) * iden, (2.0 * as * us) * iden,
       (2.0 * as * vs) * iden, (2.0 * as * ws) * iden, (-2.0 * as) * iden},
      {(-2.0 * as * hs * vs + 2.0 * as * vs * vsd) * iden, 0.0, 1.0, 0.0, 0.0},
      {(-2.0 * as * hs * ws + 2.0 * as * vsd * ws) * iden, 0.0, 0.0, 1.0, 0.0},
      {(-(hs * us) + as * us2 + as * vs2 - as * vsd + us * vsd + as * ws2) * iden, (hs - as * us - vsd) * iden,
       -(as * vs) * iden, -(as * ws) * iden, as * iden}};
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      EL[(i * 5 + j) * st] = L[i][j];
      ER[(i * 5 + j) * st] = R[i][j];
    }
}

// Euler flux in the face frame of a conserved state, with its velocity and
// pressure
template <typename S>
__host__ __device__ __forceinline__ void euler_xflux(double gamma, const S* c, S* f, S& u, S& pr) {
  const S r = c[0], ir = 1.0 / r;
  u = c[1] * ir;
  const S v = c[2] * ir, w = c[3] * ir;
  pr = (gamma - 1.0) * (c[4] - 0.5 * r * (u * u + v * v + w * w));
  f[0] = r * u;
  f[1] = r * u * u + pr;
  f[2] = r * u * v;
  f[3] = r * u * w;
  f[4] = u * (c[4] + pr);
}

// Rusanov flux (RUSANOV_RIEMANN_SOLVER, src/riemann.f90:1236-1403):
// 0.5 (FL + FR) - 0.5 max(|uL| + cL, |uR| + cR) (UR - UL).
template <typename S>
__host__ __device__ __forceinline__ void rusanov(double gamma, const S* cl, const S* cr, S* flux) {
  S fl[5], fr[5], ul, ur, pl, pr;
  euler_xflux(gamma, cl, fl, ul, pl);
  euler_xflux(gamma, cr, fr, ur, pr);
  const S sl = fabs(ul) + sqrt(gamma * pl / cl[0]), sr = fabs(ur) + sqrt(gamma * pr / cr[0]);
  const S smax = fmax(fabs(sl), fabs(sr));
#pragma unroll
  for (int k = 0; k < 5; ++k) flux[k] = 0.5 * (fl[k] + fr[k]) - 0.5 * smax * (cr[k] - cl[k]);
}

// HLL flux (HLL_RIEMANN_SOLVER, src/riemann.f90:28-217) with the Davis wave
// speeds SL = min(uL - cL, uR - cR), SR = max(uL + cL, uR + cR): FL when
// SL > 0, FR when SR < 0, else (SR FL - SL FR + SL SR (UR - UL)) / (SR - SL).
template <typename S>
__host__ __device__ __forceinline__ void hll(double gamma, const S* cl, const S* cr, S* flux) {
  S fl[5], fr[5], ul, ur, pl, pr;
  euler_xflux(gamma, cl, fl, ul, pl);
  euler_xflux(gamma, cr, fr, ur, pr);
  const S ccl = sqrt(gamma * pl / cl[0]), ccr = sqrt(gamma * pr / cr[0]);
  const S sl = fmin(ul - ccl, ur - ccr), sr = fmax(ul + ccl, ur + ccr);
  if (value(sl) <= 0.0 && value(sr) >= 0.0) {
    const S id = 1.0 / (sr - sl);
#pragma unroll
    for (int k = 0; k < 5; ++k) flux[k] = (sr * fl[k] - sl * fr[k] + (sl * sr * (cr[k] - cl[k]))) * id;
  } else if (value(sr) <= 0.0) {
#pragma unroll
    for (int k = 0; k < 5; ++k) flux[k] = fr[k];
  } else {
#pragma unroll
    for (int k = 0; k < 5; ++k) flux[k] = fl[k];
  }
}

// Roe flux with the entropy fix of the acoustic waves (ROE_RIEMANN_SOLVER,
// src/riemann.f90:433-632), in the global frame along the face normal n.
template <typename S>
__host__ __device__ __forceinline__ void roe(double gamma, const S* cl, const S* cr, const double* n, S* flux) {
  const double nx = n[0], ny = n[1], nz = n[2];
  const S rL = cl[0], uL = cl[1] / rL, vL = cl[2] / rL, wL = cl[3] / rL;
  const S pL = (gamma - 1.0) * (cl[4] - 0.5 * rL * (uL * uL + vL * vL + wL * wL));
  const S rR = cr[0], uR = cr[1] / rR, vR = cr[2] / rR, wR = cr[3] / rR;
  const S pR = (gamma - 1.0) * (cr[4] - 0.5 * rR * (uR * uR + vR * vR + wR * wR));
  const S qnL = uL * nx + vL * ny + wL * nz, qnR = uR * nx + vR * ny + wR * nz;
  const S aL = sqrt(gamma * pL / rL), aR = sqrt(gamma * pR / rR);
  const S HL = aL * aL / (gamma - 1.0) + 0.5 * (uL * uL + vL * vL + wL * wL);
  const S HR = aR * aR / (gamma - 1.0) + 0.5 * (uR * uR + vR * vR + wR * wR);
  const S RT = sqrt(rR / rL), iRT = 1.0 / (1.0 + RT);
  const S rho = RT * rL, u = (uL + RT * uR) * iRT, v = (vL + RT * vR) * iRT, w = (wL + RT * wR) * iRT;
  const S H = (HL + RT * HR) * iRT;
  const S a = sqrt((gamma - 1.0) * (H - 0.5 * (u * u + v * v + w * w)));
  const S qn = u * nx + v * ny + w * nz;
  const S drho = rR - rL, dp = pR - pL, dqn = qnR - qnL;
  const S ia2 = 1.0 / (a * a);
  const S L1 = (dp - rho * a * dqn) * (0.5 * ia2), L2 = drho - dp * ia2, L3 = (dp + rho * a * dqn) * (0.5 * ia2);
  S ws1 = fabs(qn - a), ws2 = fabs(qn), ws3 = fabs(qn + a);
  if (value(ws1) < 0.2) ws1 = 0.5 * (ws1 * ws1 / 0.2 + 0.2);
  if (value(ws3) < 0.2) ws3 = 0.5 * (ws3 * ws3 / 0.2 + 0.2);
  const S du = uR - uL, dv = vR - vL, dw = wR - wL;
  const S R1[5] = {S(1.0), u - a * nx, v - a * ny, w - a * nz, H - a * qn};
  const S R2[5] = {S(1.0), u, v, w, 0.5 * (u * u + v * v + w * w)};
  const S R3[5] = {S(1.0), u + a * nx, v + a * ny, w + a * nz, H + a * qn};
  const S R4[5] = {S(0.0), du - dqn * nx, dv - dqn * ny, dw - dqn * nz, u * du + v * dv + w * dw - qn * dqn};
  const S fL[5] = {rL * qnL, rL * qnL * uL + pL * nx, rL * qnL * vL + pL * ny, rL * qnL * wL + pL * nz, rL * qnL * HL};
  const S fR[5] = {rR * qnR, rR * qnR * uR + pR * nx, rR * qnR * vR + pR * ny, rR * qnR * wR + pR * nz, rR * qnR * HR};
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const S diss = ws1 * L1 * R1[k] + ws2 * L2 * R2[k] + ws3 * L3 * R3[k] + ws2 * rho * R4[k];
    flux[k] = 0.5 * (fL[k] + fR[k] - diss);
  }
}

// Rotated Roe-HLL flux (rROE_RIEMANN_SOLVER, src/riemann.f90:892-1234):
// HLL along n1 (the velocity-difference direction, or a direction normal to
// n when the velocity jump is below TOLSMALL), Roe along n2 normal to n1 in
// the plane of n and n1, in the global frame.
template <typename S>
__host__ __device__ __forceinline__ void rhll(double gamma, const S* cl, const S* cr, const double* n, S* flux) {
  const double nx = n[0], ny = n[1], nz = n[2];
  const S rL = cl[0], uL = cl[1] / rL, vL = cl[2] / rL, wL = cl[3] / rL;
  const S pL = (gamma - 1.0) * (cl[4] - 0.5 * rL * (uL * uL + vL * vL + wL * wL));
  const S rR = cr[0], uR = cr[1] / rR, vR = cr[2] / rR, wR = cr[3] / rR;
  const S pR = (gamma - 1.0) * (cr[4] - 0.5 * rR * (uR * uR + vR * vR + wR * wR));
  const S aL = sqrt(gamma * pL / rL), aR = sqrt(gamma * pR / rR);
  const S HL = aL * aL / (gamma - 1.0) + 0.5 * (uL * uL + vL * vL + wL * wL);
  const S HR = aR * aR / (gamma - 1.0) + 0.5 * (uR * uR + vR * vR + wR * wR);
  S qnL = uL * nx + vL * ny + wL * nz, qnR = uR * nx + vR * ny + wR * nz;
  const S fL[5] = {rL * qnL, rL * qnL * uL + pL * nx, rL * qnL * vL + pL * ny, rL * qnL * wL + pL * nz, rL * qnL * HL};
  const S fR[5] = {rR * qnR, rR * qnR * uR + pR * nx, rR * qnR * vR + pR * ny, rR * qnR * wR + pR * nz, rR * qnR * HR};
  // n1: the velocity-difference direction, oriented along n
  const S abs_dq = sqrt((uR - uL) * (uR - uL) + (vR - vL) * (vR - vL) + (wR - wL) * (wR - wL));
  S nx1, ny1, nz1;
  if (value(abs_dq) > TOLSMALL) {
    nx1 = (uR - uL) / abs_dq;
    ny1 = (vR - vL) / abs_dq;
    nz1 = (wR - wL) / abs_dq;
  } else {
    const double tx = ny * ny + nz * nz, ty = nz * nz + nx * nx, tz = nx * nx + ny * ny;
    double a1, b1, c1;
    if (tx >= ty && tx >= tz) {
      a1 = 0.0, b1 = -nz, c1 = ny;
    } else if (ty >= tx && ty >= tz) {
      a1 = -nz, b1 = 0.0, c1 = nx;
    } else {
      a1 = -ny, b1 = nx, c1 = 0.0;
    }
    const double t = sqrt(a1 * a1 + b1 * b1 + c1 * c1);
    nx1 = S(a1 / t);
    ny1 = S(b1 / t);
    nz1 = S(c1 / t);
  }
  S alpha1 = nx * nx1 + ny * ny1 + nz * nz1;
  {
    const double sg = copysign(1.0, value(alpha1));
    nx1 = sg * nx1;
    ny1 = sg * ny1;
    nz1 = sg * nz1;
    alpha1 = sg * alpha1;
  }
  // n2 = (n1 x n) x n1, normalised and oriented along n
  const S tx = ny1 * nz - nz1 * ny, ty = nz1 * nx - nx1 * nz, tz = nx1 * ny - ny1 * nx;
  S nx2 = ty * nz1 - tz * ny1, ny2 = tz * nx1 - tx * nz1, nz2 = tx * ny1 - ty * nx1;
  {
    const S t = sqrt(nx2 * nx2 + ny2 * ny2 + nz2 * nz2);
    if (value(t) > 0.0) {
      nx2 = nx2 / t;
      ny2 = ny2 / t;
      nz2 = nz2 / t;
    } else {  // n1 parallel to n: alpha2 = 0 and any n2 normal to n gives the same flux
      const double ax = ny * ny + nz * nz, ay = nz * nz + nx * nx, az = nx * nx + ny * ny;
      double a1, b1, c1;
      if (ax >= ay && ax >= az) {
        a1 = 0.0, b1 = -nz, c1 = ny;
      } else if (ay >= ax && ay >= az) {
        a1 = -nz, b1 = 0.0, c1 = nx;
      } else {
        a1 = -ny, b1 = nx, c1 = 0.0;
      }
      const double q = sqrt(a1 * a1 + b1 * b1 + c1 * c1);
      nx2 = S(a1 / q);
      ny2 = S(b1 / q);
      nz2 = S(c1 / q);
    }
  }
  S alpha2 = nx * nx2 + ny * ny2 + nz * nz2;
  {
    const double sg = copysign(1.0, value(alpha2));
    nx2 = sg * nx2;
    ny2 = sg * ny2;
    nz2 = sg * nz2;
    alpha2 = sg * alpha2;
  }
  const S RT = sqrt(rR / rL), iRT = 1.0 / (1.0 + RT);
  const S rho = RT * rL, u = (uL + RT * uR) * iRT, v = (vL + RT * vR) * iRT, w = (wL + RT * wR) * iRT;
  const S H = (HL + RT * HR) * iRT;
  const S a = sqrt((gamma - 1.0) * (H - 0.5 * (u * u + v * v + w * w)));
  // HLL wave-speed estimates along n1
  S qn = u * nx1 + v * ny1 + w * nz1;
  qnL = uL * nx1 + vL * ny1 + wL * nz1;
  qnR = uR * nx1 + vR * ny1 + wR * nz1;
  const S SLm = fmin(fmin(S(0.0), qn - a), qnL - aL);
  const S SRp = fmax(fmax(S(0.0), qn + a), qnR + aR);
  // Roe dissipation along n2
  qn = u * nx2 + v * ny2 + w * nz2;
  qnL = uL * nx2 + vL * ny2 + wL * nz2;
  qnR = uR * nx2 + vR * ny2 + wR * nz2;
  const S drho = rR - rL, dp = pR - pL, dqn = qnR - qnL;
  const S ia2 = 1.0 / (a * a);
  const S L1 = (dp - rho * a * dqn) * (0.5 * ia2), L2 = drho - dp * ia2, L3 = (dp + rho * a * dqn) * (0.5 * ia2);
  const S eig1 = qn - a, eig2 = qn, eig3 = qn + a;
  S ws1 = fabs(qn - a), ws2 = fabs(qn), ws3 = fabs(qn + a);
  if (value(ws1) < 0.2) ws1 = 0.5 * (ws1 * ws1 / 0.2 + 0.2);
  if (value(ws3) < 0.2) ws3 = 0.5 * (ws3 * ws3 / 0.2 + 0.2);
  const S isd = 1.0 / (SRp - SLm);
  ws1 = alpha2 * ws1 - (alpha1 * 2.0 * SRp * SLm + alpha2 * (SRp + SLm) * eig1) * isd;
  ws2 = alpha2 * ws2 - (alpha1 * 2.0 * SRp * SLm + alpha2 * (SRp + SLm) * eig2) * isd;
  ws3 = alpha2 * ws3 - (alpha1 * 2.0 * SRp * SLm + alpha2 * (SRp + SLm) * eig3) * isd;
  const S ws4 = ws2;
  const S du = uR - uL, dv = vR - vL, dw = wR - wL;
  const S R1[5] = {S(1.0), u - a * nx2, v - a * ny2, w - a * nz2, H - a * qn};
  const S R2[5] = {S(1.0), u, v, w, 0.5 * (u * u + v * v + w * w)};
  const S R3[5] = {S(1.0), u + a * nx2, v + a * ny2, w + a * nz2, H + a * qn};
  const S R4[5] = {S(0.0), du - dqn * nx2, dv - dqn * ny2, dw - dqn * nz2, u * du + v * dv + w * dw - qn * dqn};
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const S diss = ws1 * L1 * R1[k] + ws2 * L2 * R2[k] + ws3 * L3 * R3[k] + ws4 * rho * R4[k];
    flux[k] = (SRp * fL[k] - SLm * fR[k]) * isd - 0.5 * diss;
  }
}

// Roe flux with the two shear waves along explicit face tangents l and m
// (tROE_RIEMANN_SOLVER, src/riemann.f90:634-890), global frame.
template <typename S>
__host__ __device__ __forceinline__ void troe(double gamma, const S* cl, const S* cr, const double* n, S* flux) {
  const double nx = n[0], ny = n[1], nz = n[2];
  double lx, ly, lz;
  {
    const double tx = ny * ny + nz * nz, ty = nz * nz + nx * nx, tz = nx * nx + ny * ny;
    if (tx >= ty && tx >= tz) {
      lx = 0.0, ly = -nz, lz = ny;
    } else if (ty >= tx && ty >= tz) {
      lx = -nz, ly = 0.0, lz = nx;
    } else {
      lx = -ny, ly = nx, lz = 0.0;
    }
    const double t = sqrt(lx * lx + ly * ly + lz * lz);
    lx /= t, ly /= t, lz /= t;
  }
  double mx = ny * lz - nz * ly, my = nz * lx - nx * lz, mz = nx * ly - ny * lx;
  {
    const double t = sqrt(mx * mx + my * my + mz * mz);
    mx /= t, my /= t, mz /= t;
  }
  const S rL = cl[0], uL = cl[1] / rL, vL = cl[2] / rL, wL = cl[3] / rL;
  const S pL = (gamma - 1.0) * (cl[4] - 0.5 * rL * (uL * uL + vL * vL + wL * wL));
  const S rR = cr[0], uR = cr[1] / rR, vR = cr[2] / rR, wR = cr[3] / rR;
  const S pR = (gamma - 1.0) * (cr[4] - 0.5 * rR * (uR * uR + vR * vR + wR * wR));
  const S qnL = uL * nx + vL * ny + wL * nz, qnR = uR * nx + vR * ny + wR * nz;
  const S aL = sqrt(gamma * pL / rL), aR = sqrt(gamma * pR / rR);
  const S HL = aL * aL / (gamma - 1.0) + 0.5 * (uL * uL + vL * vL + wL * wL);
  const S HR = aR * aR / (gamma - 1.0) + 0.5 * (uR * uR + vR * vR + wR * wR);
  const S RT = sqrt(rR / rL), iRT = 1.0 / (1.0 + RT);
  const S rho = RT * rL, u = (uL + RT * uR) * iRT, v = (vL + RT * vR) * iRT, w = (wL + RT * wR) * iRT;
  const S H = (HL + RT * HR) * iRT;
  const S a = sqrt((gamma - 1.0) * (H - 0.5 * (u * u + v * v + w * w)));
  const S qn = u * nx + v * ny + w * nz, ql = u * lx + v * ly + w * lz, qm = u * mx + v * my + w * mz;
  const S drho = rR - rL, dp = pR - pL, dqn = qnR - qnL;
  const S dql = (uR - uL) * lx + (vR - vL) * ly + (wR - wL) * lz;
  const S dqm = (uR - uL) * mx + (vR - vL) * my + (wR - wL) * mz;
  const S ia2 = 1.0 / (a * a);
  const S L1 = (dp - rho * a * dqn) * (0.5 * ia2), L2 = drho - dp * ia2, L3 = (dp + rho * a * dqn) * (0.5 * ia2);
  const S L4 = rho * dql, L5 = rho * dqm;
  S ws1 = fabs(qn - a), ws3 = fabs(qn + a);
  const S ws2 = fabs(qn);
  if (value(ws1) < 0.2) ws1 = 0.5 * (ws1 * ws1 / 0.2 + 0.2);
  if (value(ws3) < 0.2) ws3 = 0.5 * (ws3 * ws3 / 0.2 + 0.2);
  const S R1[5] = {S(1.0), u - a * nx, v - a * ny, w - a * nz, H - a * qn};
  const S R2[5] = {S(1.0), u, v, w, 0.5 * (u * u + v * v + w * w)};
  const S R3[5] = {S(1.0), u + a * nx, v + a * ny, w + a * nz, H + a * qn};
  const S R4[5] = {S(0.0), S(lx), S(ly), S(lz), ql};
  const S R5[5] = {S(0.0), S(mx), S(my), S(mz), qm};
  const S fL[5] = {rL * qnL, rL * qnL * uL + pL * nx, rL * qnL * vL + pL * ny, rL * qnL * wL + pL * nz, rL * qnL * HL};
  const S fR[5] = {rR * qnR, rR * qnR * uR + pR * nx, rR * qnR * vR + pR * ny, rR * qnR * wR + pR * nz, rR * qnR * HR};
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const S diss = ws1 * L1 * R1[k] + ws2 * L2 * R2[k] + ws3 * L3 * R3[k] + ws2 * (L4 * R4[k] + L5 * R5[k]);
    flux[k] = 0.5 * (fL[k] + fR[k] - diss);
  }
}

// The face-frame flux of the configured Riemann solver (iRiemann of
// UCNS3D.DAT, src/flux_p.f90:587-660): 1 HLLC, 2 Rusanov, 9 HLL.
template <typename S>
__host__ __device__ __forceinline__ void riemann_flux(int kind, double gamma, const S* cl, const S* cr, S* flux) {
  if (kind == 2) rusanov(gamma, cl, cr, flux);
  else if (kind == 9) hll(gamma, cl, cr, flux);
  else hllc(gamma, cl, cr, flux);
}

// Venkatakrishnan limiter, SLOPE_LIMITERS case 7 (src/reconstruct_p.f90:3647-3652)
template <typename S>
__host__ __device__ __forceinline__ S venkat(S d2, S umin0, S umax0, double epsi2) {
  if (fabs(value(d2)) <= 0.0) return S(1.0);
  S dmin = copysign(1.0, value(d2)) * (fabs(d2) + TOLSMALL);
  S dplus = value(d2) > 0.0 ? umax0 : umin0;
  return (1.0 / dmin) * (((dplus * dplus + epsi2) * dmin + 2.0 * (dmin * dmin) * dplus) /
                         (dplus * dplus + 2.0 * dmin * dmin + dmin * dplus + epsi2));
}

// SLOPE_LIMITERS (src/reconstruct_p.f90:3421-3945), the limiter code of
// UCNS3D.DAT: 1 Barth-Jespersen, 2/3/9 Michalak's polynomial, 4/8
// Venkatakrishnan, 5 van Albada, 6 van Leer, each with sfd = (bound - mean)
// / d2; 2/3/9 and 4/8 are blended towards 1 where the cell's range is below
// (KAPPA_VEN MINEDGE)^3 (e3 here), 7 is plain Venkatakrishnan.
template <typename S>
__host__ __device__ __forceinline__ S slope_limiter(int kind, S d2, S lo, S hi, double e3) {
  if (kind == 7) return venkat(d2, lo, hi, e3);
  if (fabs(value(d2)) <= 0.0) return S(1.0);
  S psi;
  const bool blend = kind == 2 || kind == 3 || kind == 9 || kind == 4 || kind == 8;
  if (kind == 4 || kind == 8) {
    psi = venkat(d2, lo, hi, e3);
  } else {
    const S sfd = (value(d2) > 0.0 ? hi : lo) / d2;
    if (kind == 1) psi = fmin(S(1.0), sfd);
    else if (kind == 5) psi = (sfd * sfd + sfd) / (sfd * sfd + 1.0);
    else if (kind == 6) psi = 2.0 * sfd / (sfd + 1.0);
    else psi = value(sfd) < 1.5 ? -((4.0 / 27.0) * (sfd * sfd * sfd)) + sfd : S(1.0);
  }
  if (blend) {
    const S du = hi - lo, du2 = du * du;
    S sig;
    if (value(du2) <= e3) {
      sig = S(1.0);
    } else if (value(du2) < 2.0 * e3) {
      const S y = (du2 - e3) / e3;
      sig = (2.0 * (y * y * y)) - (3.0 * (y * y)) + 1.0;
    } else {
      sig = S(0.0);
    }
    psi = sig + (1.0 - sig) * psi;
  }
  return psi;
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
// (t1/t0)^1.5 written as r*sqrt(r).  S: double or a dual number.
template <typename S>
__device__ __forceinline__ void sutherland(const Problem& p, S rho, S pr, S* mu, S* lam) {
  const double suther = 0.412158681;
  S t1 = pr / (rho * p.r_gas);
  double t0 = p.pres / (p.rres * p.r_gas);
  S r = t1 / t0;
  *mu = p.visc * (r * sqrt(r)) * ((t0 + suther * t0) / (t1 + suther * t0));
  *lam = (*mu) * p.r_gas * p.gamma / (p.prandtl * (p.gamma - 1.0));
}

}  // namespace ucg

namespace ucg {

// ------------------------------------------------ async bulk copy helpers
// 1-D bulk copies global -> shared completed on an mbarrier (sm_90+ PTX),
// each CTA copying for itself alone.  Waits are bounded: a wait that gives up
// returns false and the caller records UCG_ETIMEOUT in the health word.
enum : unsigned { HEALTH_TIMEOUT = 2u };

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: `limit` polls (2^22: about a second), then give up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, long limit = 1L << 22) {
  for (long it = 0; it < limit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it > 64) __nanosleep(256);
  }
  return false;
}

}  // namespace ucg

namespace ucg {

// Ghost state of a physical boundary face (BOUNDARYS, src/flow_operations.f90:2860-3375)
// and the viscous face flux (CALCULATE_FLUXESHI_DIFFUSIVE, src/flux_p.f90:1614-1779).
// `bcs` is the free-stream state (primitive) of the inflow/outflow/far-field
// conditions, normally Problem::bc_state.  Codes:
//   1 inflow  (:2883): BOUNDTYPE 0 the free stream; BOUNDTYPE 1 the free stream
//             when |u|/c > 1 at the cell, else the subsonic characteristic state
//   2 outflow (:2972): BOUNDTYPE 0 the cell's own state; BOUNDTYPE 1 that state
//             when |u|/c > 1, else the state at the free-stream pressure
//   3 symmetry, 4 wall (:3102, :3140): normal momentum mirrored; a wall of a
//             Navier-Stokes run (ITESTCASE 4, :3172-3186) mirrors the whole
//             momentum (no slip)
//   6 far field (:3230): inflow or outflow by the sign of the face-frame normal
//             momentum rho*u_n of the cell, supersonic when |rho*u_n| >= c (the
//             reference compares that momentum, not the velocity, with the sound
//             speed), then the inflow or outflow states above
// Subsonic states share the formulas of cases 1 and 2 (bc_sub_in, bc_sub_out).
template <typename S>
__host__ __device__ __forceinline__ void bc_sub_in(double gm, const S* s1, const S* s2, S sps, double nx, double ny,
                                                   double nz, S* cr) {
  S s3[NV];
  s3[4] = 0.5 * (s1[4] + s2[4] - s2[0] * sps * (nx * (s1[1] - s2[1]) + ny * (s1[2] - s2[2]) + nz * (s1[3] - s2[3])));
  s3[0] = s1[0] + (s3[4] - s1[4]) / (sps * sps);
  s3[1] = s1[1] - nx * (s1[4] - s3[4]) / (sps * s2[0]);
  s3[2] = s1[2] - ny * (s1[4] - s3[4]) / (sps * s2[0]);
  s3[3] = s1[3] - nz * (s1[4] - s3[4]) / (sps * s2[0]);
  prim2cons(gm, s3, cr);
}
template <typename S>
__host__ __device__ __forceinline__ void bc_sub_out(double gm, const S* s1, const S* s2, S sps, double nx, double ny,
                                                    double nz, S* cr) {
  S s3[NV];
  s3[4] = s1[4];
  s3[0] = s2[0] + (s3[4] - s2[4]) / (sps * sps);
  s3[1] = s2[1] + nx * (s2[4] - s3[4]) / (sps * s2[0]);
  s3[2] = s2[2] + ny * (s2[4] - s3[4]) / (sps * s2[0]);
  s3[3] = s2[3] + nz * (s2[4] - s3[4]) / (sps * s2[0]);
  prim2cons(gm, s3, cr);
}

template <typename S>
__host__ __device__ __forceinline__ void boundary_ghost(const Problem& p, int code, const double* r, const S* cl, const S* bcs,
                                               S* cr) {
  const double gm = p.gamma;
  const double nx = r[0] * r[3], ny = r[1] * r[3], nz = r[2];
  if (code == 4 && p.governing == 1) {  // Navier-Stokes wall: no slip
    cr[0] = cl[0];
    cr[1] = -cl[1];
    cr[2] = -cl[2];
    cr[3] = -cl[3];
    cr[4] = cl[4];
    return;
  }
  if (code == 3 || code == 4) {  // symmetry / inviscid wall: mirror the normal momentum
    S a[NV], b[NV];
    rot_f(r, cl, a);
    b[0] = a[0];
    b[1] = -a[1];
    b[2] = a[2];
    b[3] = a[3];
    b[4] = a[4];
    rot_b(r, b, cr);
    return;
  }
  S s1[NV], s2[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) s1[k] = bcs[k];
  if (p.boundtype == 0 && (code == 1 || code == 2)) {  // BOUNDTYPE 0: supersonic treatment
    if (code == 1) {
      prim2cons(gm, s1, cr);
    } else {
#pragma unroll
      for (int k = 0; k < NV; ++k) cr[k] = cl[k];
    }
    return;
  }
  cons2prim(gm, cl, s2);
  S sps = sqrt(gm * s2[4] / s2[0]);
  bool in, super;
  if (code == 6) {
    S a[NV];
    rot_f(r, cl, a);
    in = value(a[1]) <= 0.0;
    super = fabs(value(a[1])) >= value(sps);
  } else {
    S vel = sqrt(s2[1] * s2[1] + s2[2] * s2[2] + s2[3] * s2[3]);
    in = code == 1;
    super = value(vel / (sps + TOLSMALL)) > 1.0;
  }
  if (in) {
    if (super) prim2cons(gm, s1, cr);
    else bc_sub_in(gm, s1, s2, sps, nx, ny, nz, cr);
  } else if (super) {
#pragma unroll
    for (int k = 0; k < NV; ++k) cr[k] = cl[k];
  } else {
    bc_sub_out(gm, s1, s2, sps, nx, ny, nz, cr);
  }
}

__device__ __forceinline__ void boundary_ghost(const Problem& p, int code, const double* r, const double* cl,
                                               double* cr) {
  boundary_ghost<double>(p, code, r, cl, p.bc_state, cr);
}

// `damp` multiplies the jump term: LAMX on interior and far-field faces, 0
// on faces with boundary codes 1-4 (flux_p.f90:1872-1874).  S: double or a
// dual number (the discrete adjoint and tangent).
template <typename S>
__device__ __forceinline__ void viscous_flux(const Problem& p, const double* r, double dih, const S* cl, const S* cr,
                                             const S* gl, const S* gr, S* fv, double damp) {
  double nx = r[0] * r[3], ny = r[1] * r[3], nz = r[2];
  double nn[3] = {nx, ny, nz};
  S lv[NV], rv[NV];
  cons2prim(p.gamma, cl, lv);
  cons2prim(p.gamma, cr, rv);
  S mul, mur, laml, lamr;
  sutherland(p, lv[0], lv[4], &mul, &laml);
  sutherland(p, rv[0], rv[4], &mur, &lamr);
  // gradient rows u, v, w, T; stored components are T, u, v, w
  const int src[4] = {1, 2, 3, 0};
  S jump[4] = {rv[1] - lv[1], rv[2] - lv[2], rv[3] - lv[3],
               rv[4] / (rv[0] * p.r_gas) - lv[4] / (lv[0] * p.r_gas)};
  const double vd = (4.0 / 3.0) / fabs(dih);
  S gg[4][3];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      gg[a][k] = (gl[src[a] * 3 + k] + gr[src[a] * 3 + k]) / 2.0 + damp * (vd * nn[k] * jump[a]);
  S lam2 = 0.5 * (laml + lamr), mu2 = 0.5 * (mul + mur);
  S ux = gg[0][0], uy = gg[0][1], uz = gg[0][2];
  S vx = gg[1][0], vy = gg[1][1], vz = gg[1][2];
  S wx = gg[2][0], wy = gg[2][1], wz = gg[2][2];
  S txx = mu2 * ((4.0 / 3.0) * ux - (2.0 / 3.0) * vy - (2.0 / 3.0) * wz);
  S tyy = mu2 * ((4.0 / 3.0) * vy - (2.0 / 3.0) * ux - (2.0 / 3.0) * wz);
  S tzz = mu2 * ((4.0 / 3.0) * wz - (2.0 / 3.0) * ux - (2.0 / 3.0) * vy);
  S txy = mu2 * (uy + vx), txz = mu2 * (wx + uz), tyz = mu2 * (vz + wy);
  S rho12 = 0.5 * (cl[0] + cr[0]);
  S u12 = 0.5 * (cl[1] + cr[1]) / rho12, v12 = 0.5 * (cl[2] + cr[2]) / rho12, w12 = 0.5 * (cl[3] + cr[3]) / rho12;
  S qx = lam2 * gg[3][0], qy = lam2 * gg[3][1], qz = lam2 * gg[3][2];  // -Q
  S fx4 = qx + u12 * txx + v12 * txy + w12 * txz;
  S fy4 = qy + u12 * txy + v12 * tyy + w12 * tyz;
  S fz4 = qz + u12 * txz + v12 * tyz + w12 * tzz;
  fv[0] = S(0.0);
  fv[1] = nx * txx + ny * txy + nz * txz;
  fv[2] = nx * txy + ny * tyy + nz * tyz;
  fv[3] = nx * txz + ny * tyz + nz * tzz;
  fv[4] = nx * fx4 + ny * fy4 + nz * fz4;
}

}  // namespace ucg
