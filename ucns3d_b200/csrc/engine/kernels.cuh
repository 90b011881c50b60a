// Engine kernels: reconstruction (MUSCL / WENO / CWENO with the MUSCL and
// first-order fall-backs), viscous face gradients, face fluxes fused with
// the SSP-RK3 stage update, time step and domain reductions.
#pragma once

#include "device.cuh"
#include "recon2.cuh"

#include "expand.cuh"

namespace ucg {

// ======================================================================
// MUSCL, IORDER = 1 (one quadrature point per face), one thread per cell.
// LEAST_SQUARES (gradients.f90:253-497), MUSCL + Venkatakrishnan
// (reconstruct_p.f90:2286, 1821, 2044, 3421), CHECKSOLX (3245), and for
// Navier-Stokes the viscous LSQ (gradients.f90:502-706) + SOLUTIONTRIAV2.
// VK: the limiter is Venkatakrishnan (LIMITER 7) inline; otherwise the
// SLOPE_LIMITERS code of the configuration, chosen at run time.
// ======================================================================
template <typename T, bool NS, bool VK>
__global__ void __launch_bounds__(128) k_muscl(Problem p, const double* __restrict__ U) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  const int IM = p.imax, W = IM + 1, QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const int nf = p.nfaces[c];
  double u0[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u0[v] = U[c * NV + v];
  double pm[NV];
  cons2prim(p.gamma, u0, pm);
  const double t0 = NS ? pm[4] / (pm[0] * p.r_gas) : 0.0;
  // least squares on stencil 1
  const int64_t grp = c >> 5;
  const int lane = (int)(c & 31);
  const int32_t* st = p.sten + grp * (int64_t)p.admis_max * W * 32 + lane;  // row j at st[j * 32]
  const T* M = (const T*)p.invmat + (grp * p.tstride + p.soff[0]) * 32 + lane;
  T g[3][NV];
  double gvv[3][4];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
#pragma unroll
    for (int v = 0; v < NV; ++v) g[d][v] = T(0);
#pragma unroll
    for (int v = 0; v < 4; ++v) gvv[d][v] = 0.0;
  }
  for (int k = 0; k < IM; ++k) {
    const int64_t y = st[(k + 1) * 32];
    double uy[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uy[v] = U[y * NV + v];
    T m0 = M[(k * 3 + 0) * 32], m1 = M[(k * 3 + 1) * 32], m2 = M[(k * 3 + 2) * 32];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      T du = T(uy[v] - u0[v]);
      g[0][v] += m0 * du;
      g[1][v] += m1 * du;
      g[2][v] += m2 * du;
    }
    if (NS) {
      double py[NV];
      cons2prim(p.gamma, uy, py);
      double ds[4] = {py[4] / (py[0] * p.r_gas) - t0, py[1] - pm[1], py[2] - pm[2], py[3] - pm[3]};
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        gvv[0][v] += (double)m0 * ds[v];
        gvv[1][v] += (double)m1 * ds[v];
        gvv[2][v] += (double)m2 * ds[v];
      }
    }
  }
  // bounds from the cell and its face neighbours (FIND_BOUNDS, strict)
  double umin[NV], umax[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) umin[v] = umax[v] = u0[v];
  for (int f = 0; f < nf; ++f) {
    const int64_t nb = p.neigh[c * MF + f];
    if (nb < 0) continue;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double un = U[nb * NV + v];
      umin[v] = fmin(umin[v], un);
      umax[v] = fmax(umax[v], un);
    }
  }
  // interleaved over 32-cell groups: element j at [j * 32]
  const T* qp = (const T*)p.qpts + (c >> 5) * (int64_t)MF * QS * 3 * 32 + (c & 31);
  const T* bm = (const T*)p.bmean + (c >> 5) * 3 * 32 + (c & 31);
  const double epsi2 = (p.kappa_ven * p.minedge[c]) * (p.kappa_ven * p.minedge[c]) * (p.kappa_ven * p.minedge[c]);
  // unlimited face value minus the mean (recomputed rather than stored: three terms)
  auto face_d = [&](int f, int v) -> double {
    T b0 = qp[(f * QS * 3 + 0) * 32] - bm[0], b1 = qp[(f * QS * 3 + 1) * 32] - bm[32],
      b2 = qp[(f * QS * 3 + 2) * 32] - bm[64];
    T res = b0 * g[0][v] + b1 * g[1][v] + b2 * g[2][v];
    return (u0[v] + (double)res) - u0[v];
  };
  double slope[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) slope[v] = TOLBIG;
  for (int f = 0; f < nf; ++f)
#pragma unroll
    for (int v = 0; v < NV; ++v)
      slope[v] = fmin(slope[v], VK ? venkat(face_d(f, v), umin[v] - u0[v], umax[v] - u0[v], epsi2)
                                   : slope_limiter(p.limiter, face_d(f, v), umin[v] - u0[v], umax[v] - u0[v], epsi2));
  // limited face values and CHECKSOLX
  bool first = false;
  for (int f = 0; f < nf; ++f) {
    double uf[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uf[v] = u0[v] + face_d(f, v) * slope[v];
    first = first || jump_bad(p.gamma, pm, uf, 0.95);
  }
  T* out = (T*)p.dul + c * (int64_t)MF * QS * NV;
  for (int f = 0; f < nf; ++f)
#pragma unroll
    for (int v = 0; v < NV; ++v) out[f * QS * NV + v] = first ? T(0) : T(face_d(f, v) * slope[v]);
  if (NS) {
    // face gradients: d/dxi of the linear basis is the unit vector, then
    // AINVJT = INVCCJAC^T (SOLUTIONTRIAV2)
    const double* J = p.jinv + c * 9;
    double gr[4][3];
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int k = 0; k < 3; ++k) gr[v][k] = J[0 * 3 + k] * gvv[0][v] + J[1 * 3 + k] * gvv[1][v] + J[2 * 3 + k] * gvv[2][v];
    double* o = p.ulv + c * (int64_t)MF * QS * 12;
    for (int f = 0; f < nf; ++f)
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) o[f * QS * 12 + v * 3 + k] = gr[v][k];
  }
}

// ======================================================================
// Face fluxes fused with the RK stage update.  Eight lanes per cell, lane f
// integrates face f; the face sums are added in face order
// (CALCULATE_FLUXESHI_CONVECTIVE flux_p.f90:478, CALCULATE_FLUXESHI_DIFFUSIVE
// flux_p.f90:1520), then RUNGE_KUTTA3 (time_p.f90:885-1027).
// MODE 0: write the residual; MODE 1/2/3: RK stage 1/2/3.
// ======================================================================
// One thread per owned face (the cell with the smaller index, or the only
// cell of a boundary face): the Riemann flux RK (iRiemann: 1 HLLC, 2
// Rusanov, 3 Roe, 4 rotated Roe-HLL, 5 t-Roe, 9 HLL) and viscous fluxes over the
// face's points,
// weighted by w_q * area.  The neighbour's face gets the negated sums: HLLC
// and the viscous flux are antisymmetric under swapping the two states and
// flipping the normal, so each interior face is evaluated once instead of
// twice as in the reference's per-cell loop.
// threads per block of the face kernel: 64 lets more warps share an SM at
// its 150 registers (64^3 WENO5 stage, B200: 0.51 ms against 0.66 ms at 256)
#ifndef UCG_FACE_BLOCK
#define UCG_FACE_BLOCK 64
#endif
// Navier-Stokes: six blocks per SM (168 registers instead of 202): 64^3
// MUSCL TGV step 1.278 -> 1.224 ms mixed, 1.334 -> 1.290 ms FP64, 2.1 M-cell
// CWENO4 57.3 -> 56.2 ms; eight (128 registers) gained less.  Euler keeps
// the compiler's choice (eight blocks changed the 64^3 WENO5 step by 0.5 %).
template <typename T, bool NS, int RK>
__global__ void __launch_bounds__(UCG_FACE_BLOCK, NS ? 6 : 1) k_face(Problem p, const double* __restrict__ Uc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.nown) return;
  const int32_t code = p.own[i];
  const int64_t c = code >> 3;
  const int f = code & 7;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  double u0[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u0[v] = Uc[c * NV + v];
  const int64_t nb = p.neigh[c * MF + f];
  if (p.msel && !(p.msel[c] || (nb >= 0 && p.msel[nb]))) return;  // MOOD: faces of the recomputed cells
  const int ft = p.ftype[c * MF + f];
  const int nq = face_nq(p, ft);
  const int nf = p.nface[c * MF + f];
  double r[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) r[k] = p.rot[(c * MF + f) * 4 + k];
  const double area = p.area[c * MF + f];
  double un[NV];
  if (nb >= 0)
#pragma unroll
    for (int v = 0; v < NV; ++v) un[v] = Uc[nb * NV + v];
  const T* dl = (const T*)p.dul + (c * MF + f) * QS * NV;
  const T* dr = nb >= 0 ? (const T*)p.dul + (nb * MF + nf) * QS * NV : nullptr;
  const uint8_t* qpm = p.qperm + (c * MF + f) * QS;
  double god[NV] = {0, 0, 0, 0, 0}, gvis[NV] = {0, 0, 0, 0, 0};
  for (int q = 0; q < nq; ++q) {
    double cl[NV], cr[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) cl[v] = u0[v] + (double)dl[q * NV + v];
    const int qq = qpm[q];
    if (nb >= 0) {
#pragma unroll
      for (int v = 0; v < NV; ++v) cr[v] = un[v] + (double)dr[qq * NV + v];
    } else {
      boundary_ghost(p, p.bc[c * MF + f], r, cl, cr);
    }
    double fl[NV];
    if constexpr (RK >= 3 && RK <= 5) {  // Roe family: global frame, face normal
      const double nrm[3] = {r[0] * r[3], r[1] * r[3], r[2]};
      if constexpr (RK == 3) roe(p.gamma, cl, cr, nrm, fl);
      else if constexpr (RK == 4) rhll(p.gamma, cl, cr, nrm, fl);
      else troe(p.gamma, cl, cr, nrm, fl);
    } else {
      double a[NV], b[NV], h[NV];
      rot_f(r, cr, b);
      rot_f(r, cl, a);
      riemann_flux(RK, p.gamma, a, b, h);
      rot_b(r, h, fl);
    }
    const double ws = face_weight(p, ft, q) * area;
#pragma unroll
    for (int v = 0; v < NV; ++v) god[v] = god[v] + fl[v] * ws;
    if (NS) {
      // both sides' face-point gradients as six 16-byte loads each; the WENO
      // path stores their average once per face point (both pointers at it:
      // (g + g) / 2 is g exactly).  On a physical boundary face the ghost
      // side takes the cell's own gradient (CALCULATE_BOUNDED_VISCOUS,
      // dg_functions.f90:1179-1300) and faces with codes 1-4 drop the jump
      // term (flux_p.f90:1872-1874).
      const double2* gl2 = (const double2*)(p.fgrad ? p.fgrad + (i * QS + q) * 12
                                                    : p.ulv + ((c * MF + f) * QS + q) * 12);
      const double2* gr2 = (const double2*)(p.fgrad ? p.fgrad + (i * QS + q) * 12
                                                    : nb >= 0 ? p.ulv + ((nb * MF + nf) * QS + qq) * 12
                                                              : p.ulv + ((c * MF + f) * QS + q) * 12);
      const int code = nb >= 0 ? 0 : p.bc[c * MF + f];
      double gl[12], gr[12];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double2 a2 = gl2[k], b2 = gr2[k];
        gl[2 * k] = a2.x;
        gl[2 * k + 1] = a2.y;
        gr[2 * k] = b2.x;
        gr[2 * k + 1] = b2.y;
      }
      double fv[NV];
      viscous_flux(p, r, p.dih[c * MF + f], cl, cr, gl, gr, fv, code >= 1 && code <= 4 ? 0.0 : p.lamx);
#pragma unroll
      for (int v = 0; v < NV; ++v) gvis[v] = gvis[v] + fv[v] * ws;
    }
  }
  double* o = p.fflux + (c * MF + f) * NV;
#pragma unroll
  for (int v = 0; v < NV; ++v) o[v] = god[v];
  if (NS) {
    double* ov = p.vflux + (c * MF + f) * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) ov[v] = gvis[v];
  }
  if (nb >= 0) {
    double* o2 = p.fflux + (nb * MF + nf) * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) o2[v] = -god[v];
    if (NS) {
      double* ov2 = p.vflux + (nb * MF + nf) * NV;
#pragma unroll
      for (int v = 0; v < NV; ++v) ov2[v] = -gvis[v];
    }
  }
}

// Per-cell sum of the face fluxes in face order (convective first, then the
// viscous ones subtracted, as CALCULATE_FLUXESHI_CONVECTIVE/_DIFFUSIVE add
// them to RHS) and the RUNGE_KUTTA3 stage update (time_p.f90:885-1027).
// MODE 0: write the residual; MODE 1/2/3: RK stage 1/2/3.
// CHK: test the new state (HEALTH_NONPHYS); MOOD's candidate states are
// tested after the cascades instead
template <bool NS, int MODE, bool CHK = true>
__global__ void __launch_bounds__(256) k_update(Problem p, const double* __restrict__ Uc, const double* Un,
                                                double* Uout, double dt_host) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  const int nf = p.nfaces[c];
  double R[NV] = {0, 0, 0, 0, 0};
  for (int f = 0; f < nf; ++f)
#pragma unroll
    for (int v = 0; v < NV; ++v) R[v] = R[v] + p.fflux[(c * MF + f) * NV + v];
  if (NS)
    for (int f = 0; f < nf; ++f)
#pragma unroll
      for (int v = 0; v < NV; ++v) R[v] = R[v] - p.vflux[(c * MF + f) * NV + v];
  if (MODE == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) p.rhs[c * NV + v] = R[v];
    return;
  }
  const double dt = p.dt_dev ? *p.dt_dev : dt_host;
  const double oov = 1.0 / p.vol[c];
  double out[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double rr = dt * (R[v] * oov);
    if (MODE == 1) out[v] = Un[c * NV + v] - rr;
    else if (MODE == 2) out[v] = (3.0 / 4.0) * Un[c * NV + v] + (1.0 / 4.0) * Uc[c * NV + v] - (1.0 / 4.0) * rr;
    else out[v] = (1.0 / 3.0) * Un[c * NV + v] + (2.0 / 3.0) * Uc[c * NV + v] - (2.0 / 3.0) * rr;
  }
  if (CHK) {
    double pr[NV];
    cons2prim(p.gamma, out, pr);
    if (!(pr[0] > 0.0) || !(pr[4] > 0.0) || !isfinite(out[4])) atomicOr(p.health, HEALTH_NONPHYS);
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) Uout[c * NV + v] = out[v];
}

// ======================================================================
// MOOD (RUNGE_KUTTA3_MOOD, time_p.f90:582-880; mood.f90), Euler only.
// After a stage's candidate Uk: per cascade, PAD_NAD flags the cells whose
// candidate is not admissible, FIX_LIST adds their face neighbours, the
// faces of the selected cells are recomputed (first cascade: MUSCL on the
// selected reduced cells; second: the flagged cells at first order, their
// stage-input mean on every face) and the selected cells' stage is redone.
// ======================================================================

// PAD_NAD (mood.f90:35-330): PAD if the candidate's density or pressure is
// not positive (or NaN); else NAD if its density or energy leaves the
// bounds of the stage-input state over the cell and its face neighbours
// (interior and periodic faces), widened by max(d1, d2 * (max - min)) in
// the relaxed mode.  p.mood[c] = PAD or NAD.
__global__ void k_mood_detect(Problem p, const double* __restrict__ Uc, const double* __restrict__ Uk, double d1,
                              double d2, int relaxed) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  double u[NV], pr[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u[v] = Uk[c * NV + v];
  cons2prim(p.gamma, u, pr);
  bool bad = !(pr[0] > 0.0) || !(pr[4] > 0.0);
  if (!bad) {
    constexpr int VS[2] = {0, NV - 1};  // density and energy
    double lo[2], hi[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) lo[k] = hi[k] = Uc[c * NV + VS[k]];
    const int nf = p.nfaces[c];
    for (int f = 0; f < nf; ++f) {
      const int64_t nb = p.neigh[c * MF + f];
      if (nb < 0) continue;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const double un = Uc[nb * NV + VS[k]];
        lo[k] = fmin(lo[k], un);
        hi[k] = fmax(hi[k], un);
      }
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const double x = u[VS[k]];
      if (relaxed) {
        const double dl = fmax(d1, d2 * (hi[k] - lo[k]));
        bad = bad || x < lo[k] - dl || x > hi[k] + dl;
      } else {
        bad = bad || x < lo[k] || x > hi[k];
      }
    }
  }
  p.mood[c] = bad ? 1 : 0;
}

// FIX_LIST (mood.f90:440-518): sel[c] = the cell or a face neighbour
// (interior and periodic faces) is flagged; mus (first cascade) = sel and
// the cell's reconstruction was reduced (MUSCL, mood.f90:353 with
// reconstruct_p.f90:2306-2315)
__global__ void k_mood_fix(Problem p, int8_t* __restrict__ sel, int8_t* __restrict__ mus) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  bool s = p.mood[c] != 0;
  const int nf = p.nfaces[c];
  for (int f = 0; f < nf; ++f) {
    const int64_t nb = p.neigh[c * MF + f];
    if (nb >= 0 && p.mood[nb]) s = true;
  }
  sel[c] = s ? 1 : 0;
  if (mus) mus[c] = (s && p.wflag[c]) ? 1 : 0;
}

// second cascade: the flagged cells' face values become their stage-input
// mean (CALCULATE_FLUXESHI_CONVECTIVE_MOOD with CASCADE 2, flux_p.f90:2722-2733)
template <typename T>
__global__ void k_mood_first(Problem p) {
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const int64_t W = (int64_t)MF * QS * NV;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n * W) return;
  if (p.mood[i / W]) ((T*)p.dul)[i] = T(0);
}

// the stage redone on the selected cells (p.msel) from the recomputed face
// fluxes, the other cells keep the candidate Uk; FIN (second cascade): into
// Uo, MOOD_O and the HEALTH_NONPHYS test of every cell
template <int MODE, bool FIN>
__global__ void __launch_bounds__(256) k_mood_update(Problem p, const double* __restrict__ Uc, const double* Un,
                                                     const double* Uk, double* Uo, const int8_t* __restrict__ sel1,
                                                     double dt_host) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  double out[NV];
  if (p.msel[c]) {
    const int nf = p.nfaces[c];
    double R[NV] = {0, 0, 0, 0, 0};
    for (int f = 0; f < nf; ++f)
#pragma unroll
      for (int v = 0; v < NV; ++v) R[v] = R[v] + p.fflux[(c * MF + f) * NV + v];
    const double dt = p.dt_dev ? *p.dt_dev : dt_host;
    const double oov = 1.0 / p.vol[c];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double rr = dt * (R[v] * oov);
      if (MODE == 1) out[v] = Un[c * NV + v] - rr;
      else if (MODE == 2) out[v] = (3.0 / 4.0) * Un[c * NV + v] + (1.0 / 4.0) * Uc[c * NV + v] - (1.0 / 4.0) * rr;
      else out[v] = (1.0 / 3.0) * Un[c * NV + v] + (2.0 / 3.0) * Uc[c * NV + v] - (2.0 / 3.0) * rr;
    }
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = Uk[c * NV + v];
  }
  if (FIN) {
    double pr[NV];
    cons2prim(p.gamma, out, pr);
    if (!(pr[0] > 0.0) || !(pr[4] > 0.0) || !isfinite(out[4])) atomicOr(p.health, HEALTH_NONPHYS);
    p.mord[c] = (int8_t)(p.msel[c] ? 1 : sel1[c] ? 2 : p.iorder + 1);
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) Uo[c * NV + v] = out[v];
}

// ======================================================================
// CALCULATE_CFL (time_p.f90:27-191): dt = min over cells; positive doubles
// order like their bit patterns, so atomicMin on the bits is exact.
// ======================================================================
__global__ void k_dt_init(double* dt) { *dt = TOLBIG; }

__global__ void k_cfl(Problem p, const double* __restrict__ U, double ccfl, double* dt) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double d = TOLBIG;
  if (c < p.n) {
    double pr[NV];
    cons2prim(p.gamma, U + c * NV, pr);
    double agrt = sqrt(pr[4] * p.gamma / pr[0]);
    double veln = fmax(fmax(fabs(pr[1]), fabs(pr[2])), fabs(pr[3])) + agrt;
    double me = p.minedge[c];
    if (p.governing == 1) {
      double mu, lam;
      sutherland(p, pr[0], pr[4], &mu, &lam);
      d = ccfl * (1.0 / (fabs(veln) / me + 0.5 * (lam + mu) / (me * me)));
    } else {
      d = ccfl * (me / fabs(veln));
    }
    if (!(d > 0.0)) d = TOLBIG;  // unphysical states are reported by the health word
  }
  __shared__ double s[256];
  s[threadIdx.x] = d;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) s[threadIdx.x] = fmin(s[threadIdx.x], s[threadIdx.x + k]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    atomicMin((unsigned long long*)dt, (unsigned long long)__double_as_longlong(s[0]));
}

// Domain sums, deterministic two-pass tree (time_p.f90:4145-4198)
__global__ void k_reduce_partial(Problem p, const double* __restrict__ U, int what, double* partial) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (c < p.n) {
    const double* u = U + c * NV;
    double x;
    if (what == UCG_REDUCE_ENSTROPHY) {
      // cell-centre velocity gradients g[i][j] = du_i/dx_j: the viscous
      // least-squares face gradients of a linear polynomial (face 0, point 0)
      const double* g = p.ulv + c * (int64_t)MF * 12 + 3;
      double on = 0.0;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const double d = g[i * 3 + j] - g[j * 3 + i];
          on += d * d;
        }
      x = u[0] * 0.5 * (0.5 * (on * u[0]));
    } else {
      x = what == UCG_REDUCE_KE ? 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]
                                : (what == UCG_REDUCE_MASS ? u[0] : u[4]);
    }
    v = p.vol[c] * x;
  }
  __shared__ double s[256];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

__global__ void k_reduce_final(const double* partial, int64_t np, double* out) {
  __shared__ double s[1024];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < np; i += blockDim.x) acc += partial[i];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

// ======================================================================
// Table upload: per-cell rows dst[c][0..len) from src[table_id[c]] (or
// src[c - first] without ids), converted to the engine precision.
// [n][5] rows between orders: GATHER dst[c] = src[map[c]], else the
// scatter dst[map[c]] = src[c] (map = the device-to-caller cell map).
template <bool GATHER>
__global__ void k_perm_rows(const int32_t* __restrict__ map, const double* __restrict__ src, double* __restrict__ dst,
                            int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * NV) return;
  const int64_t c = i / NV, v = i - c * NV, o = map[c];
  if (GATHER) dst[i] = src[o * NV + v];
  else dst[o * NV + v] = src[i];
}

}  // namespace ucg
