// Engine kernels: reconstruction (MUSCL / WENO / CWENO with the MUSCL and
// first-order fall-backs), viscous face gradients, face fluxes fused with
// the SSP-RK3 stage update, time step and domain reductions.
#pragma once

#include "device.cuh"

namespace ucg {

// ======================================================================
// MUSCL, IORDER = 1 (one quadrature point per face), one thread per cell.
// LEAST_SQUARES (gradients.f90:253-497), MUSCL + Venkatakrishnan
// (reconstruct_p.f90:2286, 1821, 2044, 3421), CHECKSOLX (3245), and for
// Navier-Stokes the viscous LSQ (gradients.f90:502-706) + SOLUTIONTRIAV2.
// ======================================================================
template <typename T, bool NS>
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
  const int32_t* st = p.sten + c * (int64_t)p.admis_max * W;
  const T* M = (const T*)p.invmat + c * (int64_t)p.admis_max * IM * 3;
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
    const int64_t y = st[k + 1];
    double uy[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uy[v] = U[y * NV + v];
    T m0 = M[k * 3 + 0], m1 = M[k * 3 + 1], m2 = M[k * 3 + 2];
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
  const T* qp = (const T*)p.qpts + c * (int64_t)MF * QS * 3;
  const T* bm = (const T*)p.bmean + c * 3;
  const double epsi2 = (p.kappa_ven * p.minedge[c]) * (p.kappa_ven * p.minedge[c]) * (p.kappa_ven * p.minedge[c]);
  double d2[MF][NV], slope[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) slope[v] = TOLBIG;
  for (int f = 0; f < MF; ++f) {
    if (f >= nf) break;
    T b0 = qp[f * QS * 3 + 0] - bm[0], b1 = qp[f * QS * 3 + 1] - bm[1], b2 = qp[f * QS * 3 + 2] - bm[2];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      T res = b0 * g[0][v] + b1 * g[1][v] + b2 * g[2][v];
      double usol = u0[v] + (double)res;
      double dd = usol - u0[v];
      d2[f][v] = dd;
      slope[v] = fmin(slope[v], venkat(dd, umin[v] - u0[v], umax[v] - u0[v], epsi2));
    }
  }
  // limited face values and CHECKSOLX
  bool first = false;
  for (int f = 0; f < nf; ++f) {
    double uf[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      d2[f][v] = d2[f][v] * slope[v];
      uf[v] = u0[v] + d2[f][v];
    }
    first = first || jump_bad(p.gamma, pm, uf, 0.95);
  }
  T* out = (T*)p.dul + c * (int64_t)MF * QS * NV;
  for (int f = 0; f < nf; ++f)
#pragma unroll
    for (int v = 0; v < NV; ++v) out[f * QS * NV + v] = first ? T(0) : T(d2[f][v]);
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
// WENO / CWENO, cooperative: a thread block reconstructs `cpc` cells.
// LEAST_SQUARES -> WENOWEIGHTS/CP_RECONSTRUCTION (reconstruct_p.f90:407-1250)
// -> CHECKSOL (3126) -> MUSCL on flagged cells -> CHECKSOLX (3245).
// ======================================================================
struct WenoSmem {
  int u0, du, G, g1, S, S2, gh, w, dul, psi, bnd, slope, flag, total;
};

template <typename T>
__host__ __device__ inline WenoSmem weno_smem_layout(int cpc, int A, int IM, int ID, int ID2, int QS, bool cw) {
  WenoSmem s;
  int off = 0;
  auto take = [&](int bytes) {
    int o = off;
    off += (bytes + 15) & ~15;
    return o;
  };
  s.u0 = take(cpc * NV * 8);
  int du_bytes = cpc * A * IM * NV * (int)sizeof(T);
  int psi_bytes = cpc * MF * QS * NV * 8;
  s.du = take(du_bytes > psi_bytes ? du_bytes : psi_bytes);
  s.psi = s.du;  // the gathered differences are dead once G is formed
  s.G = take(cpc * A * ID * NV * (int)sizeof(T));
  s.g1 = take(cw ? cpc * ID * NV * (int)sizeof(T) : 0);
  s.S = take(cpc * ID * ID * (int)sizeof(T));
  s.S2 = take(cw ? cpc * ID2 * ID2 * (int)sizeof(T) : 0);
  s.gh = take(cpc * ID * NV * (int)sizeof(T));
  s.w = take(cpc * A * NV * 8);
  s.dul = take(cpc * MF * QS * NV * (int)sizeof(T));
  s.bnd = take(cpc * 2 * NV * 8);
  s.slope = take(cpc * NV * 8);
  s.flag = take(cpc * 2 * 4);
  s.total = off;
  return s;
}

template <int P, typename T>
__global__ void __launch_bounds__(256) k_weno(Problem p, const double* __restrict__ U, int cpc) {
  constexpr int ID = Deg<P>::ideg;
  const int A = p.admis_max, IM = p.imax, W = IM + 1;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const bool cw = p.ees == 5;
  const bool weno = p.scheme == 3;  // scheme 2: MUSCL with a degree-P polynomial
  const int ID2 = p.ideg2, IM2 = p.imax2;
  extern __shared__ __align__(16) unsigned char smem[];
  const WenoSmem L = weno_smem_layout<T>(cpc, A, IM, ID, ID2, QS, cw);
  double* s_u0 = (double*)(smem + L.u0);
  T* s_du = (T*)(smem + L.du);
  double* s_psi = (double*)(smem + L.psi);
  T* s_G = (T*)(smem + L.G);
  T* s_g1 = (T*)(smem + L.g1);
  T* s_S = (T*)(smem + L.S);
  T* s_S2 = (T*)(smem + L.S2);
  T* s_gh = (T*)(smem + L.gh);
  double* s_w = (double*)(smem + L.w);
  T* s_dul = (T*)(smem + L.dul);
  double* s_bnd = (double*)(smem + L.bnd);
  double* s_slope = (double*)(smem + L.slope);
  int* s_flag = (int*)(smem + L.flag);  // [cpc][2]: reduce, first order

  const int64_t c0 = (int64_t)blockIdx.x * cpc;
  const int nc = (int)((p.n - c0) < cpc ? (p.n - c0) : cpc);
  const int tid = threadIdx.x, nt = blockDim.x;
  const T* IND = (const T*)p.ind;
  const T* IND2 = (const T*)p.ind2;

  for (int i = tid; i < nc * NV; i += nt) s_u0[i] = U[c0 * NV + i];
  if (weno)
    for (int i = tid; i < nc * ID * ID; i += nt) s_S[i] = IND[c0 * ID * ID + i];
  if (cw)
    for (int i = tid; i < nc * ID2 * ID2; i += nt) s_S2[i] = IND2[c0 * ID2 * ID2 + i];
  for (int i = tid; i < nc * 2; i += nt) s_flag[i] = 0;
  __syncthreads();

  // ---- gather U_k - U_i for every stencil cell
  for (int i = tid; i < nc * A * IM; i += nt) {
    int cl = i / (A * IM), r = i - cl * (A * IM), ll = r / IM, k = r - ll * IM;
    int64_t c = c0 + cl;
    int nk = (cw && ll > 0) ? IM2 : IM;
    T* o = s_du + (size_t)i * NV;
    if (ll < p.admis[c] && k < nk) {
      int64_t y = p.sten[(c * A + ll) * W + k + 1];
#pragma unroll
      for (int v = 0; v < NV; ++v) o[v] = T(U[y * NV + v] - s_u0[cl * NV + v]);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) o[v] = T(0);
    }
  }
  __syncthreads();

  // ---- least squares: G[ll][d][v] = sum_k invmat[ll][k][d] du[ll][k][v]
  for (int i = tid; i < nc * A * ID; i += nt) {
    int cl = i / (A * ID), r = i - cl * (A * ID), ll = r / ID, d = r - ll * ID;
    int64_t c = c0 + cl;
    bool low = cw && ll > 0;
    int nk = low ? IM2 : IM, nd = low ? ID2 : ID;
    T acc[NV] = {T(0), T(0), T(0), T(0), T(0)};
    if (ll < p.admis[c] && d < nd) {
      const T* M = low ? (const T*)p.invmat2 + ((c * A + ll) * (int64_t)IM2) * ID2 + d
                       : (const T*)p.invmat + ((c * A + ll) * (int64_t)IM) * ID + d;
      const T* du = s_du + (size_t)(cl * A + ll) * IM * NV;
#pragma unroll 8
      for (int k = 0; k < nk; ++k) {
        T m = M[(int64_t)k * nd];
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] += m * du[k * NV + v];
      }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) s_G[(size_t)i * NV + v] = acc[v];
  }
  __syncthreads();

  // ---- CWENO: central polynomial with the low-order part removed (reconstruct_p.f90:956-965)
  if (cw) {
    for (int i = tid; i < nc * ID * NV; i += nt) {
      int cl = i / (ID * NV), r = i - cl * (ID * NV), d = r / NV, v = r - d * NV;
      int adm = p.admis[c0 + cl];
      double lc1 = 1.0 - 1.0 / p.lwci;
      double lk = adm > 1 ? (1.0 - lc1) / (adm - 1) : 0.0;
      T g3 = T(0);
      if (d < ID2)
        for (int ll = 1; ll < adm; ++ll) g3 = g3 + T(lk) * s_G[((size_t)(cl * A + ll) * ID + d) * NV + v];
      s_g1[i] = T(1.0 / lc1) * (s_G[((size_t)(cl * A) * ID + d) * NV + v] - g3);
    }
    __syncthreads();
  }

  // ---- smoothness indicators IS = g^T S g
  for (int i = tid; weno && i < nc * A * NV; i += nt) {
    int cl = i / (A * NV), r = i - cl * (A * NV), ll = r / NV, v = r - ll * NV;
    if (ll >= p.admis[c0 + cl]) continue;
    bool low = cw && ll > 0;
    int nd = low ? ID2 : ID;
    const T* S = low ? s_S2 + cl * ID2 * ID2 : s_S + cl * ID * ID;
    const T* gg = (cw && ll == 0) ? s_g1 + (size_t)cl * ID * NV : s_G + (size_t)(cl * A + ll) * ID * NV;
    T is = T(0);
    for (int d = 0; d < nd; ++d) {
      T sg = T(0);
      for (int e = 0; e < nd; ++e) sg += S[d * nd + e] * gg[e * NV + v];
      is += gg[d * NV + v] * sg;
    }
    s_w[i] = (double)is;
  }
  __syncthreads();

  // ---- nonlinear weights (FP64: eps^4 underflows FP32)
  for (int i = tid; weno && i < nc * NV; i += nt) {
    int cl = i / NV, v = i - cl * NV;
    int adm = p.admis[c0 + cl];
    double* w = s_w + cl * A * NV;
    double lam0, lamk;
    if (cw) {
      lam0 = 1.0 - 1.0 / p.lwci;
      lamk = adm > 1 ? (1.0 - lam0) / (adm - 1) : 0.0;
    } else {
      lam0 = p.lwci;
      lamk = 1.0;
    }
    double sum = 0.0, tau = 0.0;
    if (cw && p.wenoz) {
      for (int ll = 0; ll < adm; ++ll) tau += fabs(w[0 * NV + v] - w[ll * NV + v]);
      tau = tau / (adm - 1);
    }
    for (int ll = 0; ll < adm; ++ll) {
      double e = p.weno_eps + w[ll * NV + v];
      double lam = ll == 0 ? lam0 : lamk;
      double wt;
      if (cw && p.wenoz) {
        double q = tau / e;
        q = q * q;
        wt = lam * (1.0 + q * q);
      } else {
        double e2 = e * e;
        wt = lam / (e2 * e2);
      }
      w[ll * NV + v] = wt;
      sum += wt;
    }
    for (int ll = 0; ll < adm; ++ll) w[ll * NV + v] = w[ll * NV + v] / sum;
  }
  __syncthreads();

  // ---- combined polynomial: sum of weights times stencil polynomials
  for (int i = tid; weno && i < nc * ID * NV; i += nt) {
    int cl = i / (ID * NV), r = i - cl * (ID * NV), d = r / NV, v = r - d * NV;
    int adm = p.admis[c0 + cl];
    const double* w = s_w + cl * A * NV;
    const T* g0 = cw ? s_g1 + (size_t)cl * ID * NV : s_G + (size_t)(cl * A) * ID * NV;
    T acc = T(w[v]) * g0[d * NV + v];
    for (int ll = 1; ll < adm; ++ll)
      if (!cw || d < ID2) acc += T(w[ll * NV + v]) * s_G[((size_t)(cl * A + ll) * ID + d) * NV + v];
    s_gh[i] = acc;
  }
  __syncthreads();

  // ---- face values and CHECKSOL
  const T* QP = (const T*)p.qpts;
  const T* BM = (const T*)p.bmean;
  for (int i = tid; i < nc * MF * QS; i += nt) {
    int cl = i / (MF * QS), r = i - cl * (MF * QS), f = r / QS, q = r - f * QS;
    int64_t c = c0 + cl;
    T* o = s_dul + (size_t)i * NV;
    if (f >= p.nfaces[c] || q >= face_nq(p, p.ftype[c * MF + f])) {
#pragma unroll
      for (int v = 0; v < NV; ++v) o[v] = T(0);
      continue;
    }
    const T* xi = QP + ((c * MF + f) * QS + q) * 3;
    T b[ID];
    monomials<P, T>(xi[0], xi[1], xi[2], b);
#pragma unroll
    for (int d = 0; d < ID; ++d) b[d] -= BM[c * ID + d];
    if (!weno || !p.full[c]) {  // MUSCL everywhere / CHECKSOL: FULL=0 -> REDUCE
      s_flag[cl * 2 + 0] = 1;
      continue;
    }
    const T* gh = s_gh + (size_t)cl * ID * NV;
    double uf[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      T res = T(0);
#pragma unroll
      for (int d = 0; d < ID; ++d) res += b[d] * gh[d * NV + v];
      o[v] = res;
      uf[v] = s_u0[cl * NV + v] + (double)res;
    }
    double pm[NV];
    cons2prim(p.gamma, s_u0 + cl * NV, pm);
    if (jump_bad(p.gamma, pm, uf, 0.85)) s_flag[cl * 2 + 0] = 1;
  }
  __syncthreads();

  // ---- MUSCL on flagged cells, using the central stencil polynomial
  for (int i = tid; i < nc * NV; i += nt) {
    int cl = i / NV, v = i - cl * NV;
    if (!s_flag[cl * 2]) continue;
    int64_t c = c0 + cl;
    double u0 = s_u0[cl * NV + v], mn = u0, mx = u0;
    for (int f = 0; f < p.nfaces[c]; ++f) {
      int64_t nb = p.neigh[c * MF + f];
      if (nb < 0) continue;
      double un = U[nb * NV + v];
      mn = fmin(mn, un);
      mx = fmax(mx, un);
    }
    s_bnd[(cl * 2 + 0) * NV + v] = mn - u0;
    s_bnd[(cl * 2 + 1) * NV + v] = mx - u0;
  }
  __syncthreads();
  for (int i = tid; i < nc * MF * QS; i += nt) {
    int cl = i / (MF * QS), r = i - cl * (MF * QS), f = r / QS, q = r - f * QS;
    if (!s_flag[cl * 2]) continue;
    int64_t c = c0 + cl;
    double* ps = s_psi + (size_t)i * NV;
    if (f >= p.nfaces[c] || q >= face_nq(p, p.ftype[c * MF + f])) {
#pragma unroll
      for (int v = 0; v < NV; ++v) ps[v] = TOLBIG;
      continue;
    }
    const T* xi = QP + ((c * MF + f) * QS + q) * 3;
    T b[ID];
    monomials<P, T>(xi[0], xi[1], xi[2], b);
#pragma unroll
    for (int d = 0; d < ID; ++d) b[d] -= BM[c * ID + d];
    const T* g0 = s_G + (size_t)(cl * A) * ID * NV;
    double e = p.kappa_ven * p.minedge[c];
    double epsi2 = e * e * e;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      T res = T(0);
#pragma unroll
      for (int d = 0; d < ID; ++d) res += b[d] * g0[d * NV + v];
      double u0 = s_u0[cl * NV + v];
      double dd = (u0 + (double)res) - u0;
      s_dul[(size_t)i * NV + v] = T(dd);
      ps[v] = venkat(dd, s_bnd[(cl * 2 + 0) * NV + v], s_bnd[(cl * 2 + 1) * NV + v], epsi2);
    }
  }
  __syncthreads();
  for (int i = tid; i < nc * NV; i += nt) {
    int cl = i / NV, v = i - cl * NV;
    if (!s_flag[cl * 2]) continue;
    double mn = TOLBIG;
    for (int j = 0; j < MF * QS; ++j) mn = fmin(mn, s_psi[((size_t)cl * MF * QS + j) * NV + v]);
    s_slope[cl * NV + v] = mn;
  }
  __syncthreads();
  for (int i = tid; i < nc * MF * QS; i += nt) {
    int cl = i / (MF * QS);
    if (!s_flag[cl * 2]) continue;
#pragma unroll
    for (int v = 0; v < NV; ++v) s_dul[(size_t)i * NV + v] = T((double)s_dul[(size_t)i * NV + v] * s_slope[cl * NV + v]);
  }
  __syncthreads();

  // ---- CHECKSOLX: first order where a face value jumps by 95 %
  for (int i = tid; i < nc * MF * QS; i += nt) {
    int cl = i / (MF * QS), r = i - cl * (MF * QS), f = r / QS, q = r - f * QS;
    int64_t c = c0 + cl;
    if (f >= p.nfaces[c] || q >= face_nq(p, p.ftype[c * MF + f])) continue;
    double uf[NV], pm[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uf[v] = s_u0[cl * NV + v] + (double)s_dul[(size_t)i * NV + v];
    cons2prim(p.gamma, s_u0 + cl * NV, pm);
    if (jump_bad(p.gamma, pm, uf, 0.95)) s_flag[cl * 2 + 1] = 1;
  }
  __syncthreads();
  T* out = (T*)p.dul + c0 * MF * QS * NV;
  for (int i = tid; i < nc * MF * QS * NV; i += nt) {
    int cl = i / (MF * QS * NV);
    out[i] = s_flag[cl * 2 + 1] ? T(0) : s_dul[i];
  }
}

// ======================================================================
// Viscous gradients for WENO/CWENO + Navier-Stokes: LSQ on (T,u,v,w) with
// stencil 1 (gradients.f90:502-706), then face gradients (SOLUTIONTRIAV2).
// ======================================================================
template <int P, typename T>
__global__ void k_visc_lsq(Problem p, const double* __restrict__ U) {
  constexpr int ID = Deg<P>::ideg;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n * 4) return;
  const int64_t c = i >> 2;
  const int var = (int)(i & 3);
  const int IM = p.imax, W = IM + 1;
  double pm[NV];
  cons2prim(p.gamma, U + c * NV, pm);
  const double s0 = var == 0 ? pm[4] / (pm[0] * p.r_gas) : pm[var];
  const int32_t* st = p.sten + c * (int64_t)p.admis_max * W;
  const T* M = (const T*)p.invmat + c * (int64_t)p.admis_max * IM * ID;
  double acc[ID];
#pragma unroll
  for (int d = 0; d < ID; ++d) acc[d] = 0.0;
  for (int k = 0; k < IM; ++k) {
    double py[NV];
    cons2prim(p.gamma, U + (int64_t)st[k + 1] * NV, py);
    double ds = (var == 0 ? py[4] / (py[0] * p.r_gas) : py[var]) - s0;
#pragma unroll
    for (int d = 0; d < ID; ++d) acc[d] += (double)M[k * ID + d] * ds;
  }
#pragma unroll
  for (int d = 0; d < ID; ++d) p.gv[(c * ID + d) * 4 + var] = acc[d];
}

template <int P, typename T>
__global__ void k_visc_face(Problem p) {
  constexpr int ID = Deg<P>::ideg;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n * MF * QS) return;
  const int64_t c = i / (MF * QS);
  const int r = (int)(i - c * MF * QS), f = r / QS, q = r - f * QS;
  if (f >= p.nfaces[c] || q >= face_nq(p, p.ftype[c * MF + f])) return;
  const T* xi = (const T*)p.qpts + ((c * MF + f) * QS + q) * 3;
  double dx[ID], dy[ID], dz[ID];
  dmonomials<P>((double)xi[0], (double)xi[1], (double)xi[2], dx, dy, dz);
  const double* J = p.jinv + c * 9;
  double* o = p.ulv + ((c * MF + f) * QS + q) * 12;
#pragma unroll
  for (int var = 0; var < 4; ++var) {
    double gl[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < ID; ++d) {
      double g = p.gv[(c * ID + d) * 4 + var];
      gl[0] += g * dx[d];
      gl[1] += g * dy[d];
      gl[2] += g * dz[d];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) o[var * 3 + k] = J[0 * 3 + k] * gl[0] + J[1 * 3 + k] * gl[1] + J[2 * 3 + k] * gl[2];
  }
}

// ======================================================================
// Face fluxes fused with the RK stage update.  Eight lanes per cell, lane f
// integrates face f; the face sums are added in face order
// (CALCULATE_FLUXESHI_CONVECTIVE flux_p.f90:478, CALCULATE_FLUXESHI_DIFFUSIVE
// flux_p.f90:1520), then RUNGE_KUTTA3 (time_p.f90:885-1027).
// MODE 0: write the residual; MODE 1/2/3: RK stage 1/2/3.
// ======================================================================
__device__ __forceinline__ void boundary_ghost(const Problem& p, int code, const double* r, const double* cl,
                                               double* cr) {
  const double gm = p.gamma;
  const double nx = r[0] * r[3], ny = r[1] * r[3], nz = r[2];
  if (code == 3 || code == 4) {  // symmetry / inviscid wall: mirror the normal momentum
    double a[NV], b[NV];
    rot_f(r, cl, a);
    b[0] = a[0];
    b[1] = -a[1];
    b[2] = a[2];
    b[3] = a[3];
    b[4] = a[4];
    rot_b(r, b, cr);
    return;
  }
  double s1[NV], s2[NV], s3[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) s1[k] = p.bc_state[k];
  cons2prim(gm, cl, s2);
  double sps = sqrt(gm * s2[4] / s2[0]);
  double vel = sqrt(s2[1] * s2[1] + s2[2] * s2[2] + s2[3] * s2[3]);
  bool super = vel / (sps + TOLSMALL) > 1.0;
  if (code == 1) {  // inflow (BOUNDARYS case 1, subsonic characteristic treatment)
    if (super) {
      prim2cons(gm, s1, cr);
      return;
    }
    s3[4] = 0.5 * (s1[4] + s2[4] - s2[0] * sps * (nx * (s1[1] - s2[1]) + ny * (s1[2] - s2[2]) + nz * (s1[3] - s2[3])));
    s3[0] = s1[0] + (s3[4] - s1[4]) / (sps * sps);
    s3[1] = s1[1] - nx * (s1[4] - s3[4]) / (sps * s2[0]);
    s3[2] = s1[2] - ny * (s1[4] - s3[4]) / (sps * s2[0]);
    s3[3] = s1[3] - nz * (s1[4] - s3[4]) / (sps * s2[0]);
  } else if (code == 2) {  // outflow (case 2)
    if (super) {
#pragma unroll
      for (int k = 0; k < NV; ++k) cr[k] = cl[k];
      return;
    }
    s3[4] = s1[4];
    s3[0] = s2[0] + (s3[4] - s2[4]) / (sps * sps);
    s3[1] = s2[1] + nx * (s2[4] - s3[4]) / (sps * s2[0]);
    s3[2] = s2[2] + ny * (s2[4] - s3[4]) / (sps * s2[0]);
    s3[3] = s2[3] + nz * (s2[4] - s3[4]) / (sps * s2[0]);
  } else {
    prim2cons(gm, s1, cr);
    return;
  }
  prim2cons(gm, s3, cr);
}

__device__ __forceinline__ void viscous_flux(const Problem& p, const double* r, double dih, const double* cl,
                                             const double* cr, const double* gl, const double* gr, double* fv) {
  double nx = r[0] * r[3], ny = r[1] * r[3], nz = r[2];
  double nn[3] = {nx, ny, nz};
  double lv[NV], rv[NV];
  cons2prim(p.gamma, cl, lv);
  cons2prim(p.gamma, cr, rv);
  double mul, mur, laml, lamr;
  sutherland(p, lv[0], lv[4], &mul, &laml);
  sutherland(p, rv[0], rv[4], &mur, &lamr);
  // gradient rows u, v, w, T; stored components are T, u, v, w
  const int src[4] = {1, 2, 3, 0};
  double jump[4] = {rv[1] - lv[1], rv[2] - lv[2], rv[3] - lv[3],
                    rv[4] / (rv[0] * p.r_gas) - lv[4] / (lv[0] * p.r_gas)};
  const double vd = (4.0 / 3.0) / fabs(dih);
  double gg[4][3];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      gg[a][k] = (gl[src[a] * 3 + k] + gr[src[a] * 3 + k]) / 2.0 + p.lamx * (vd * nn[k] * jump[a]);
  double lam2 = 0.5 * (laml + lamr), mu2 = 0.5 * (mul + mur);
  double ux = gg[0][0], uy = gg[0][1], uz = gg[0][2];
  double vx = gg[1][0], vy = gg[1][1], vz = gg[1][2];
  double wx = gg[2][0], wy = gg[2][1], wz = gg[2][2];
  double txx = mu2 * ((4.0 / 3.0) * ux - (2.0 / 3.0) * vy - (2.0 / 3.0) * wz);
  double tyy = mu2 * ((4.0 / 3.0) * vy - (2.0 / 3.0) * ux - (2.0 / 3.0) * wz);
  double tzz = mu2 * ((4.0 / 3.0) * wz - (2.0 / 3.0) * ux - (2.0 / 3.0) * vy);
  double txy = mu2 * (uy + vx), txz = mu2 * (wx + uz), tyz = mu2 * (vz + wy);
  double rho12 = 0.5 * (cl[0] + cr[0]);
  double u12 = 0.5 * (cl[1] + cr[1]) / rho12, v12 = 0.5 * (cl[2] + cr[2]) / rho12, w12 = 0.5 * (cl[3] + cr[3]) / rho12;
  double qx = lam2 * gg[3][0], qy = lam2 * gg[3][1], qz = lam2 * gg[3][2];  // -Q
  double fx4 = qx + u12 * txx + v12 * txy + w12 * txz;
  double fy4 = qy + u12 * txy + v12 * tyy + w12 * tyz;
  double fz4 = qz + u12 * txz + v12 * tyz + w12 * tzz;
  fv[0] = 0.0;
  fv[1] = nx * txx + ny * txy + nz * txz;
  fv[2] = nx * txy + ny * tyy + nz * tyz;
  fv[3] = nx * txz + ny * tyz + nz * tzz;
  fv[4] = nx * fx4 + ny * fy4 + nz * fz4;
}

template <typename T, bool NS, int MODE>
__global__ void __launch_bounds__(256) k_flux(Problem p, const double* __restrict__ Uc, const double* Un,
                                              double* Uout, double dt_host) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t c = gid >> 3;
  const int f = (int)(gid & 7);
  const int lane = threadIdx.x & 31, base = lane & ~7;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  double god[NV] = {0, 0, 0, 0, 0}, gvis[NV] = {0, 0, 0, 0, 0};
  const bool live = c < p.n && f < p.nfaces[c];
  if (live) {
    double u0[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) u0[v] = Uc[c * NV + v];
    const int ft = p.ftype[c * MF + f];
    const int nq = face_nq(p, ft);
    const int64_t nb = p.neigh[c * MF + f];
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
    for (int q = 0; q < nq; ++q) {
      double cl[NV], cr[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) cl[v] = u0[v] + (double)dl[q * NV + v];
      int qq = qpm[q];
      if (nb >= 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) cr[v] = un[v] + (double)dr[qq * NV + v];
      } else {
        boundary_ghost(p, p.bc[c * MF + f], r, cl, cr);
      }
      double a[NV], b[NV], h[NV], fl[NV];
      rot_f(r, cr, b);
      rot_f(r, cl, a);
      hllc(p.gamma, a, b, h);
      rot_b(r, h, fl);
      const double ws = face_weight(p, ft, q) * area;
#pragma unroll
      for (int v = 0; v < NV; ++v) god[v] = god[v] + fl[v] * ws;
      if (NS && nb >= 0) {
        const double* gl = p.ulv + ((c * MF + f) * QS + q) * 12;
        const double* gr = p.ulv + ((nb * MF + nf) * QS + qq) * 12;
        double fv[NV];
        viscous_flux(p, r, p.dih[c * MF + f], cl, cr, gl, gr, fv);
#pragma unroll
        for (int v = 0; v < NV; ++v) gvis[v] = gvis[v] + fv[v] * ws;
      }
    }
  }
  // face sums in face order: convective first, then viscous (subtracted)
  double R[NV] = {0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < MF; ++k)
#pragma unroll
    for (int v = 0; v < NV; ++v) R[v] = R[v] + __shfl_sync(0xffffffffu, god[v], base + k);
  if (NS) {
#pragma unroll
    for (int k = 0; k < MF; ++k)
#pragma unroll
      for (int v = 0; v < NV; ++v) R[v] = R[v] - __shfl_sync(0xffffffffu, gvis[v], base + k);
  }
  if (f != 0 || c >= p.n) return;
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
  double pr[NV];
  cons2prim(p.gamma, out, pr);
  if (!(pr[0] > 0.0) || !(pr[4] > 0.0) || !isfinite(out[4])) atomicOr(p.health, HEALTH_NONPHYS);
#pragma unroll
  for (int v = 0; v < NV; ++v) Uout[c * NV + v] = out[v];
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
    double x = what == UCG_REDUCE_KE ? 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]
                                     : (what == UCG_REDUCE_MASS ? u[0] : u[4]);
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
// ======================================================================
template <typename T>
__global__ void k_expand(T* __restrict__ dst, const double* __restrict__ src, const int32_t* __restrict__ tid,
                         int64_t first, int64_t count, int64_t len, int64_t tlo, int64_t thi) {
  const int64_t total = count * len;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t cl = i / len, j = i - cl * len;
    int64_t t = tid ? tid[cl] : cl;
    if (t < tlo || t >= thi) continue;
    dst[(first + cl) * len + j] = T(src[(t - tlo) * len + j]);
  }
}

}  // namespace ucg
