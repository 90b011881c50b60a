// Discrete adjoint (VJP) of the WENO and CWENO reconstruction (conserved
// variables, EES 0 or 5, CWENO with or without WENO-Z, FP64 form): the reverse of CP_RECONSTRUCTION's nonlinear weights
// and smoothness indicators (src/reconstruct_p.f90:920-1250) and of the
// stencil least squares (LEAST_SQUARES, src/gradients.f90:253-497).
//
// Forward, per cell c and variable v (k_lsq, k_wpost):
//   G_l  = M_l (U_st(l,k) - U_c)                         l < ADMIS
// (The tangent, k_jvp_wpost, pushes dG = M_l (dU_st - dU_c) forward instead.)
//   IS_l = G_l^T S G_l,  wt_l = lam_l / (eps + IS_l)^4,  om_l = wt_l / sum wt
//   u(x) = U_c + sum_l om_l b(x) . G_l                   at every face point
// Reverse, given ub(x) = dJ/du(x) at the face points:
//   Bb      = sum_x ub(x) b(x)                (the basis with its mean removed)
//   omb_l   = Bb . G_l
//   wtb_l   = (omb_l - sum_m omb_m om_m) / sum wt
//   ISb_l   = -4 wtb_l wt_l / (eps + IS_l)
//   Gb_l    = om_l Bb + ISb_l 2 S G_l
//   U_c    += sum_x ub(x);  U_st(l,k) += M_l[k]^T Gb_l;  U_c -= sum_k M_l[k]^T Gb_l
// A cell whose CHECKSOL test (or FULL = 0) put it on the MUSCL fall-back
// takes the reverse (and tangent) of that branch instead: the central
// polynomial G_0 limited by Venkatakrishnan with FIND_BOUNDS over the face
// neighbours, and CHECKSOLX.
#include <cuda_runtime.h>

#include "ad.cuh"
#include "engine_internal.h"
#include "recon2.cuh"

using namespace ucg;

namespace {

// gr += 2 S g for the packed triangle P of S (rows padded to vectors; P_dd =
// S_dd, P_de = 2 S_de), over the first nd <= NMAX rows
template <int NMAX>
__device__ __forceinline__ void tri_grad(const double* __restrict__ P, const double (&g)[NMAX], int nd,
                                         double (&gr)[NMAX]) {
  constexpr int VEC = Vec<double>::N;
  int rs = 0;
#pragma unroll
  for (int d = 0; d < NMAX; ++d) {
    if (d < nd) {
#pragma unroll
      for (int q = 0; q < (NMAX - d + VEC - 1) / VEC; ++q)
        if (d + q * VEC < nd) {
          double sv[VEC];
          ldv(P + (int64_t)(rs + q) * 32 * VEC, sv);
#pragma unroll
          for (int i = 0; i < VEC; ++i) {
            const int e = d + q * VEC + i;
            if (e < NMAX && e < nd) {
              if (e == d) {
                gr[d] += 2.0 * sv[i] * g[d];
              } else {
                gr[d] += sv[i] * g[e];
                gr[e] += sv[i] * g[d];
              }
            }
          }
        }
      rs += (nd - d + VEC - 1) / VEC;
      asm volatile("" ::: "memory");
    }
  }
}

// IS = g^T S g and gr = 2 S g in one pass over the packed triangle
template <int NMAX>
__device__ __forceinline__ double is_and_grad(const double* __restrict__ P, const double (&g)[NMAX], int nd,
                                              double (&gr)[NMAX]) {
#pragma unroll
  for (int d = 0; d < NMAX; ++d) gr[d] = 0.0;
  tri_grad<NMAX>(P, g, nd, gr);
  double is = 0.0;
#pragma unroll
  for (int d = 0; d < NMAX; ++d)
    if (d < nd) is += g[d] * gr[d];
  return 0.5 * is;
}

// Thread layout of the WENO post-processing adjoint and tangent: one block
// per group of 32 cells (the group of the interleaved tables), NV warps,
// warp v takes variable v of every cell of the group (lane = cell).  The
// weights of one variable need no other variable, so the warps only meet
// at the CHECKSOL test (all five variables of a face value); and the five
// warps read the same smoothness matrices at about the same time, so those
// come from DRAM about once per pass instead of once per variable.
constexpr int WP_THREADS = NV * 32;
#ifndef UCG_AWP_MINB
#define UCG_AWP_MINB 2  // blocks per SM the register budget is sized for
#endif

// CHECKSOL (0.85) of the combined polynomial sGH (all variables, shared
// memory) at the face points of cell c; warp w tests the points whose
// running index is w modulo NV.  True if a face value of the cell fails.
template <int P>
__device__ __forceinline__ bool checksol_split(const Problem& p, const double* __restrict__ U, int64_t c, int nf,
                                               const double* __restrict__ xq, const double* __restrict__ bmv,
                                               const double (*sGH)[NV][32], int lane, int w) {
  constexpr int ID = Deg<P>::ideg;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  double u0[NV], pm[NV], cb[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u0[v] = U[c * NV + v];
  cons2prim(p.gamma, u0, pm);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    cb[v] = 0.0;
#pragma unroll
    for (int d = 0; d < ID; ++d) cb[v] += bmv[d * 32] * sGH[d][v][lane];
  }
  bool bad = false;
  int k = 0;
  for (int f = 0; f < nf; ++f) {
    const int nq = face_nq(p, p.ftype[c * MF + f]);
    for (int q = 0; q < nq; ++q, ++k) {
      if (k % NV != w || bad) continue;
      const double* xi = xq + (int64_t)(f * QS + q) * 3 * 32;
      double m[ID], uf[NV];
      monomials<P, double>(xi[0], xi[32], xi[64], m);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        // re-read the combined polynomial from shared memory at every point:
        // kept in registers across the points it does not fit
        asm volatile("" ::: "memory");
        double r = 0.0;
#pragma unroll
        for (int d = 0; d < ID; ++d) r += m[d] * sGH[d][v][lane];
        uf[v] = u0[v] + (r - cb[v]);
      }
      bad = jump_bad(p.gamma, pm, uf, 0.85);
    }
  }
  return bad;
}

// CHECKSOLX (0.95) of the MUSCL fall-back face values u0 + dd(x) slope of
// cell c, dd(x) = (u0 + m(x).g0 - mean) - u0 with the central polynomial g0
// (sG, all variables) and the limiter value (sS); warp w tests the points
// whose running index is w modulo NV.  True if a face value of the cell fails.
template <int P>
__device__ __forceinline__ bool checksolx_split(const Problem& p, const double* __restrict__ U, int64_t c, int nf,
                                                const double* __restrict__ xq, const double* __restrict__ bmv,
                                                const double (*sG)[NV][32], const double (*sS)[32], int lane, int w) {
  constexpr int ID = Deg<P>::ideg;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  double u0[NV], pm[NV], cb[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u0[v] = U[c * NV + v];
  cons2prim(p.gamma, u0, pm);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    cb[v] = 0.0;
#pragma unroll
    for (int d = 0; d < ID; ++d) cb[v] += bmv[d * 32] * sG[d][v][lane];
  }
  bool bad = false;
  int k = 0;
  for (int f = 0; f < nf; ++f) {
    const int nq = face_nq(p, p.ftype[c * MF + f]);
    for (int q = 0; q < nq; ++q, ++k) {
      if (k % NV != w || bad) continue;
      const double* xi = xq + (int64_t)(f * QS + q) * 3 * 32;
      double m[ID], uf[NV];
      monomials<P, double>(xi[0], xi[32], xi[64], m);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        asm volatile("" ::: "memory");  // re-read the polynomial from shared memory at every point
        double r = 0.0;
#pragma unroll
        for (int d = 0; d < ID; ++d) r += m[d] * sG[d][v][lane];
        r = r - cb[v];
        const double dd = (u0[v] + r) - u0[v];
        uf[v] = u0[v] + dd * sS[v][lane];
      }
      bad = jump_bad(p.gamma, pm, uf, 0.95);
    }
  }
  return bad;
}

// k_adj_wpost: writes Gb (layout of the stencil polynomials G), the direct
// adjoint of the cell mean (selfc) and the face slots of the MUSCL
// fall-back's bounds; scr holds Bb (interleaved like G).  Gb first receives
// 2 S G_l (the gradient of IS_l), read back once the weights' adjoints are
// known.  The branch of every cell is decided as in the forward: FULL = 0
// or a failed CHECKSOL (0.85) takes the MUSCL fall-back (the central
// stencil polynomial G_0, FIND_BOUNDS over the face neighbours and the
// Venkatakrishnan limiter, src/reconstruct_p.f90:3126-3406), whose reverse
// is
//   out(x) = dd(x) slope,  slope = min_x phi(dd(x), lo, hi):
//   Gb_0 = slope Bb + sb dphi/ddd(x*) (m(x*) - mean),  sb = sum_x ub(x) dd(x),
//   lo/hi's adjoints sb dphi/dlo, sb dphi/dhi to the face neighbour that set
//   the bound (face slot) and minus that to the cell;
// a fall-back that CHECKSOLX (0.95) reduced to first order has no
// dependence on the polynomials or the bounds.
template <int P>
__global__ void __launch_bounds__(WP_THREADS, UCG_AWP_MINB) k_adj_wpost(Problem p, const double* __restrict__ U,
                                                                        const double* __restrict__ adjF,
                                                                        double* __restrict__ gbar,
                                                                        double* __restrict__ scr,
                                                                        double* __restrict__ selfc,
                                                                        double* __restrict__ contrib) {
  constexpr int ID = Deg<P>::ideg;
  constexpr int VEC = Vec<double>::N;
  __shared__ double sGH[ID][NV][32];  // WENO combined polynomial, then the fall-back's G_0
  __shared__ double sSlope[NV][32];
  __shared__ int sFall[32];  // bit 0: MUSCL fall-back, bit 1: reduced to first order
  const int lane = threadIdx.x & 31, v = threadIdx.x >> 5;
  const int64_t grp = blockIdx.x;
  const int64_t c = grp * 32 + lane;
  const bool cell = c < p.n;
  const bool full = cell && p.full[c];
  if (v == 0) sFall[lane] = cell && !full ? 1 : 0;
  const int A = p.admis_max, IM = p.imax;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const int FQ = MF * QS;
  const bool cw = p.ees == 5;
  const int64_t fslot = (cw ? 1 + IM + (int64_t)(A - 1) * p.imax2 : 1 + (int64_t)A * IM);
  const double* xq = (const double*)p.qpts + grp * (int64_t)FQ * 3 * 32 + lane;
  const double* bmv = (const double*)p.bmean + grp * (int64_t)ID * 32 + lane;
  const int adm = cell ? p.admis[c] : 0, nf = cell ? p.nfaces[c] : 0;
  const double* Gc = (const double*)p.gbuf + grp * (int64_t)(A * ID * NV) * 32 + lane;
  auto G = [&](int ll, int d) -> double { return Gc[(int64_t)((ll * ID + d) * NV + v) * 32]; };
  double* Gb = gbar + grp * (int64_t)(A * ID * NV) * 32 + lane;
  auto GB = [&](int ll, int d) -> double& { return Gb[(int64_t)((ll * ID + d) * NV + v) * 32]; };
  double* BBp = scr + grp * (int64_t)(ID * NV) * 32 + lane;
  auto BB = [&](int d) -> double& { return BBp[(int64_t)(d * NV + v) * 32]; };
  const double* aF = adjF + c * (int64_t)FQ * NV + v;
  const int ID2 = p.ideg2;
  constexpr int L2 = ID < 9 ? ID : 9;
  auto nd_of = [&](int ll) { return cw && ll > 0 ? ID2 : ID; };
  // ---- the direct term and Bb = sum_x ub(x) (m(x) - mean(m))
  if (cell) {
    double acc[ID], sa = 0.0;
#pragma unroll
    for (int d = 0; d < ID; ++d) acc[d] = 0.0;
    for (int f = 0; f < nf; ++f) {
      const int nq = face_nq(p, p.ftype[c * MF + f]);
      for (int q = 0; q < nq; ++q) {
        const double* xi = xq + (int64_t)(f * QS + q) * 3 * 32;
        double m[ID];
        monomials<P, double>(xi[0], xi[32], xi[64], m);
        const double a = aF[(f * QS + q) * NV];
        sa += a;
#pragma unroll
        for (int d = 0; d < ID; ++d) acc[d] += m[d] * a;
      }
    }
#pragma unroll
    for (int d = 0; d < ID; ++d) BB(d) = acc[d] - bmv[d * 32] * sa;
    selfc[c * NV + v] = sa;
  }
  // ---- WENO branch: indicators and weights.  CWENO (EES 5): the central
  // polynomial is g1 = (G_0 - sum_l lk G_l) / lc1 (rows below IDEGFREE2 for
  // the lower-order stencils), the lower-order stencils have IDEGFREE2 rows
  // and the S2 triangle, the linear weights are lc1, lk.
  const double* Pc = (const double*)p.ind + grp * p.istride * 32 + lane * VEC;
  const double* Pc2 = Pc + (int64_t)(p.i2off / VEC) * 32 * VEC;
  const double lc1 = 1.0 - 1.0 / p.lwci;
  const double lk = adm > 1 ? (1.0 - lc1) / (adm - 1) : 0.0;
  double g3[L2];
#pragma unroll
  for (int d = 0; d < L2; ++d) g3[d] = 0.0;
  if (cw && full)
    for (int l2 = 1; l2 < adm; ++l2)
#pragma unroll
      for (int d = 0; d < L2; ++d)
        if (d < ID2) g3[d] = g3[d] + lk * G(l2, d);
  // row d of stencil polynomial ll as the reconstruction uses it
  auto poly = [&](int ll, int d) -> double {
    if (d >= nd_of(ll)) return 0.0;
    if (cw && ll == 0) return (1.0 / lc1) * (G(0, d) - (d < L2 ? g3[d] : 0.0));
    return G(ll, d);
  };
  const bool wz = cw && p.wenoz;
  double is[7], wt[7], om[7], omb[7];
  double tau = 0.0, sum = 0.0, dot = 0.0;
  if (full) {
#pragma unroll 1
    for (int ll = 0; ll < adm; ++ll) {
      double s;
      if (cw && ll > 0) {
        double g[L2], gr[L2];
#pragma unroll
        for (int d = 0; d < L2; ++d) g[d] = poly(ll, d);
        s = is_and_grad<L2>(Pc2, g, ID2, gr);
#pragma unroll
        for (int d = 0; d < L2; ++d)
          if (d < ID2) GB(ll, d) = gr[d];
      } else {
        double g[ID], gr[ID];
#pragma unroll
        for (int d = 0; d < ID; ++d) g[d] = poly(ll, d);
        s = is_and_grad<ID>(Pc, g, ID, gr);
#pragma unroll
        for (int d = 0; d < ID; ++d) GB(ll, d) = gr[d];
      }
      is[ll] = s;
    }
    // weights: lam / (eps + IS)^4, or WENO-Z (CWENO only)
    // lam (1 + (tau / (eps + IS))^4) with tau = sum_l |IS_0 - IS_l| / (adm - 1)
    if (wz) {
      for (int ll = 0; ll < adm; ++ll) tau += fabs(is[0] - is[ll]);
      tau = tau / (adm - 1);
    }
    for (int ll = 0; ll < adm; ++ll) {
      const double e = p.weno_eps + is[ll];
      const double lam = cw ? (ll == 0 ? lc1 : lk) : (ll == 0 ? p.lwci : 1.0);
      if (wz) {
        double q = tau / e;
        q = q * q;
        wt[ll] = lam * (1.0 + q * q);
      } else {
        const double e2 = e * e;
        wt[ll] = lam / (e2 * e2);
      }
      sum += wt[ll];
    }
    for (int ll = 0; ll < adm; ++ll) om[ll] = wt[ll] / sum;
    // combined polynomial (CHECKSOL, in shared memory) and the weights' adjoints
#pragma unroll
    for (int d = 0; d < ID; ++d) sGH[d][v][lane] = 0.0;
#pragma unroll 1
    for (int ll = 0; ll < adm; ++ll) {
      double ob = 0.0;
#pragma unroll
      for (int d = 0; d < ID; ++d) {
        const double gd = poly(ll, d);
        ob += BB(d) * gd;
        sGH[d][v][lane] += om[ll] * gd;
        if ((d & 7) == 7) asm volatile("" ::: "memory");  // bound the loads in flight
      }
      omb[ll] = ob;
      dot += ob * om[ll];
    }
  }
  __syncthreads();
  // ---- CHECKSOL (0.85) on the WENO face values
  if (full && checksol_split<P>(p, U, c, nf, xq, bmv, sGH, lane, v)) atomicOr(&sFall[lane], 1);
  __syncthreads();
  const bool fall = cell && (sFall[lane] & 1);
  if (full && !fall) {
    // ---- Gb_l = om_l Bb + ISb_l 2 S G_l (+ the CWENO central share)
    double corr[L2];
#pragma unroll
    for (int d = 0; d < L2; ++d) corr[d] = 0.0;
    // WENO-Z: wt_l = lam_l (1 + q_l^4), q_l = tau / (eps + IS_l):
    // d wt_l / d tau = 4 (wt_l - lam_l) / tau, d wt_l / d IS_l = -4 (wt_l - lam_l) / (eps + IS_l);
    // tau's adjoint goes back to the IS through sign(IS_0 - IS_l) / (adm - 1)
    double taub = 0.0;
    if (wz && tau > 0.0)
      for (int ll = 0; ll < adm; ++ll) {
        const double lam = ll == 0 ? lc1 : lk;
        taub += (omb[ll] - dot) / sum * 4.0 * (wt[ll] - lam) / tau;
      }
    double tsg = 0.0;  // sum_l sign(IS_0 - IS_l)
    if (wz)
      for (int ll = 1; ll < adm; ++ll) tsg += is[0] > is[ll] ? 1.0 : (is[0] < is[ll] ? -1.0 : 0.0);
#pragma unroll 1
    for (int ll = 0; ll < adm; ++ll) {
      const double wtb = (omb[ll] - dot) / sum;
      double isb;
      if (wz) {
        const double lam = ll == 0 ? lc1 : lk;
        const double sg = ll == 0 ? tsg : (is[0] > is[ll] ? -1.0 : (is[0] < is[ll] ? 1.0 : 0.0));
        isb = wtb * (-4.0 * (wt[ll] - lam) / (p.weno_eps + is[ll])) + taub * sg / (adm - 1);
      } else {
        isb = wtb * (-4.0 * wt[ll] / (p.weno_eps + is[ll]));
      }
      if (cw && ll > 0) {
#pragma unroll
        for (int d = 0; d < L2; ++d)
          if (d < ID2) GB(ll, d) = om[ll] * BB(d) + isb * GB(ll, d) + corr[d];
      } else {
#pragma unroll
        for (int d = 0; d < ID; ++d) {
          const double gb = om[ll] * BB(d) + isb * GB(ll, d);  // adjoint of the polynomial used
          if (cw) {  // ll == 0: g1 = (G_0 - sum lk G_l) / lc1
            GB(0, d) = (1.0 / lc1) * gb;
            if (d < L2) corr[d] = -lk * ((1.0 / lc1) * gb);
          } else {
            GB(ll, d) = gb;
          }
        }
      }
    }
  }
  // ---- MUSCL fall-back: the forward again (bounds, limiter and its
  // limiting point), G_0 and the limiter value shared for CHECKSOLX
  double lo = 0.0, hi = 0.0, slope = TOLBIG, ddx = 0.0, sb = 0.0, epsi2 = 0.0;
  int flo = -1, fhi = -1, xs = -1;
  if (fall) {
    const double u0v = U[c * NV + v];
    lo = hi = u0v;
    for (int f = 0; f < nf; ++f) {
      const int64_t nb = p.neigh[c * MF + f];
      if (nb < 0) continue;
      const double un = U[nb * NV + v];
      if (un < lo) lo = un, flo = f;
      if (un > hi) hi = un, fhi = f;
    }
    lo -= u0v;
    hi -= u0v;
    const double e3 = p.kappa_ven * p.minedge[c];
    epsi2 = e3 * e3 * e3;
    double g0[ID], cb = 0.0;
#pragma unroll
    for (int d = 0; d < ID; ++d) {
      g0[d] = G(0, d);
      cb += bmv[d * 32] * g0[d];
    }
    for (int f = 0; f < nf; ++f) {
      const int nq = face_nq(p, p.ftype[c * MF + f]);
      for (int q = 0; q < nq; ++q) {
        const double* xi = xq + (int64_t)(f * QS + q) * 3 * 32;
        double m[ID];
        monomials<P, double>(xi[0], xi[32], xi[64], m);
        double r = 0.0;
#pragma unroll
        for (int d = 0; d < ID; ++d) r += m[d] * g0[d];
        r = r - cb;
        const double dd = (u0v + r) - u0v;
        const double phi = venkat(dd, lo, hi, epsi2);
        if (phi < slope) slope = phi, xs = f * QS + q, ddx = dd;
        sb += aF[(f * QS + q) * NV] * dd;
      }
    }
#pragma unroll
    for (int d = 0; d < ID; ++d) sGH[d][v][lane] = g0[d];
    sSlope[v][lane] = slope;
  }
  __syncthreads();
  if (fall && checksolx_split<P>(p, U, c, nf, xq, bmv, sGH, sSlope, lane, v)) atomicOr(&sFall[lane], 2);
  __syncthreads();
  double fb[MF];
#pragma unroll
  for (int f = 0; f < MF; ++f) fb[f] = 0.0;
  if (fall) {
    const bool first = sFall[lane] & 2;
    if (!first && xs >= 0) {
      ad::Dual<3> dd(ddx), dlo(lo), dhi(hi);
      dd.d[0] = 1.0;
      dlo.d[1] = 1.0;
      dhi.d[2] = 1.0;
      const ad::Dual<3> ph = venkat(dd, dlo, dhi, epsi2);
      const double ddb = sb * ph.d[0], lob = sb * ph.d[1], hib = sb * ph.d[2];
      const double* xi = xq + (int64_t)xs * 3 * 32;
      double m[ID];
      monomials<P, double>(xi[0], xi[32], xi[64], m);
#pragma unroll
      for (int d = 0; d < ID; ++d) GB(0, d) = slope * BB(d) + ddb * (m[d] - bmv[d * 32]);
      // lo = U_nb - u0 (or 0 when the cell itself is the minimum)
      double selfb = 0.0;
#pragma unroll
      for (int f = 0; f < MF; ++f) {
        if (f == flo) fb[f] += lob, selfb -= lob;
        if (f == fhi) fb[f] += hib, selfb -= hib;
      }
      selfc[c * NV + v] += selfb;
    } else {
#pragma unroll
      for (int d = 0; d < ID; ++d) GB(0, d) = 0.0;
    }
    for (int ll = 1; ll < adm; ++ll)
      for (int d = 0; d < nd_of(ll); ++d) GB(ll, d) = 0.0;
  }
  if (cell)
#pragma unroll
    for (int f = 0; f < MF; ++f) contrib[((fslot + f) * p.n + c) * NV + v] = fb[f];
}

// k_adj_lsq: one lane per cell, the transpose of the stencil least squares,
// shaped like k_lsq: DH rows of Gb in registers per pass, the members of
// the stencil streamed; a member's contribution is the sum of its row
// passes (the first writes, the next add).  Contributions go to slot-major
// buffers: slot 0 the cell, 1 + l*IMAX + k member k of stencil l (CWENO:
// 1 + IMAX + (l-1)*IMAX2 + k for the lower-order stencils).
template <int P>
__global__ void __launch_bounds__(128) k_adj_lsq(Problem p, const double* __restrict__ gbar,
                                                 const double* __restrict__ selfc, double* __restrict__ contrib) {
  constexpr int ID = Deg<P>::ideg;
  constexpr int DH = LsqRows<P, double>::value;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n = p.n;
  if (c >= n) return;
  const int A = p.admis_max, IM = p.imax;
  const int adm = p.admis[c];
  const int64_t grp = c >> 5;
  const int lane = (int)(c & 31);
  const double* Gb = gbar + grp * (int64_t)(A * ID * NV) * 32 + lane;
  const double* Mi = (const double*)p.invmat + grp * p.tstride * 32 + lane;
  double self[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) self[v] = selfc[c * NV + v];
  const bool cw = p.ees == 5;
  for (int ll = 0; ll < adm; ++ll) {
    const bool low = cw && ll > 0;
    const int nk = low ? p.imax2 : IM, nd = low ? p.ideg2 : ID;
    const int64_t slot0 = ll == 0 ? 1 : (cw ? 1 + IM + (int64_t)(ll - 1) * p.imax2 : 1 + (int64_t)ll * IM);
    for (int d0 = 0; d0 < nd; d0 += DH) {
      double gb[DH][NV];
#pragma unroll
      for (int j = 0; j < DH; ++j)
#pragma unroll
        for (int v = 0; v < NV; ++v) gb[j][v] = d0 + j < nd ? Gb[(int64_t)((ll * ID + d0 + j) * NV + v) * 32] : 0.0;
      const double* M = Mi + (int64_t)(p.soff[ll] + d0) * 32;
#pragma unroll 2
      for (int k = 0; k < nk; ++k) {
        const double* Mk = M + (int64_t)k * nd * 32;
        double a[NV] = {0, 0, 0, 0, 0};
#pragma unroll
        for (int j = 0; j < DH; ++j)
          if (d0 + j < nd) {
            const double m = Mk[j * 32];
#pragma unroll
            for (int v = 0; v < NV; ++v) a[v] += m * gb[j][v];
          }
        double* o = contrib + ((slot0 + k) * n + c) * NV;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          o[v] = d0 == 0 ? a[v] : o[v] + a[v];
          self[v] -= a[v];
        }
      }
    }
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) contrib[(int64_t)c * NV + v] = self[v];
}


// k_jvp_wpost: the tangent of the WENO face values (minus the cell mean)
// from the tangent stencil polynomials dG, thread layout of k_adj_wpost:
//   dIS_l = d(G_l^T S G_l),  dwt_l = -4 wt_l dIS_l / (eps + IS_l),
//   dom_l = (dwt_l - om_l sum dwt) / sum wt,
//   du(x) - dU_c = b(x) . sum_l (dom_l G_l + om_l dG_l).
// Cells on the MUSCL fall-back (decided as in k_adj_wpost): with
// out(x) = dd(x) slope, dout(x) = ddt(x) slope + dd(x) dslope,
//   dslope = dphi/ddd ddt(x*) + dphi/dlo dlo + dphi/dhi dhi,
// dlo = dU_nb - dU_c for the neighbour that set the bound; zero where
// CHECKSOLX reduced the cell to first order.
template <int P>
__global__ void __launch_bounds__(WP_THREADS, UCG_AWP_MINB) k_jvp_wpost(Problem p, const double* __restrict__ U,
                                                                        const double* __restrict__ dU,
                                                                        const double* __restrict__ dG,
                                                                        double* __restrict__ tdul) {
  constexpr int ID = Deg<P>::ideg;
  constexpr int VEC = Vec<double>::N;
  __shared__ double sGH[ID][NV][32];  // WENO combined polynomial, then the fall-back's G_0
  __shared__ double sSlope[NV][32];
  __shared__ int sFall[32];  // bit 0: MUSCL fall-back, bit 1: reduced to first order
  const int lane = threadIdx.x & 31, v = threadIdx.x >> 5;
  const int64_t grp = blockIdx.x;
  const int64_t c = grp * 32 + lane;
  const bool cell = c < p.n;
  const bool live = cell && p.full[c];
  if (v == 0) sFall[lane] = cell && !live ? 1 : 0;
  const int A = p.admis_max;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const int FQ = MF * QS;
  const double* xq = (const double*)p.qpts + grp * (int64_t)FQ * 3 * 32 + lane;
  const double* bmv = (const double*)p.bmean + grp * (int64_t)ID * 32 + lane;
  const int nf = cell ? p.nfaces[c] : 0;
  const double* Gc = (const double*)p.gbuf + grp * (int64_t)(A * ID * NV) * 32 + lane;
  const double* dGc = dG + grp * (int64_t)(A * ID * NV) * 32 + lane;
  auto G = [&](int ll, int d) -> double { return Gc[(int64_t)((ll * ID + d) * NV + v) * 32]; };
  auto dGv = [&](int ll, int d) -> double { return dGc[(int64_t)((ll * ID + d) * NV + v) * 32]; };
  if (live) {
    const int adm = p.admis[c];
    const double* Pc = (const double*)p.ind + grp * p.istride * 32 + lane * VEC;
    const double* Pc2 = Pc + (int64_t)(p.i2off / VEC) * 32 * VEC;
    const bool cw = p.ees == 5;
    const int ID2 = p.ideg2;
    constexpr int L2 = ID < 9 ? ID : 9;
    const double lc1 = 1.0 - 1.0 / p.lwci;
    const double lk = adm > 1 ? (1.0 - lc1) / (adm - 1) : 0.0;
    auto nd_of = [&](int ll) { return cw && ll > 0 ? ID2 : ID; };
    double g3[L2], dg3[L2];
#pragma unroll
    for (int d = 0; d < L2; ++d) g3[d] = dg3[d] = 0.0;
    if (cw)
      for (int l2 = 1; l2 < adm; ++l2)
#pragma unroll
        for (int d = 0; d < L2; ++d)
          if (d < ID2) {
            g3[d] = g3[d] + lk * G(l2, d);
            dg3[d] = dg3[d] + lk * dGv(l2, d);
          }
    auto poly = [&](int ll, int d) -> double {
      if (d >= nd_of(ll)) return 0.0;
      if (cw && ll == 0) return (1.0 / lc1) * (G(0, d) - (d < L2 ? g3[d] : 0.0));
      return G(ll, d);
    };
    auto dpoly = [&](int ll, int d) -> double {
      if (d >= nd_of(ll)) return 0.0;
      if (cw && ll == 0) return (1.0 / lc1) * (dGv(0, d) - (d < L2 ? dg3[d] : 0.0));
      return dGv(ll, d);
    };
    double is[7], dis[7], wt[7], dwt[7];
#pragma unroll 1
    for (int ll = 0; ll < adm; ++ll) {
      // IS = g^T S g and dIS = dg . (2 S g)
      double a, da = 0.0;
      if (cw && ll > 0) {
        double g[L2], gr[L2];
#pragma unroll
        for (int d = 0; d < L2; ++d) g[d] = poly(ll, d);
        a = is_and_grad<L2>(Pc2, g, ID2, gr);
#pragma unroll
        for (int d = 0; d < L2; ++d) da += dpoly(ll, d) * gr[d];
      } else {
        double g[ID], gr[ID];
#pragma unroll
        for (int d = 0; d < ID; ++d) g[d] = poly(ll, d);
        a = is_and_grad<ID>(Pc, g, ID, gr);
#pragma unroll
        for (int d = 0; d < ID; ++d) da += dpoly(ll, d) * gr[d];
      }
      is[ll] = a;
      dis[ll] = da;
    }
    // weights and their tangents (WENO-Z: wt = lam (1 + (tau / e)^4),
    // dwt = 4 (wt - lam) (dtau / tau - dIS / e))
    const bool wz = cw && p.wenoz;
    double tau = 0.0, dtau = 0.0, sum = 0.0, dsum = 0.0;
    if (wz) {
      for (int ll = 1; ll < adm; ++ll) {
        tau += fabs(is[0] - is[ll]);
        dtau += (is[0] > is[ll] ? 1.0 : (is[0] < is[ll] ? -1.0 : 0.0)) * (dis[0] - dis[ll]);
      }
      tau = tau / (adm - 1);
      dtau = dtau / (adm - 1);
    }
    for (int ll = 0; ll < adm; ++ll) {
      const double e = p.weno_eps + is[ll];
      const double lam = cw ? (ll == 0 ? lc1 : lk) : (ll == 0 ? p.lwci : 1.0);
      if (wz) {
        double q = tau / e;
        q = q * q;
        wt[ll] = lam * (1.0 + q * q);
        dwt[ll] = 4.0 * (wt[ll] - lam) * ((tau > 0.0 ? dtau / tau : 0.0) - dis[ll] / e);
      } else {
        const double e2 = e * e;
        wt[ll] = lam / (e2 * e2);
        dwt[ll] = -4.0 * wt[ll] * dis[ll] / e;
      }
      sum += wt[ll];
      dsum += dwt[ll];
    }
    // tangent and value of the combined polynomial (the value in shared
    // memory, for CHECKSOL)
    double td[ID];
#pragma unroll
    for (int d = 0; d < ID; ++d) {
      td[d] = 0.0;
      sGH[d][v][lane] = 0.0;
    }
#pragma unroll 1
    for (int ll = 0; ll < adm; ++ll) {
      const double om = wt[ll] / sum;
      const double dom = (dwt[ll] - om * dsum) / sum;
#pragma unroll
      for (int d = 0; d < ID; ++d) {
        const double gd = poly(ll, d);
        td[d] += dom * gd + om * dpoly(ll, d);
        sGH[d][v][lane] += om * gd;
        if ((d & 7) == 7) asm volatile("" ::: "memory");  // bound the loads in flight
      }
    }
    double tb = 0.0;
#pragma unroll
    for (int d = 0; d < ID; ++d) tb += bmv[d * 32] * td[d];
    for (int f = 0; f < MF; ++f) {
      const int nq = f < nf ? face_nq(p, p.ftype[c * MF + f]) : 0;
      for (int q = 0; q < QS; ++q) {
        double t = 0.0;
        if (q < nq) {
          const double* xi = xq + (int64_t)(f * QS + q) * 3 * 32;
          double m[ID];
          monomials<P, double>(xi[0], xi[32], xi[64], m);
#pragma unroll
          for (int d = 0; d < ID; ++d) t += m[d] * td[d];
          t -= tb;
        }
        tdul[(c * FQ + f * QS + q) * NV + v] = t;
      }
    }
  }
  __syncthreads();
  if (live && checksol_split<P>(p, U, c, nf, xq, bmv, sGH, lane, v)) atomicOr(&sFall[lane], 1);
  __syncthreads();
  // ---- MUSCL fall-back: the forward again, G_0 and the limiter value
  // shared for CHECKSOLX
  const bool fall = cell && (sFall[lane] & 1);
  double lo = 0.0, hi = 0.0, slope = TOLBIG, ddx = 0.0, epsi2 = 0.0, cb = 0.0, dcb = 0.0;
  int flo = -1, fhi = -1, xs = -1;
  const double u0v = cell ? U[c * NV + v] : 0.0;
  if (fall) {
    lo = hi = u0v;
    for (int f = 0; f < nf; ++f) {
      const int64_t nb = p.neigh[c * MF + f];
      if (nb < 0) continue;
      const double un = U[nb * NV + v];
      if (un < lo) lo = un, flo = f;
      if (un > hi) hi = un, fhi = f;
    }
    lo -= u0v;
    hi -= u0v;
    const double e3 = p.kappa_ven * p.minedge[c];
    epsi2 = e3 * e3 * e3;
    double g0[ID];
#pragma unroll
    for (int d = 0; d < ID; ++d) {
      g0[d] = G(0, d);
      cb += bmv[d * 32] * g0[d];
    }
    for (int f = 0; f < nf; ++f) {
      const int nq = face_nq(p, p.ftype[c * MF + f]);
      for (int q = 0; q < nq; ++q) {
        const double* xi = xq + (int64_t)(f * QS + q) * 3 * 32;
        double m[ID];
        monomials<P, double>(xi[0], xi[32], xi[64], m);
        double r = 0.0;
#pragma unroll
        for (int d = 0; d < ID; ++d) r += m[d] * g0[d];
        r = r - cb;
        const double dd = (u0v + r) - u0v;
        const double phi = venkat(dd, lo, hi, epsi2);
        if (phi < slope) slope = phi, xs = f * QS + q, ddx = dd;
      }
    }
#pragma unroll
    for (int d = 0; d < ID; ++d) sGH[d][v][lane] = g0[d];
    sSlope[v][lane] = slope;
  }
  __syncthreads();
  if (fall && checksolx_split<P>(p, U, c, nf, xq, bmv, sGH, sSlope, lane, v)) atomicOr(&sFall[lane], 2);
  __syncthreads();
  if (fall) {
    const bool first = (sFall[lane] & 2) || xs < 0;
    double dslope = 0.0;
    if (!first) {
#pragma unroll
      for (int d = 0; d < ID; ++d) dcb += bmv[d * 32] * dGv(0, d);
      const double* xi = xq + (int64_t)xs * 3 * 32;
      double m[ID];
      monomials<P, double>(xi[0], xi[32], xi[64], m);
      double ddt = 0.0;
#pragma unroll
      for (int d = 0; d < ID; ++d) ddt += m[d] * dGv(0, d);
      ddt -= dcb;
      ad::Dual<3> dd(ddx), dlo(lo), dhi(hi);
      dd.d[0] = 1.0;
      dlo.d[1] = 1.0;
      dhi.d[2] = 1.0;
      const ad::Dual<3> ph = venkat(dd, dlo, dhi, epsi2);
      const double du0 = dU[c * NV + v];
      const double tlo = flo >= 0 ? dU[(int64_t)p.neigh[c * MF + flo] * NV + v] - du0 : 0.0;
      const double thi = fhi >= 0 ? dU[(int64_t)p.neigh[c * MF + fhi] * NV + v] - du0 : 0.0;
      dslope = ph.d[0] * ddt + ph.d[1] * tlo + ph.d[2] * thi;
    }
    for (int f = 0; f < MF; ++f) {
      const int nq = f < nf ? face_nq(p, p.ftype[c * MF + f]) : 0;
      for (int q = 0; q < QS; ++q) {
        double t = 0.0;
        if (q < nq && !first) {
          const double* xi = xq + (int64_t)(f * QS + q) * 3 * 32;
          double m[ID];
          monomials<P, double>(xi[0], xi[32], xi[64], m);
          double r = 0.0, rt = 0.0;
#pragma unroll
          for (int d = 0; d < ID; ++d) {
            r += m[d] * sGH[d][v][lane];
            rt += m[d] * dGv(0, d);
            if ((d & 7) == 7) asm volatile("" ::: "memory");  // bound the loads in flight
          }
          const double dd = (u0v + (r - cb)) - u0v;
          t = (rt - dcb) * slope + dd * dslope;
        }
        tdul[(c * FQ + f * QS + q) * NV + v] = t;
      }
    }
  }
}

// ------------------------------------------------------------ viscous terms
// Navier-Stokes: the forward pass forms, per cell, the coefficients of the
// viscous least squares on (T, u, v, w) over the central stencil,
//   gv[c][d][a] = sum_k M_0[k][d] (S_a(U_st(k)) - S_a(U_c))   (k_visc_lsq),
// per face point the gradient of each side, J_c^T sum_d gv[c][d][a] dm_d(xi)
// (SOLUTIONTRIAV2, k_visc_facegrad), and the viscous flux from their mean.
// gpt[c][f][q][12] holds the adjoint of cell c's own gradient at its point
// q of face f (k_adj_visc); these kernels take it back to U.

// thread per (cell, variable a): gvb[c][d][a] = sum over the cell's face
// points of (J_c gpt_a) . dm_d(xi)
template <int P>
__global__ void __launch_bounds__(128) k_adj_visc_coef(Problem p, const double* __restrict__ gpt,
                                                       double* __restrict__ gvb) {
  constexpr int ID = Deg<P>::ideg;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t c = t >> 2;
  const int a = (int)(t & 3);
  if (c >= p.n) return;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const double* J = p.jinv + c * 9;
  double acc[ID];
#pragma unroll
  for (int d = 0; d < ID; ++d) acc[d] = 0.0;
  const int nf = p.nfaces[c];
  for (int f = 0; f < nf; ++f) {
    const int nq = face_nq(p, p.ftype[c * MF + f]);
    for (int q = 0; q < nq; ++q) {
      const double* g = gpt + (((c * MF + f) * QS + q) * 12 + a * 3);
      // the gradient's component k is sum_j J[j][k] (d/dxi_j of the polynomial)
      const double t0 = J[0] * g[0] + J[1] * g[1] + J[2] * g[2];
      const double t1 = J[3] * g[0] + J[4] * g[1] + J[5] * g[2];
      const double t2 = J[6] * g[0] + J[7] * g[1] + J[8] * g[2];
      const double* xi = (const double*)p.qpts + ((c >> 5) * MF * QS * 3 + (f * QS + q) * 3) * 32 + (c & 31);
      double dx[ID], dy[ID], dz[ID];
      dmonomials<P, double>(xi[0], xi[32], xi[64], dx, dy, dz);
#pragma unroll
      for (int d = 0; d < ID; ++d) acc[d] += t0 * dx[d] + t1 * dy[d] + t2 * dz[d];
    }
  }
#pragma unroll
  for (int d = 0; d < ID; ++d) gvb[(c * ID + d) * 4 + a] = acc[d];
}

// thread per cell: the transpose of the viscous least squares into the
// slots of k_adj_lsq (slot 0 the cell, 1 + k member k of the central
// stencil), added to what k_adj_lsq wrote there: one writer per slot
template <int P>
__global__ void __launch_bounds__(128) k_adj_visc_lsq(Problem p, const double* __restrict__ U,
                                                      const double* __restrict__ gvb, double* __restrict__ contrib) {
  constexpr int ID = Deg<P>::ideg;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n = p.n;
  if (c >= n) return;
  const int IM = p.imax, W = IM + 1;
  const int64_t grp = c >> 5;
  const int lane = (int)(c & 31);
  const int32_t* st = p.sten + grp * (int64_t)p.admis_max * W * 32 + lane;
  const double* M = (const double*)p.invmat + (grp * p.tstride + p.soff[0]) * 32 + lane;
  const double* gb = gvb + c * ID * 4;
  double sc[4] = {0, 0, 0, 0};
  for (int k = 0; k < IM; ++k) {
    double a[4] = {0, 0, 0, 0};
#pragma unroll 4
    for (int d = 0; d < ID; ++d) {
      const double m = M[(k * ID + d) * 32];
#pragma unroll
      for (int j = 0; j < 4; ++j) a[j] += m * gb[d * 4 + j];
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) sc[j] -= a[j];
    double out[NV];
    ad::visc_vars_rev(p, U + (int64_t)st[(k + 1) * 32] * NV, a, out);
    double* o = contrib + ((1 + k) * n + c) * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] += out[v];
  }
  double out[NV];
  ad::visc_vars_rev(p, U + c * NV, sc, out);
#pragma unroll
  for (int v = 0; v < NV; ++v) contrib[c * NV + v] += out[v];
}

// thread per (cell, variable a): the tangent of the coefficients,
// dgv[c][d][a] = sum_k M_0[k][d] (dS_a(st(k)) - dS_a(c)), in k_visc_lsq's
// layout [n][ID][4]
template <int P>
__global__ void __launch_bounds__(128) k_jvp_visc_coef(Problem p, const double* __restrict__ U,
                                                       const double* __restrict__ dU, double* __restrict__ dgv) {
  constexpr int ID = Deg<P>::ideg;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t c = t >> 2;
  const int a = (int)(t & 3);
  if (c >= p.n) return;
  const int IM = p.imax, W = IM + 1;
  const int64_t grp = c >> 5;
  const int lane = (int)(c & 31);
  const int32_t* st = p.sten + grp * (int64_t)p.admis_max * W * 32 + lane;
  const double* M = (const double*)p.invmat + (grp * p.tstride + p.soff[0]) * 32 + lane;
  const double sc = ad::visc_var_tan(p, U + c * NV, dU + c * NV, a);
  double acc[ID];
#pragma unroll
  for (int d = 0; d < ID; ++d) acc[d] = 0.0;
  for (int k = 0; k < IM; ++k) {
    const int64_t y = st[(k + 1) * 32];
    const double ds = ad::visc_var_tan(p, U + y * NV, dU + y * NV, a) - sc;
#pragma unroll
    for (int d = 0; d < ID; ++d) acc[d] += M[(k * ID + d) * 32] * ds;
  }
#pragma unroll
  for (int d = 0; d < ID; ++d) dgv[(c * ID + d) * 4 + a] = acc[d];
}

template <int P>
void launch_visc_t(const Problem& p, const double* U, const double* gpt, double* gvb, double* contrib,
                   cudaStream_t st) {
  k_adj_visc_coef<P><<<(unsigned)((p.n * 4 + 127) / 128), 128, 0, st>>>(p, gpt, gvb);
  k_adj_visc_lsq<P><<<(unsigned)((p.n + 127) / 128), 128, 0, st>>>(p, U, gvb, contrib);
}

// the tangent of the face-point gradients: the coefficients' tangent, then
// k_visc_facegrad itself (linear in the coefficients) on it
template <int P>
void launch_visc_jvp_t(const Problem& p, const double* U, const double* dU, double* dgv, double* tfg,
                       cudaStream_t st) {
  k_jvp_visc_coef<P><<<(unsigned)((p.n * 4 + 127) / 128), 128, 0, st>>>(p, U, dU, dgv);
  Problem pt = p;
  pt.gv = dgv;
  pt.fgrad = tfg;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const int64_t nfp = p.nown * QS;
  k_visc_facegrad<P, double><<<(unsigned)((nfp + 127) / 128), 128, 0, st>>>(pt);
}

template <int P>
void launch_t(const Problem& p, const double* U, const double* adjF, double* gbar, double* scr, double* selfc,
              double* contrib, cudaStream_t st) {
  k_adj_wpost<P><<<(unsigned)((p.n + 31) / 32), WP_THREADS, 0, st>>>(p, U, adjF, gbar, scr, selfc, contrib);
  k_adj_lsq<P><<<(unsigned)((p.n + 127) / 128), 128, 0, st>>>(p, gbar, selfc, contrib);
}

template <int P>
void launch_jvp_t(const Problem& p, const double* U, const double* dU, const double* dG, double* tdul,
                  cudaStream_t st) {
  k_jvp_wpost<P><<<(unsigned)((p.n + 31) / 32), WP_THREADS, 0, st>>>(p, U, dU, dG, tdul);
}

}  // namespace

namespace ucg_host {

int launch_weno_tangent(ucg_engine* e, const Problem& p, const double* U, const double* dU, const double* dG,
                        double* tdul) {
  switch (e->cfg.iorder) {
    case 1: launch_jvp_t<1>(p, U, dU, dG, tdul, e->stream); break;
    case 2: launch_jvp_t<2>(p, U, dU, dG, tdul, e->stream); break;
    case 3: launch_jvp_t<3>(p, U, dU, dG, tdul, e->stream); break;
    case 4: launch_jvp_t<4>(p, U, dU, dG, tdul, e->stream); break;
    default: return fail(e, UCG_EINVAL, "iorder out of range");
  }
  e->launches++;
  CK(cudaGetLastError());
  return UCG_OK;
}


int launch_weno_visc_adjoint(ucg_engine* e, const Problem& p, const double* U, const double* gpt, double* gvb,
                             double* contrib) {
  switch (e->cfg.iorder) {
    case 1: launch_visc_t<1>(p, U, gpt, gvb, contrib, e->stream); break;
    case 2: launch_visc_t<2>(p, U, gpt, gvb, contrib, e->stream); break;
    case 3: launch_visc_t<3>(p, U, gpt, gvb, contrib, e->stream); break;
    case 4: launch_visc_t<4>(p, U, gpt, gvb, contrib, e->stream); break;
    default: return fail(e, UCG_EINVAL, "iorder out of range");
  }
  e->launches += 2;
  CK(cudaGetLastError());
  return UCG_OK;
}

int launch_weno_visc_tangent(ucg_engine* e, const Problem& p, const double* U, const double* dU, double* dgv,
                             double* tfg) {
  switch (e->cfg.iorder) {
    case 1: launch_visc_jvp_t<1>(p, U, dU, dgv, tfg, e->stream); break;
    case 2: launch_visc_jvp_t<2>(p, U, dU, dgv, tfg, e->stream); break;
    case 3: launch_visc_jvp_t<3>(p, U, dU, dgv, tfg, e->stream); break;
    case 4: launch_visc_jvp_t<4>(p, U, dU, dgv, tfg, e->stream); break;
    default: return fail(e, UCG_EINVAL, "iorder out of range");
  }
  e->launches += 2;
  CK(cudaGetLastError());
  return UCG_OK;
}

int launch_weno_adjoint(ucg_engine* e, const Problem& p, const double* U, const double* adjF, double* gbar,
                        double* scr, double* selfc, double* contrib) {
  switch (e->cfg.iorder) {
    case 1: launch_t<1>(p, U, adjF, gbar, scr, selfc, contrib, e->stream); break;
    case 2: launch_t<2>(p, U, adjF, gbar, scr, selfc, contrib, e->stream); break;
    case 3: launch_t<3>(p, U, adjF, gbar, scr, selfc, contrib, e->stream); break;
    case 4: launch_t<4>(p, U, adjF, gbar, scr, selfc, contrib, e->stream); break;
    default: return fail(e, UCG_EINVAL, "iorder out of range");
  }
  e->launches += 2;
  CK(cudaGetLastError());
  return UCG_OK;
}

}  // namespace ucg_host
