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
// A cell whose CHECKSOL test (or FULL = 0) put it on the MUSCL fall-back is
// not covered: the kernel raises a flag and the VJP returns UCG_EINVAL.
#include <cuda_runtime.h>

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

// k_adj_wpost: writes Gb (layout of the stencil polynomials G) and the
// direct adjoint of the cell mean (selfc); scr holds Bb (interleaved like
// G).  Gb first receives 2 S G_l (the gradient of IS_l), read back once the
// weights' adjoints are known.
template <int P>
__global__ void __launch_bounds__(WP_THREADS, UCG_AWP_MINB) k_adj_wpost(Problem p, const double* __restrict__ U,
                                                             const double* __restrict__ adjF,
                                                             double* __restrict__ gbar, double* __restrict__ scr,
                                                             double* __restrict__ selfc, int* __restrict__ flag) {
  constexpr int ID = Deg<P>::ideg;
  constexpr int VEC = Vec<double>::N;
  __shared__ double sGH[ID][NV][32];
  const int lane = threadIdx.x & 31, v = threadIdx.x >> 5;
  const int64_t grp = blockIdx.x;
  const int64_t c = grp * 32 + lane;
  const bool live = c < p.n && p.full[c];
  if (c < p.n && !p.full[c] && v == 0) atomicOr(flag, 1);
  const int A = p.admis_max;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const int FQ = MF * QS;
  const double* xq = (const double*)p.qpts + grp * (int64_t)FQ * 3 * 32 + lane;
  const double* bmv = (const double*)p.bmean + grp * (int64_t)ID * 32 + lane;
  if (live) {
    const int adm = p.admis[c], nf = p.nfaces[c];
    const double* Gc = (const double*)p.gbuf + grp * (int64_t)(A * ID * NV) * 32 + lane;
    auto G = [&](int ll, int d) -> double { return Gc[(int64_t)((ll * ID + d) * NV + v) * 32]; };
    double* Gb = gbar + grp * (int64_t)(A * ID * NV) * 32 + lane;
    auto GB = [&](int ll, int d) -> double& { return Gb[(int64_t)((ll * ID + d) * NV + v) * 32]; };
    double* BBp = scr + grp * (int64_t)(ID * NV) * 32 + lane;
    auto BB = [&](int d) -> double& { return BBp[(int64_t)(d * NV + v) * 32]; };
    const double* aF = adjF + c * (int64_t)FQ * NV + v;
    // ---- the direct term and Bb = sum_x ub(x) (m(x) - mean(m))
    {
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
    // ---- indicators and weights.  CWENO (EES 5): the central polynomial is
    // g1 = (G_0 - sum_l lk G_l) / lc1 (rows below IDEGFREE2 for the
    // lower-order stencils), the lower-order stencils have IDEGFREE2 rows and
    // the S2 triangle, the linear weights are lc1, lk.
    const double* Pc = (const double*)p.ind + grp * p.istride * 32 + lane * VEC;
    const double* Pc2 = Pc + (int64_t)(p.i2off / VEC) * 32 * VEC;
    const bool cw = p.ees == 5;
    const int ID2 = p.ideg2;
    constexpr int L2 = ID < 9 ? ID : 9;
    const double lc1 = 1.0 - 1.0 / p.lwci;
    const double lk = adm > 1 ? (1.0 - lc1) / (adm - 1) : 0.0;
    auto nd_of = [&](int ll) { return cw && ll > 0 ? ID2 : ID; };
    double g3[L2];
#pragma unroll
    for (int d = 0; d < L2; ++d) g3[d] = 0.0;
    if (cw)
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
    double is[7], wt[7], om[7], omb[7];
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
    const bool wz = cw && p.wenoz;
    double tau = 0.0, sum = 0.0;
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
    // ---- combined polynomial (CHECKSOL) and the weights' adjoints
    double dot = 0.0;
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
  __syncthreads();
  // ---- CHECKSOL (0.85) on the WENO face values: a flagged cell took the
  // MUSCL fall-back in the forward, which this adjoint does not cover
  if (live && checksol_split<P>(p, U, c, p.nfaces[c], xq, bmv, sGH, lane, v)) atomicOr(flag, 1);
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
// Same fall-back flag as k_adj_wpost; a cell on it gets a zero tangent.
template <int P>
__global__ void __launch_bounds__(WP_THREADS, UCG_AWP_MINB) k_jvp_wpost(Problem p, const double* __restrict__ U,
                                                                        const double* __restrict__ dG,
                                                                        double* __restrict__ tdul,
                                                                        int* __restrict__ flag) {
  constexpr int ID = Deg<P>::ideg;
  constexpr int VEC = Vec<double>::N;
  __shared__ double sGH[ID][NV][32];
  const int lane = threadIdx.x & 31, v = threadIdx.x >> 5;
  const int64_t grp = blockIdx.x;
  const int64_t c = grp * 32 + lane;
  const bool live = c < p.n && p.full[c];
  if (c < p.n && !p.full[c] && v == 0) atomicOr(flag, 1);
  const int A = p.admis_max;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const int FQ = MF * QS;
  const double* xq = (const double*)p.qpts + grp * (int64_t)FQ * 3 * 32 + lane;
  const double* bmv = (const double*)p.bmean + grp * (int64_t)ID * 32 + lane;
  if (c < p.n && !live)
    for (int i = 0; i < FQ; ++i) tdul[(c * FQ + i) * NV + v] = 0.0;
  if (live) {
    const int adm = p.admis[c], nf = p.nfaces[c];
    const double* Gc = (const double*)p.gbuf + grp * (int64_t)(A * ID * NV) * 32 + lane;
    const double* dGc = dG + grp * (int64_t)(A * ID * NV) * 32 + lane;
    auto G = [&](int ll, int d) -> double { return Gc[(int64_t)((ll * ID + d) * NV + v) * 32]; };
    auto dGv = [&](int ll, int d) -> double { return dGc[(int64_t)((ll * ID + d) * NV + v) * 32]; };
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
  if (live && checksol_split<P>(p, U, c, p.nfaces[c], xq, bmv, sGH, lane, v)) atomicOr(flag, 1);
}

template <int P>
void launch_t(const Problem& p, const double* U, const double* adjF, double* gbar, double* scr, double* selfc,
              double* contrib, int* flag, cudaStream_t st) {
  k_adj_wpost<P><<<(unsigned)((p.n + 31) / 32), WP_THREADS, 0, st>>>(p, U, adjF, gbar, scr, selfc, flag);
  k_adj_lsq<P><<<(unsigned)((p.n + 127) / 128), 128, 0, st>>>(p, gbar, selfc, contrib);
}

template <int P>
void launch_jvp_t(const Problem& p, const double* U, const double* dG, double* tdul, int* flag, cudaStream_t st) {
  k_jvp_wpost<P><<<(unsigned)((p.n + 31) / 32), WP_THREADS, 0, st>>>(p, U, dG, tdul, flag);
}

}  // namespace

namespace ucg_host {

int launch_weno_tangent(ucg_engine* e, const Problem& p, const double* U, const double* dG, double* tdul,
                        int* flag) {
  switch (e->cfg.iorder) {
    case 1: launch_jvp_t<1>(p, U, dG, tdul, flag, e->stream); break;
    case 2: launch_jvp_t<2>(p, U, dG, tdul, flag, e->stream); break;
    case 3: launch_jvp_t<3>(p, U, dG, tdul, flag, e->stream); break;
    case 4: launch_jvp_t<4>(p, U, dG, tdul, flag, e->stream); break;
    default: return fail(e, UCG_EINVAL, "iorder out of range");
  }
  e->launches++;
  CK(cudaGetLastError());
  return UCG_OK;
}


int launch_weno_adjoint(ucg_engine* e, const Problem& p, const double* U, const double* adjF, double* gbar,
                        double* scr, double* selfc, double* contrib, int* flag) {
  switch (e->cfg.iorder) {
    case 1: launch_t<1>(p, U, adjF, gbar, scr, selfc, contrib, flag, e->stream); break;
    case 2: launch_t<2>(p, U, adjF, gbar, scr, selfc, contrib, flag, e->stream); break;
    case 3: launch_t<3>(p, U, adjF, gbar, scr, selfc, contrib, flag, e->stream); break;
    case 4: launch_t<4>(p, U, adjF, gbar, scr, selfc, contrib, flag, e->stream); break;
    default: return fail(e, UCG_EINVAL, "iorder out of range");
  }
  e->launches += 2;
  CK(cudaGetLastError());
  return UCG_OK;
}

}  // namespace ucg_host
