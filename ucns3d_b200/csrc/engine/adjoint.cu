// Discrete adjoint (VJP) and tangent (JVP) of the engine's MUSCL residual,
// of the wall pressure force and of SSP-RK3 steps, for the FP64 form of a
// MUSCL (scheme 2, IORDER 1) Euler or Navier-Stokes configuration; the
// host side of the WENO/CWENO residual's (adjoint_weno.cu), whose viscous
// fluxes are reversed here too (k_adj_visc over the face points).
//
// Residual R(U) = net outward flux (CALL_FLUX_SUBROUTINES_3D,
// src/time_p.f90:2253-2497); force J(U) = sum over wall faces (BC code 4) of
// (sum_q w_q p(u_face,q) - PRES) * area * n_x (COMPUTEFORCE,
// src/io.f90:18752-18915, inviscid part).
//
// VJP of R: mu = (dR/dU)^T lambda, pbar = (dR/dp)^T lambda (p: the
// free-stream state of the inflow/outflow conditions, Problem::bc_state).
//   0. k_adj_fwd       one thread per cell: the MUSCL reconstruction (the
//                      face values k_muscl writes) with its intermediates
//                      kept, field-major, for step 2.
//   1. k_adj_face      one thread per interior or mirror face: the reverse
//                      sweep of HLLC (ad::hllc_adj) applied to
//                      lambda_c - lambda_nb; k_adj_face_bnd, one thread per
//                      other boundary face and input direction: one column
//                      of the 5x10 Jacobian w.r.t. the face value and p
//                      from dual numbers.  Together they
//                      give the adjoint of every face value.
//   2. k_adj_muscl     one thread per cell: the MUSCL reconstruction (LSQ,
//                      FIND_BOUNDS, Venkatakrishnan, CHECKSOLX) reversed by
//                      hand; its contributions to the cell, its stencil
//                      cells and the face neighbours outside the stencil go
//                      to per-slot buffers, each written once.
//   3. k_adj_gather    one thread per cell: sums the slots that point at it,
//                      through a reverse map built on the host in a fixed
//                      order, so results are deterministic (no atomics).
//   4. k_colsum5_part, k_colsum5: pbar, summed over the other boundary faces
//                      in a fixed order.
// Navier-Stokes adds k_adj_visc (the viscous flux reversed at each face
// point, after step 1) and the reverse of the viscous gradients in step 2.
// JVP: the same reconstruction and fluxes on Dual<1> numbers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "ad.cuh"
#include "engine_internal.h"

using namespace ucg;
using namespace ucg_host;
using ad::cons2prim_rev;
using ad::Dual;
using ad::visc_vars_rev;

namespace {

// ------------------------------------------------------------ set-up checks
int adj_check(ucg_engine* e) {
  if (!e) return UCG_EINVAL;
  const ucg_config& c = e->cfg;
  if (!(c.scheme == 2 && c.iorder == 1 && (c.governing == 2 || c.governing == 1) && c.precision == UCG_FP64 &&
        c.riemann == 1 && c.limiter == 7 && !c.mood))
    return fail(e, UCG_EINVAL,
                "the adjoint covers MUSCL (scheme 2, IORDER 1, Venkatakrishnan), HLLC, Euler or Navier-Stokes, FP64 form");
  if (e->QS != 1) return fail(e, UCG_EINVAL, "the adjoint needs one face point per face (IORDER 1)");
  if (!ready(e) || !e->have_state) return fail(e, UCG_ESTATE, "geometry, tables and state are needed");
  if (!e->roles.empty()) return fail(e, UCG_EINVAL, "the adjoint covers whole meshes (no partition roles)");
  return UCG_OK;
}

// elementwise: y = a*x + b*y  (n*5)
__global__ void k_axpby(int64_t m, double a, const double* __restrict__ x, double b, double* __restrict__ y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) y[i] = a * x[i] + b * y[i];
}
// lam[c][v] = s * x[c][v] / V_c
__global__ void k_over_vol(Problem p, double s, const double* __restrict__ x, double* __restrict__ lam) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < p.n * NV) lam[i] = s * x[i] / p.vol[i / NV];
}
// acc[k] += s * part[k], k < 5
__global__ void k_pacc(double s, const double* __restrict__ part, double* __restrict__ acc) {
  if (threadIdx.x < NV) acc[threadIdx.x] += s * part[threadIdx.x];
}

// deterministic column sums of a [m][5] array: block k sums column k
__global__ void __launch_bounds__(256) k_colsum5(const double* __restrict__ a, int64_t m, double* __restrict__ out) {
  const int k = blockIdx.x;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < m; i += blockDim.x) s += a[i * NV + k];
  __shared__ double sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[k] = sh[0];
}
// deterministic sum of a [m] array
__global__ void __launch_bounds__(1024) k_sum1(const double* __restrict__ a, int64_t m, double* __restrict__ out) {
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < m; i += blockDim.x) s += a[i];
  __shared__ double sh[1024];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// ------------------------------------------------------------ face VJP
// adjF[c][f][q] = adjoint of the face value of cell c at point q of face f
// ([n][F][QS][5]; one point per face for MUSCL IORDER 1).  The owned faces
// come grouped (interior, mirror boundaries, other boundaries), and the two
// kinds of kernel below take disjoint ranges of that list.
struct FaceRef {
  int64_t c, nb;
  int f, nf, nq, QS;
};
__device__ __forceinline__ FaceRef face_ref(const Problem& p, int64_t i) {
  FaceRef F;
  const int32_t code = p.own[i];
  F.c = code >> 3;
  F.f = code & 7;
  F.nb = p.neigh[F.c * MF + F.f];
  F.nf = p.nface[F.c * MF + F.f];
  F.nq = face_nq(p, p.ftype[F.c * MF + F.f]);
  F.QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  return F;
}
// inputs of face point q: the two face values (the free-stream state as the
// second input of a boundary face), the weighted adjoint difference g, and
// the neighbour's point qq
__device__ __forceinline__ void adj_face_inputs(const Problem& p, const double* __restrict__ U,
                                                const double* __restrict__ lam, const FaceRef& F, int q,
                                                double* r, double* ul, double* ur, double* g, int& qq) {
  const int64_t c = F.c, nb = F.nb;
  const int f = F.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) r[k] = p.rot[(c * MF + f) * 4 + k];
  const double ws = face_weight(p, p.ftype[c * MF + f], q) * p.area[c * MF + f];
  const double* dul = (const double*)p.dul;
  qq = nb >= 0 ? p.qperm[(c * MF + f) * F.QS + q] : 0;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    ul[v] = U[c * NV + v] + dul[((c * MF + f) * F.QS + q) * NV + v];
    if (nb >= 0) {
      ur[v] = U[nb * NV + v] + dul[((nb * MF + F.nf) * F.QS + qq) * NV + v];
      g[v] = ws * (lam[c * NV + v] - lam[nb * NV + v]);
    } else {
      ur[v] = p.bc_state[v];  // free-stream state, the second input of a boundary face
      g[v] = ws * lam[c * NV + v];
    }
  }
}

// Interior and mirror faces, owned faces [0, nplain): reverse sweep of HLLC
// (ad::hllc_adj) in the face frame at every face point.  The rotations are
// orthogonal (rot_b = rot_f^T), and a mirror ghost is b = S a in the face
// frame (S flips the normal momentum; a Navier-Stokes wall, no slip, flips
// the whole momentum).
__global__ void __launch_bounds__(64) k_adj_face(Problem p, int64_t nplain, const double* __restrict__ U,
                                                  const double* __restrict__ lam, double* __restrict__ adjF) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nplain) return;
  const FaceRef F = face_ref(p, i);
  for (int q = 0; q < F.nq; ++q) {
    double r[4], ul[NV], ur[NV], g[NV];
    int qq;
    adj_face_inputs(p, U, lam, F, q, r, ul, ur, g, qq);
    double a[NV], b[NV], hb[NV], ab[NV] = {0, 0, 0, 0, 0}, bb[NV] = {0, 0, 0, 0, 0}, o[NV];
    rot_f(r, ul, a);
    const bool noslip = F.nb < 0 && p.governing == 1 && p.bc[F.c * MF + F.f] == 4;
    auto flip = [&](int v) { return noslip ? (v >= 1 && v <= 3) : v == 1; };
    if (F.nb >= 0) {
      rot_f(r, ur, b);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) b[v] = flip(v) ? -a[v] : a[v];
    }
    rot_f(r, g, hb);
    ad::hllc_adj(p.gamma, a, b, hb, ab, bb);
    if (F.nb < 0)
#pragma unroll
      for (int v = 0; v < NV; ++v) ab[v] += flip(v) ? -bb[v] : bb[v];
    rot_b(r, ab, o);
#pragma unroll
    for (int k = 0; k < NV; ++k) adjF[((F.c * MF + F.f) * F.QS + q) * NV + k] = o[k];
    if (F.nb >= 0) {
      rot_b(r, bb, o);
#pragma unroll
      for (int k = 0; k < NV; ++k) adjF[((F.nb * MF + F.nf) * F.QS + qq) * NV + k] = o[k];
    }
  }
}

// The other boundary faces, owned faces [nplain, nown): their ghost state
// depends on the free stream, so the 5x10 Jacobian of the face flux w.r.t.
// the face value and the free-stream state is formed one input direction
// at a time (Dual<1>), one thread per face and direction k (k < 5: the face
// value, k >= 5: the free-stream state).  pown[i - nplain] = adjoint of the
// free-stream state, summed over the face's points.
__global__ void __launch_bounds__(128) k_adj_face_bnd(Problem p, int64_t nplain, const double* __restrict__ U,
                                                      const double* __restrict__ lam, double* __restrict__ adjF,
                                                      double* __restrict__ pown) {
  using D = Dual<1>;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = nplain + t / 10;
  const int k = (int)(t % 10);
  if (i >= p.nown) return;
  const FaceRef F = face_ref(p, i);
  const int bcode = p.bc[F.c * MF + F.f];
  double sp = 0.0;
  for (int q = 0; q < F.nq; ++q) {
    double r[4], ul[NV], ur[NV], g[NV];
    int qq;
    adj_face_inputs(p, U, lam, F, q, r, ul, ur, g, qq);
    D L[NV], R[NV], bcs[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      L[v] = D(ul[v]);
      L[v].d[0] = v == k ? 1.0 : 0.0;
      bcs[v] = D(ur[v]);
      bcs[v].d[0] = v + 5 == k ? 1.0 : 0.0;
    }
    boundary_ghost(p, bcode, r, L, bcs, R);
    D a[NV], b[NV], h[NV], fl[NV];
    rot_f(r, R, b);
    rot_f(r, L, a);
    hllc(p.gamma, a, b, h);
    rot_b(r, h, fl);
    double s = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) s += g[v] * fl[v].d[0];
    if (k < NV) adjF[((F.c * MF + F.f) * F.QS + q) * NV + k] = s;
    else sp += s;
  }
  if (k >= NV) pown[(i - nplain) * NV + (k - NV)] = sp;
}

// Viscous face fluxes (Navier-Stokes): the adjoint of their inputs, one
// Reverse of viscous_flux (CALCULATE_FLUXESHI_DIFFUSIVE, flux_p.f90:1520-2107,
// with SUTHERLAND) for one face point: given fb = the adjoint of the face's
// viscous flux, the adjoints of its inputs, the two face states cl, cr and
// the face gradients gl, gr ([T, u, v, w][x, y, z]), which the flux takes
// only as their mean gm = (gl + gr)/2, so that both have the adjoint gb.
// The forward
// quantities are recomputed in FP64; the flux is linear in the averaged
// gradients and in the stresses, so the sweep is written out by hand, and
// only Sutherland's law in (rho, p) takes dual numbers (2 columns).
// Overwrites clb, crb, gb.
__device__ __forceinline__ void viscous_flux_rev(const Problem& p, const double* r, double dih, const double* cl,
                                                 const double* cr, const double* gm, double damp, const double* fb,
                                                 double* clb, double* crb, double* gb) {
  const double nn[3] = {r[0] * r[3], r[1] * r[3], r[2]};
  double lv[NV], rv[NV];
  cons2prim(p.gamma, cl, lv);
  cons2prim(p.gamma, cr, rv);
  Dual<2> mul, laml, mur, lamr;
  {
    Dual<2> rho(lv[0]), pr(lv[4]);
    rho.d[0] = 1.0;
    pr.d[1] = 1.0;
    sutherland(p, rho, pr, &mul, &laml);
    rho = Dual<2>(rv[0]);
    pr = Dual<2>(rv[4]);
    rho.d[0] = 1.0;
    pr.d[1] = 1.0;
    sutherland(p, rho, pr, &mur, &lamr);
  }
  const double Tl = lv[4] / (lv[0] * p.r_gas), Tr = rv[4] / (rv[0] * p.r_gas);
  const double jump[4] = {rv[1] - lv[1], rv[2] - lv[2], rv[3] - lv[3], Tr - Tl};
  const int src[4] = {1, 2, 3, 0};
  const double vd = (4.0 / 3.0) / fabs(dih);
  double gg[4][3];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      gg[a][k] = gm[src[a] * 3 + k] + damp * (vd * nn[k] * jump[a]);
  const double lam2 = 0.5 * (laml.v + lamr.v), mu2 = 0.5 * (mul.v + mur.v);
  const double ux = gg[0][0], uy = gg[0][1], uz = gg[0][2];
  const double vx = gg[1][0], vy = gg[1][1], vz = gg[1][2];
  const double wx = gg[2][0], wy = gg[2][1], wz = gg[2][2];
  const double axx = (4.0 / 3.0) * ux - (2.0 / 3.0) * vy - (2.0 / 3.0) * wz;
  const double ayy = (4.0 / 3.0) * vy - (2.0 / 3.0) * ux - (2.0 / 3.0) * wz;
  const double azz = (4.0 / 3.0) * wz - (2.0 / 3.0) * ux - (2.0 / 3.0) * vy;
  const double axy = uy + vx, axz = wx + uz, ayz = vz + wy;
  const double txx = mu2 * axx, tyy = mu2 * ayy, tzz = mu2 * azz;
  const double txy = mu2 * axy, txz = mu2 * axz, tyz = mu2 * ayz;
  const double rho12 = 0.5 * (cl[0] + cr[0]);
  const double u12 = 0.5 * (cl[1] + cr[1]) / rho12, v12 = 0.5 * (cl[2] + cr[2]) / rho12,
               w12 = 0.5 * (cl[3] + cr[3]) / rho12;
  // fv1..3 = n . tau, fv4 = n . (-Q + tau u12)
  const double f4x = nn[0] * fb[4], f4y = nn[1] * fb[4], f4z = nn[2] * fb[4];
  double txxb = nn[0] * fb[1] + f4x * u12;
  double tyyb = nn[1] * fb[2] + f4y * v12;
  double tzzb = nn[2] * fb[3] + f4z * w12;
  double txyb = nn[1] * fb[1] + nn[0] * fb[2] + f4x * v12 + f4y * u12;
  double txzb = nn[2] * fb[1] + nn[0] * fb[3] + f4x * w12 + f4z * u12;
  double tyzb = nn[2] * fb[2] + nn[1] * fb[3] + f4y * w12 + f4z * v12;
  const double u12b = f4x * txx + f4y * txy + f4z * txz;
  const double v12b = f4x * txy + f4y * tyy + f4z * tyz;
  const double w12b = f4x * txz + f4y * tyz + f4z * tzz;
  const double lam2b = f4x * gg[3][0] + f4y * gg[3][1] + f4z * gg[3][2];
  const double mu2b = txxb * axx + tyyb * ayy + tzzb * azz + txyb * axy + txzb * axz + tyzb * ayz;
  double ggb[4][3];
  ggb[0][0] = mu2 * ((4.0 / 3.0) * txxb - (2.0 / 3.0) * tyyb - (2.0 / 3.0) * tzzb);
  ggb[1][1] = mu2 * ((4.0 / 3.0) * tyyb - (2.0 / 3.0) * txxb - (2.0 / 3.0) * tzzb);
  ggb[2][2] = mu2 * ((4.0 / 3.0) * tzzb - (2.0 / 3.0) * txxb - (2.0 / 3.0) * tyyb);
  ggb[0][1] = ggb[1][0] = mu2 * txyb;
  ggb[0][2] = ggb[2][0] = mu2 * txzb;
  ggb[1][2] = ggb[2][1] = mu2 * tyzb;
  ggb[3][0] = lam2 * f4x;
  ggb[3][1] = lam2 * f4y;
  ggb[3][2] = lam2 * f4z;
  double jumpb[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    jumpb[a] = damp * vd * (nn[0] * ggb[a][0] + nn[1] * ggb[a][1] + nn[2] * ggb[a][2]);
#pragma unroll
    for (int k = 0; k < 3; ++k) gb[src[a] * 3 + k] = 0.5 * ggb[a][k];
  }
  // primitive adjoints: the jumps in (u, v, w, T) and the face viscosity
  double lvb[NV], rvb[NV];
  lvb[1] = -jumpb[0];
  lvb[2] = -jumpb[1];
  lvb[3] = -jumpb[2];
  rvb[1] = jumpb[0];
  rvb[2] = jumpb[1];
  rvb[3] = jumpb[2];
  lvb[4] = -jumpb[3] / (lv[0] * p.r_gas) + 0.5 * (mu2b * mul.d[1] + lam2b * laml.d[1]);
  lvb[0] = jumpb[3] * Tl / lv[0] + 0.5 * (mu2b * mul.d[0] + lam2b * laml.d[0]);
  rvb[4] = jumpb[3] / (rv[0] * p.r_gas) + 0.5 * (mu2b * mur.d[1] + lam2b * lamr.d[1]);
  rvb[0] = -jumpb[3] * Tr / rv[0] + 0.5 * (mu2b * mur.d[0] + lam2b * lamr.d[0]);
  const double rho12b = -(u12b * u12 + v12b * v12 + w12b * w12) / rho12;
  cons2prim_rev(p.gamma, lv, lvb, clb);
  cons2prim_rev(p.gamma, rv, rvb, crb);
  clb[0] += 0.5 * rho12b;
  crb[0] += 0.5 * rho12b;
  clb[1] += 0.5 * u12b / rho12;
  crb[1] += 0.5 * u12b / rho12;
  clb[2] += 0.5 * v12b / rho12;
  crb[2] += 0.5 * v12b / rho12;
  clb[3] += 0.5 * w12b / rho12;
  crb[3] += 0.5 * w12b / rho12;
}

// thread per owned face, over its points: the flux leaves R_c and enters
// R_nb, so its adjoint is fb = w_q area (lam_nb - lam_c), -w_q area lam_c
// on a boundary face, whose ghost side takes the cell's own gradient
// (CALCULATE_BOUNDED_VISCOUS) and its ghost state from boundary_ghost; the
// ghost's Jacobians in the face state and (second face group) in the
// free-stream state are dual-number columns.  The face-point gradient is,
// with fg == null (MUSCL), the mean of the two cells' gradients (slot 0 of
// ulv, written by k_adj_fwd) and, with fg (WENO: the averaged face-point
// gradients of k_visc_facegrad, [nown][QS][12]), fg at the point.  Adds to
// adjF and pown (written before by the face kernels, one thread per
// element) and writes gadj[c][f][q] (the adjoint of cell c's own gradient
// at its point q of face f: half the mean's on an interior face, all of it
// on a boundary face, where both sides are the cell's).
__global__ void __launch_bounds__(128, 4) k_adj_visc(Problem p, int64_t nplain, const double* __restrict__ U,
                                                     const double* __restrict__ lam, double* __restrict__ adjF,
                                                     double* __restrict__ pown, double* __restrict__ gadj,
                                                     const double* __restrict__ fg) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.nown) return;
  const FaceRef F = face_ref(p, i);
  const bool bnd = F.nb < 0;
  const int64_t c = F.c, nb = F.nb;
  const int f = F.f, nf = F.nf, QS = F.QS;
  const int code = bnd ? p.bc[c * MF + f] : 0;
  double r[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) r[j] = p.rot[(c * MF + f) * 4 + j];
  const double* dul = (const double*)p.dul;
  const double damp = code >= 1 && code <= 4 ? 0.0 : p.lamx;
  double pb[NV] = {0, 0, 0, 0, 0};  // adjoint of the free-stream state, summed over the points
  for (int q = 0; q < F.nq; ++q) {
    const double ws = face_weight(p, p.ftype[c * MF + f], q) * p.area[c * MF + f];
    const int qq = bnd ? 0 : p.qperm[(c * MF + f) * QS + q];
    const int64_t sl = (c * MF + f) * QS + q, sr = bnd ? sl : (nb * MF + nf) * QS + qq;
    double L[NV], R[NV], fb[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      L[v] = U[c * NV + v] + dul[sl * NV + v];
      fb[v] = bnd ? -ws * lam[c * NV + v] : ws * (lam[nb * NV + v] - lam[c * NV + v]);
    }
    if (!bnd) {
#pragma unroll
      for (int v = 0; v < NV; ++v) R[v] = U[nb * NV + v] + dul[sr * NV + v];
    } else {
      boundary_ghost(p, code, r, L, R);
    }
    double gm[12];
    if (fg) {
#pragma unroll
      for (int j = 0; j < 12; ++j) gm[j] = fg[(i * QS + q) * 12 + j];
    } else {  // each cell's gradient is the same at all its face points: slot 0
      const double* g0 = p.ulv + c * (int64_t)MF * QS * 12;
      const double* g1 = bnd ? g0 : p.ulv + nb * (int64_t)MF * QS * 12;
#pragma unroll
      for (int j = 0; j < 12; ++j) gm[j] = (g0[j] + g1[j]) / 2.0;
    }
    double Lb[NV], Rb[NV], gb[12];
    viscous_flux_rev(p, r, p.dih[c * MF + f], L, R, gm, damp, fb, Lb, Rb, gb);
    if (!bnd) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        adjF[sl * NV + v] += Lb[v];
        adjF[sr * NV + v] += Rb[v];
      }
#pragma unroll
      for (int j = 0; j < 12; ++j) {
        gadj[sl * 12 + j] = gb[j];
        gadj[sr * 12 + j] = gb[j];
      }
      continue;
    }
#pragma unroll
    for (int j = 0; j < 12; ++j) gadj[sl * 12 + j] = 2.0 * gb[j];
    // ghost R = G(L, bcs), one dual-number column per input (the face state,
    // then for the second face group the free-stream state)
    const int ncol = i < nplain ? NV : 2 * NV;
#pragma unroll 1
    for (int k = 0; k < ncol; ++k) {
      Dual<1> Ld[NV], bd[NV], Rd[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        Ld[v] = Dual<1>(L[v]);
        Ld[v].d[0] = k == v ? 1.0 : 0.0;
        bd[v] = Dual<1>(p.bc_state[v]);
        bd[v].d[0] = k == NV + v ? 1.0 : 0.0;
      }
      boundary_ghost(p, code, r, Ld, bd, Rd);
      double s = 0.0;
#pragma unroll
      for (int v = 0; v < NV; ++v) s += Rb[v] * Rd[v].d[0];
      if (k < NV) adjF[sl * NV + k] += Lb[k] + s;
      else pb[k - NV] += s;
    }
  }
  if (bnd && i >= nplain)
#pragma unroll
    for (int v = 0; v < NV; ++v) pown[(i - nplain) * NV + v] += pb[v];
}

// deterministic column sums of a [m][5] array in two passes: k_colsum5_part
// sums fixed row ranges per block, k_colsum5 then sums the block partials
__global__ void __launch_bounds__(256) k_colsum5_part(const double* __restrict__ a, int64_t m, int64_t rows,
                                                      double* __restrict__ part) {
  const int64_t r0 = (int64_t)blockIdx.x * rows, r1 = r0 + rows < m ? r0 + rows : m;
  __shared__ double sh[NV][256];
  double s[NV] = {0, 0, 0, 0, 0};
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x)
#pragma unroll
    for (int k = 0; k < NV; ++k) s[k] += a[r * NV + k];
#pragma unroll
  for (int k = 0; k < NV; ++k) sh[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < NV; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < NV) part[blockIdx.x * NV + threadIdx.x] = sh[threadIdx.x][0];
}

// ------------------------------------------------------------ MUSCL reverse
// Forward quantities of the MUSCL reconstruction of cell c (k_muscl,
// IORDER 1), kept for the reverse sweep.
struct MusclFwd {
  double u0[NV];
  double g[3][NV];
  double lo[NV], hi[NV];   // bounds relative to u0
  int amin[NV], amax[NV];  // slot of the bound: 0 the cell, 1 + IMAX + f face neighbour f
  double slope[NV];
  int fstar[NV];           // face of the limiting value, -1 if none
  double epsi2;
  bool first;              // CHECKSOLX: first order
  int fmask;               // bit f: face neighbour f has a slot of its own (not in the stencil)
};

// The records of all cells, field-major so that a warp's loads and stores of
// one field are contiguous: double field j of cell c at d[j * n + c], byte
// field j at b[j * n + c].
constexpr int FWD_D = 4 * NV + 3 * NV + 1;  // u0, g, lo, hi, slope, epsi2
constexpr int FWD_B = 3 * NV + 2;           // amin, amax, fstar, first, fmask
struct FwdStore {
  double* d;
  int8_t* b;
  int64_t n;
  __device__ void put(int64_t c, const MusclFwd& m) const {
    int j = 0;
#pragma unroll
    for (int v = 0; v < NV; ++v) d[(j++) * n + c] = m.u0[v];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int v = 0; v < NV; ++v) d[(j++) * n + c] = m.g[k][v];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      d[(j++) * n + c] = m.lo[v];
      d[(j++) * n + c] = m.hi[v];
      d[(j++) * n + c] = m.slope[v];
    }
    d[j * n + c] = m.epsi2;
    j = 0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      b[(j++) * n + c] = (int8_t)m.amin[v];
      b[(j++) * n + c] = (int8_t)m.amax[v];
      b[(j++) * n + c] = (int8_t)m.fstar[v];
    }
    b[(j++) * n + c] = (int8_t)m.first;
    b[j * n + c] = (int8_t)m.fmask;
  }
  __device__ void get(int64_t c, MusclFwd& m) const {
    int j = 0;
#pragma unroll
    for (int v = 0; v < NV; ++v) m.u0[v] = d[(j++) * n + c];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int v = 0; v < NV; ++v) m.g[k][v] = d[(j++) * n + c];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      m.lo[v] = d[(j++) * n + c];
      m.hi[v] = d[(j++) * n + c];
      m.slope[v] = d[(j++) * n + c];
    }
    m.epsi2 = d[j * n + c];
    j = 0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      m.amin[v] = b[(j++) * n + c];
      m.amax[v] = b[(j++) * n + c];
      m.fstar[v] = b[(j++) * n + c];
    }
    m.first = b[(j++) * n + c] != 0;
    m.fmask = b[j * n + c];
  }
};

__device__ __forceinline__ void muscl_basis(const Problem& p, int64_t c, int f, double* b) {
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const double* qp = (const double*)p.qpts + (c >> 5) * (int64_t)MF * QS * 3 * 32 + (c & 31);
  const double* bm = (const double*)p.bmean + (c >> 5) * 3 * 32 + (c & 31);
  b[0] = qp[(f * QS * 3 + 0) * 32] - bm[0];
  b[1] = qp[(f * QS * 3 + 1) * 32] - bm[32];
  b[2] = qp[(f * QS * 3 + 2) * 32] - bm[64];
}

__device__ __forceinline__ double muscl_dd(const MusclFwd& m, const double* b, int v) {
  const double res = b[0] * m.g[0][v] + b[1] * m.g[1][v] + b[2] * m.g[2][v];
  return (m.u0[v] + res) - m.u0[v];
}

__device__ void muscl_forward(const Problem& p, const double* __restrict__ U, int64_t c, MusclFwd& m) {
  const int IM = p.imax, W = IM + 1, nf = p.nfaces[c];
#pragma unroll
  for (int v = 0; v < NV; ++v) m.u0[v] = U[c * NV + v];
  const int64_t grp = c >> 5;
  const int lane = (int)(c & 31);
  const int32_t* st = p.sten + grp * (int64_t)p.admis_max * W * 32 + lane;
  const double* M = (const double*)p.invmat + (grp * p.tstride + p.soff[0]) * 32 + lane;
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int v = 0; v < NV; ++v) m.g[d][v] = 0.0;
  for (int k = 0; k < IM; ++k) {
    const int64_t y = st[(k + 1) * 32];
    const double m0 = M[(k * 3 + 0) * 32], m1 = M[(k * 3 + 1) * 32], m2 = M[(k * 3 + 2) * 32];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double du = U[y * NV + v] - m.u0[v];
      m.g[0][v] += m0 * du;
      m.g[1][v] += m1 * du;
      m.g[2][v] += m2 * du;
    }
  }
  double mn[NV], mx[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    mn[v] = mx[v] = m.u0[v];
    m.amin[v] = m.amax[v] = 0;
  }
  for (int f = 0; f < nf; ++f) {
    const int64_t nb = p.neigh[c * MF + f];
    if (nb < 0) continue;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double un = U[nb * NV + v];
      if (un < mn[v]) {
        mn[v] = un;
        m.amin[v] = 1 + IM + f;
      }
      if (un > mx[v]) {
        mx[v] = un;
        m.amax[v] = 1 + IM + f;
      }
    }
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    m.lo[v] = mn[v] - m.u0[v];
    m.hi[v] = mx[v] - m.u0[v];
  }
  const double e3 = p.kappa_ven * p.minedge[c];
  m.epsi2 = e3 * e3 * e3;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    m.slope[v] = TOLBIG;
    m.fstar[v] = -1;
  }
  for (int f = 0; f < nf; ++f) {
    double b[3];
    muscl_basis(p, c, f, b);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double ps = venkat(muscl_dd(m, b, v), m.lo[v], m.hi[v], m.epsi2);
      if (ps < m.slope[v]) {
        m.slope[v] = ps;
        m.fstar[v] = f;
      }
    }
  }
  double pm[NV];
  cons2prim(p.gamma, m.u0, pm);
  m.first = false;
  for (int f = 0; f < nf; ++f) {
    double b[3], uf[NV];
    muscl_basis(p, c, f, b);
#pragma unroll
    for (int v = 0; v < NV; ++v) uf[v] = m.u0[v] + muscl_dd(m, b, v) * m.slope[v];
    m.first = m.first || jump_bad(p.gamma, pm, uf, 0.95);
  }
}

// Navier-Stokes: the cell's gradient of (T, u, v, w) ([T, u, v, w][x, y,
// z]) from the viscous least squares on stencil 1 and the frame (AINVJT),
// in the operations and order of k_muscl's viscous part (gradients.f90:
// 502-706, SOLUTIONTRIAV2), which writes the same 12 values to every face
// slot of ulv.
__device__ __forceinline__ void visc_cell_gradient(const Problem& p, const double* __restrict__ U, int64_t c,
                                                   double* gr) {
  const int IM = p.imax, W = IM + 1;
  double u0[NV], pm[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u0[v] = U[c * NV + v];
  cons2prim(p.gamma, u0, pm);
  const double t0 = pm[4] / (pm[0] * p.r_gas);
  const int64_t grp = c >> 5;
  const int lane = (int)(c & 31);
  const int32_t* st = p.sten + grp * (int64_t)p.admis_max * W * 32 + lane;
  const double* M = (const double*)p.invmat + (grp * p.tstride + p.soff[0]) * 32 + lane;
  double gvv[3][4] = {};
  for (int k = 0; k < IM; ++k) {
    const int64_t y = st[(k + 1) * 32];
    double uy[NV], py[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uy[v] = U[y * NV + v];
    const double m0 = M[(k * 3 + 0) * 32], m1 = M[(k * 3 + 1) * 32], m2 = M[(k * 3 + 2) * 32];
    cons2prim(p.gamma, uy, py);
    const double ds[4] = {py[4] / (py[0] * p.r_gas) - t0, py[1] - pm[1], py[2] - pm[2], py[3] - pm[3]};
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      gvv[0][v] += m0 * ds[v];
      gvv[1][v] += m1 * ds[v];
      gvv[2][v] += m2 * ds[v];
    }
  }
  const double* J = p.jinv + c * 9;
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      gr[v * 3 + k] = J[0 * 3 + k] * gvv[0][v] + J[1 * 3 + k] * gvv[1][v] + J[2 * 3 + k] * gvv[2][v];
}

// The reconstruction of every cell with its intermediates kept for the
// reverse sweep: face values (minus the mean) to dul exactly as k_muscl
// writes them, the MusclFwd record to fwd[c]; for Navier-Stokes the cell's
// viscous gradient to face slot 0 of ulv (the slot that k_adj_visc reads).
// A face neighbour that is also a cell of the stencil shares the stencil
// cell's slot: the bound slots amin/amax are remapped to it, and fmask keeps
// the faces whose neighbour has a slot of its own (the reverse map in
// adj_setup makes the same choice).
__global__ void __launch_bounds__(128) k_adj_fwd(Problem p, const double* __restrict__ U, FwdStore fwd) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  MusclFwd m;
  muscl_forward(p, U, c, m);
  const int IM = p.imax, nf = p.nfaces[c];
  double* out = (double*)p.dul + c * (int64_t)MF * NV;
  for (int f = 0; f < nf; ++f) {
    double b[3];
    muscl_basis(p, c, f, b);
#pragma unroll
    for (int v = 0; v < NV; ++v) out[f * NV + v] = m.first ? 0.0 : muscl_dd(m, b, v) * m.slope[v];
  }
  const int32_t* st = p.sten + (c >> 5) * (int64_t)p.admis_max * (IM + 1) * 32 + (c & 31);
  int slot_of[MF];
  m.fmask = 0;
  for (int f = 0; f < MF; ++f) {
    const int64_t nb = f < nf ? p.neigh[c * MF + f] : -1;
    slot_of[f] = 1 + IM + f;
    if (nb < 0) continue;
    for (int k = 0; k < IM; ++k)
      if (st[(k + 1) * 32] == nb) {
        slot_of[f] = 1 + k;
        break;
      }
    if (slot_of[f] == 1 + IM + f) m.fmask |= 1 << f;
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    if (m.amin[v] > IM) m.amin[v] = slot_of[m.amin[v] - 1 - IM];
    if (m.amax[v] > IM) m.amax[v] = slot_of[m.amax[v] - 1 - IM];
  }
  fwd.put(c, m);
  if (p.governing == 1) {
    double gr[12];
    visc_cell_gradient(p, U, c, gr);
    const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
    double* o = p.ulv + c * (int64_t)MF * QS * 12;
#pragma unroll
    for (int j = 0; j < 12; ++j) o[j] = gr[j];
  }
}

// Contributions to mu, slot-major: contrib[(slot * n + c) * NV + v], slot 0
// the cell, 1..IMAX its stencil cells, 1 + IMAX + f its face neighbour f
// (only the faces of fmask).  Each slot that the reverse map reads is
// written exactly once.  Face values u_f = u0 + dd_f * slope (or u0 when
// CHECKSOLX chose first order).
// gadj (Navier-Stokes, else null): the adjoint of each cell's gradient of
// (T, u, v, w) through each of its faces (k_adj_visc); reversed through the
// frame (AINVJT), the viscous least squares on stencil 1 and (T, u, v, w)(U)
// into the same slots as the MUSCL reconstruction's.
__global__ void __launch_bounds__(128) k_adj_muscl(Problem p, FwdStore fwd, const double* __restrict__ adjF,
                                                   double* __restrict__ contrib, const double* __restrict__ U,
                                                   const double* __restrict__ gadj) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n = p.n;
  if (c >= n) return;
  const int IM = p.imax, nf = p.nfaces[c];
  MusclFwd m;
  fwd.get(c, m);
  double self[NV] = {0, 0, 0, 0, 0};
  for (int f = 0; f < nf; ++f)
#pragma unroll
    for (int v = 0; v < NV; ++v) self[v] += adjF[(c * MF + f) * NV + v];
  // viscous gradients: gr[a][k] = sum_d J[d][k] gvv[d][a], gvv[d][a] =
  // sum_k M_dk (s_a(U_k) - s_a(U_c)); vslot(k, v) adds to stencil slot 1 + k
  const int64_t vgrp = c >> 5;
  const int vlane = (int)(c & 31);
  const double* Mv = (const double*)p.invmat + (vgrp * p.tstride + p.soff[0]) * 32 + vlane;
  const int32_t* stv = p.sten + vgrp * (int64_t)p.admis_max * (IM + 1) * 32 + vlane;
  double gvvb[3][4] = {}, sc[4] = {0, 0, 0, 0};
  if (gadj) {
    double gb[12] = {};
    for (int f = 0; f < nf; ++f)
#pragma unroll
      for (int j = 0; j < 12; ++j) gb[j] += gadj[(c * MF + f) * 12 + j];
    const double* Jc = p.jinv + c * 9;
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int a = 0; a < 4; ++a)
        gvvb[d][a] = Jc[d * 3 + 0] * gb[a * 3 + 0] + Jc[d * 3 + 1] * gb[a * 3 + 1] + Jc[d * 3 + 2] * gb[a * 3 + 2];
  }
  // the viscous contribution to stencil slot 1 + k (member state adjoint)
  auto vslot = [&](int k, double (&out)[NV]) {
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = 0.0;
    if (!gadj) return;
    const double m0 = Mv[(k * 3 + 0) * 32], m1 = Mv[(k * 3 + 1) * 32], m2 = Mv[(k * 3 + 2) * 32];
    double sb[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      sb[a] = m0 * gvvb[0][a] + m1 * gvvb[1][a] + m2 * gvvb[2][a];
      sc[a] -= sb[a];
    }
    const int64_t y = stv[(k + 1) * 32];
    visc_vars_rev(p, U + y * NV, sb, out);
  };
  // the cell's own viscous term (after every vslot)
  auto vself = [&](double (&out)[NV]) {
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = 0.0;
    if (!gadj) return;
    visc_vars_rev(p, U + c * NV, sc, out);
  };
  auto put = [&](int slot, int v, double x) { contrib[((int64_t)slot * n + c) * NV + v] = x; };
  if (m.first) {
    for (int k = 0; k < IM; ++k) {
      double vk[NV];
      vslot(k, vk);
#pragma unroll
      for (int v = 0; v < NV; ++v) put(1 + k, v, vk[v]);
    }
    double vs[NV];
    vself(vs);
#pragma unroll
    for (int v = 0; v < NV; ++v) put(0, v, self[v] + vs[v]);
    for (int f = 0; f < MF; ++f)
      if (m.fmask >> f & 1)
#pragma unroll
        for (int v = 0; v < NV; ++v) put(1 + IM + f, v, 0.0);
    return;
  }
  // reverse of u_f = u0 + dd_f * slope, slope = psi_{f*}, dd_f = b_f . g
  double gbar[3][NV] = {};
  double lob[NV] = {0, 0, 0, 0, 0}, hib[NV] = {0, 0, 0, 0, 0};
  double sbar[NV] = {0, 0, 0, 0, 0};
  for (int f = 0; f < nf; ++f) {
    double b[3];
    muscl_basis(p, c, f, b);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double ub = adjF[(c * MF + f) * NV + v];
      sbar[v] += ub * muscl_dd(m, b, v);
      const double ddb = ub * m.slope[v];
#pragma unroll
      for (int d = 0; d < 3; ++d) gbar[d][v] += ddb * b[d];
    }
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const int fs = m.fstar[v];
    if (fs < 0) continue;
    double b[3];
    muscl_basis(p, c, fs, b);
    Dual<3> dd(muscl_dd(m, b, v)), lo(m.lo[v]), hi(m.hi[v]);
    dd.d[0] = 1.0;
    lo.d[1] = 1.0;
    hi.d[2] = 1.0;
    const Dual<3> ps = venkat(dd, lo, hi, m.epsi2);
    const double ddb = sbar[v] * ps.d[0];
#pragma unroll
    for (int d = 0; d < 3; ++d) gbar[d][v] += ddb * b[d];
    lob[v] += sbar[v] * ps.d[1];
    hib[v] += sbar[v] * ps.d[2];
  }
  // lo = min(...) - u0, hi = max(...) - u0: the bound cells get lob/hib
  auto bounds = [&](int slot, int v) {
    return (m.amin[v] == slot ? lob[v] : 0.0) + (m.amax[v] == slot ? hib[v] : 0.0);
  };
  // g = sum_k M_k (u_k - u0)
  const int64_t grp = c >> 5;
  const int lane = (int)(c & 31);
  const double* M = (const double*)p.invmat + (grp * p.tstride + p.soff[0]) * 32 + lane;
  for (int k = 0; k < IM; ++k) {
    const double m0 = M[(k * 3 + 0) * 32], m1 = M[(k * 3 + 1) * 32], m2 = M[(k * 3 + 2) * 32];
    double vk[NV];
    vslot(k, vk);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double ck = m0 * gbar[0][v] + m1 * gbar[1][v] + m2 * gbar[2][v];
      put(1 + k, v, ck + bounds(1 + k, v) + vk[v]);
      self[v] -= ck;
    }
  }
  for (int f = 0; f < MF; ++f)
    if (m.fmask >> f & 1)
#pragma unroll
      for (int v = 0; v < NV; ++v) put(1 + IM + f, v, bounds(1 + IM + f, v));
  double vs[NV];
  vself(vs);
#pragma unroll
  for (int v = 0; v < NV; ++v) put(0, v, self[v] - (lob[v] + hib[v]) + bounds(0, v) + vs[v]);
}

// mu[j] = sum over the slots that point at cell j (reverse map, fixed order)
__global__ void k_adj_gather(int64_t n, const int64_t* __restrict__ rptr, const int64_t* __restrict__ rsrc,
                             const double* __restrict__ contrib, double* __restrict__ mu) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double s[NV] = {0, 0, 0, 0, 0};
  for (int64_t e = rptr[j]; e < rptr[j + 1]; ++e) {
    const double* x = contrib + rsrc[e] * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] += x[v];
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) mu[j * NV + v] = s[v];
}

// ------------------------------------------------------------ tangent
struct Dp5 {
  double v[NV];
};

// tangent of the face values: tdul[c][f] = d(u_f - u0) along dU; tgr
// (Navier-Stokes, else null): the tangent of the cell's gradient of
// (T, u, v, w), [n][12] in the layout of ulv.  With `base` the value parts,
// which are the reconstruction itself, go out as k_muscl writes it (in place
// of a k_muscl launch): the face values to dul and, with tgr, the cell's
// viscous gradient to face slot 0 of ulv (the slot that k_jvp_face reads).
__global__ void __launch_bounds__(128) k_jvp_muscl(Problem p, const double* __restrict__ U,
                                                   const double* __restrict__ dU, double* __restrict__ tdul,
                                                   double* __restrict__ tgr, bool base) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  using D = Dual<1>;
  const int IM = p.imax, W = IM + 1, nf = p.nfaces[c];
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  D u0[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    u0[v] = D(U[c * NV + v]);
    u0[v].d[0] = dU[c * NV + v];
  }
  const int64_t grp = c >> 5;
  const int lane = (int)(c & 31);
  const int32_t* st = p.sten + grp * (int64_t)p.admis_max * W * 32 + lane;
  const double* M = (const double*)p.invmat + (grp * p.tstride + p.soff[0]) * 32 + lane;
  D g[3][NV], gvv[3][4];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
#pragma unroll
    for (int v = 0; v < NV; ++v) g[d][v] = D(0.0);
#pragma unroll
    for (int a = 0; a < 4; ++a) gvv[d][a] = D(0.0);
  }
  D s0[4];
  if (tgr) {
    D pm0[NV];
    cons2prim(p.gamma, u0, pm0);
    s0[0] = pm0[4] / (pm0[0] * p.r_gas);
    s0[1] = pm0[1];
    s0[2] = pm0[2];
    s0[3] = pm0[3];
  }
  for (int k = 0; k < IM; ++k) {
    const int64_t y = st[(k + 1) * 32];
    const double m0 = M[(k * 3 + 0) * 32], m1 = M[(k * 3 + 1) * 32], m2 = M[(k * 3 + 2) * 32];
    D uy[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      uy[v] = D(U[y * NV + v]);
      uy[v].d[0] = dU[y * NV + v];
      const D du = uy[v] - u0[v];
      g[0][v] = g[0][v] + m0 * du;
      g[1][v] = g[1][v] + m1 * du;
      g[2][v] = g[2][v] + m2 * du;
    }
    if (tgr) {
      D py[NV];
      cons2prim(p.gamma, uy, py);
      const D ds[4] = {py[4] / (py[0] * p.r_gas) - s0[0], py[1] - s0[1], py[2] - s0[2], py[3] - s0[3]};
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        gvv[0][a] = gvv[0][a] + m0 * ds[a];
        gvv[1][a] = gvv[1][a] + m1 * ds[a];
        gvv[2][a] = gvv[2][a] + m2 * ds[a];
      }
    }
  }
  if (tgr) {
    const double* Jc = p.jinv + c * 9;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int kk = 0; kk < 3; ++kk) {
        const D t = Jc[0 * 3 + kk] * gvv[0][a] + Jc[1 * 3 + kk] * gvv[1][a] + Jc[2 * 3 + kk] * gvv[2][a];
        tgr[c * 12 + a * 3 + kk] = t.d[0];
        if (base) p.ulv[c * (int64_t)MF * QS * 12 + a * 3 + kk] = t.v;
      }
  }
  D mn[NV], mx[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) mn[v] = mx[v] = u0[v];
  for (int f = 0; f < nf; ++f) {
    const int64_t nb = p.neigh[c * MF + f];
    if (nb < 0) continue;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      D un(U[nb * NV + v]);
      un.d[0] = dU[nb * NV + v];
      if (un.v < mn[v].v) mn[v] = un;
      if (un.v > mx[v].v) mx[v] = un;
    }
  }
  const double e3 = p.kappa_ven * p.minedge[c];
  const double epsi2 = e3 * e3 * e3;
  const double* qp = (const double*)p.qpts + grp * (int64_t)MF * QS * 3 * 32 + lane;
  const double* bm = (const double*)p.bmean + grp * 3 * 32 + lane;
  auto face_d = [&](int f, int v) -> D {
    const double b0 = qp[(f * QS * 3 + 0) * 32] - bm[0], b1 = qp[(f * QS * 3 + 1) * 32] - bm[32],
                 b2 = qp[(f * QS * 3 + 2) * 32] - bm[64];
    const D res = b0 * g[0][v] + b1 * g[1][v] + b2 * g[2][v];
    return (u0[v] + res) - u0[v];
  };
  D slope[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) slope[v] = D(TOLBIG);
  for (int f = 0; f < nf; ++f)
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const D ps = venkat(face_d(f, v), mn[v] - u0[v], mx[v] - u0[v], epsi2);
      if (ps.v < slope[v].v) slope[v] = ps;
    }
  double pm[NV], u0v[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u0v[v] = u0[v].v;
  cons2prim(p.gamma, u0v, pm);
  bool first = false;
  for (int f = 0; f < nf; ++f) {
    double uf[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uf[v] = u0v[v] + face_d(f, v).v * slope[v].v;
    first = first || jump_bad(p.gamma, pm, uf, 0.95);
  }
  double* dul = (double*)p.dul;
  for (int f = 0; f < nf; ++f)
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const D x = face_d(f, v) * slope[v];
      tdul[(c * MF + f) * NV + v] = first ? 0.0 : x.d[0];
      if (base) dul[(c * MF + f) * NV + v] = first ? 0.0 : x.v;
    }
}

// tangent of the face fluxes (owner and negated neighbour copy); with tgr
// (Navier-Stokes) the viscous flux's tangent subtracted, as the residual
// subtracts the viscous fluxes
__global__ void __launch_bounds__(128) k_jvp_face(Problem p, const double* __restrict__ U,
                                                  const double* __restrict__ dU, const double* __restrict__ tdul,
                                                  Dp5 dp, double* __restrict__ tflux, const double* __restrict__ tgr,
                                                  const double* __restrict__ tfg) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.nown) return;
  using D = Dual<1>;
  const FaceRef F = face_ref(p, i);
  const int64_t c = F.c, nb = F.nb;
  const int f = F.f, nf = F.nf, QS = F.QS;
  double r[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) r[k] = p.rot[(c * MF + f) * 4 + k];
  const double* dul = (const double*)p.dul;
  double tf[NV] = {0, 0, 0, 0, 0};
  for (int q = 0; q < F.nq; ++q) {
    const double ws = face_weight(p, p.ftype[c * MF + f], q) * p.area[c * MF + f];
    D L[NV], R[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      L[v] = D(U[c * NV + v] + dul[((c * MF + f) * QS + q) * NV + v]);
      L[v].d[0] = dU[c * NV + v] + tdul[((c * MF + f) * QS + q) * NV + v];
    }
    if (nb >= 0) {
      const int qq = p.qperm[(c * MF + f) * QS + q];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        R[v] = D(U[nb * NV + v] + dul[((nb * MF + nf) * QS + qq) * NV + v]);
        R[v].d[0] = dU[nb * NV + v] + tdul[((nb * MF + nf) * QS + qq) * NV + v];
      }
    } else {
      D bcs[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        bcs[v] = D(p.bc_state[v]);
        bcs[v].d[0] = dp.v[v];
      }
      boundary_ghost(p, (int)p.bc[c * MF + f], r, L, bcs, R);
    }
    D a[NV], b[NV], h[NV], fl[NV];
    rot_f(r, R, b);
    rot_f(r, L, a);
    hllc(p.gamma, a, b, h);
    rot_b(r, h, fl);
#pragma unroll
    for (int v = 0; v < NV; ++v) tf[v] = tf[v] + fl[v].d[0] * ws;
    if (tgr) {
      const double* g0 = p.ulv + c * (int64_t)MF * QS * 12;  // slot 0: see k_jvp_muscl
      const double* g1 = nb >= 0 ? p.ulv + nb * (int64_t)MF * QS * 12 : g0;
      const double* t0 = tgr + c * 12;
      const double* t1 = nb >= 0 ? tgr + nb * 12 : t0;
      D gl[12], gr[12], fv[NV];
#pragma unroll
      for (int j = 0; j < 12; ++j) {
        gl[j] = D(g0[j]);
        gl[j].d[0] = t0[j];
        gr[j] = D(g1[j]);
        gr[j].d[0] = t1[j];
      }
      const int code = nb >= 0 ? 0 : p.bc[c * MF + f];
      viscous_flux(p, r, p.dih[c * MF + f], L, R, gl, gr, fv, code >= 1 && code <= 4 ? 0.0 : p.lamx);
#pragma unroll
      for (int v = 0; v < NV; ++v) tf[v] = tf[v] - fv[v].d[0] * ws;
    } else if (tfg) {  // WENO: both sides take the averaged face-point gradient and its tangent
      D g[12], fv[NV];
#pragma unroll
      for (int j = 0; j < 12; ++j) {
        g[j] = D(p.fgrad[(i * QS + q) * 12 + j]);
        g[j].d[0] = tfg[(i * QS + q) * 12 + j];
      }
      const int code = nb >= 0 ? 0 : p.bc[c * MF + f];
      viscous_flux(p, r, p.dih[c * MF + f], L, R, g, g, fv, code >= 1 && code <= 4 ? 0.0 : p.lamx);
#pragma unroll
      for (int v = 0; v < NV; ++v) tf[v] = tf[v] - fv[v].d[0] * ws;
    }
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) tflux[(c * MF + f) * NV + v] = tf[v];
  if (nb >= 0)
#pragma unroll
    for (int v = 0; v < NV; ++v) tflux[(nb * MF + nf) * NV + v] = -tf[v];
}

// tangent of the residual: face sums in face order
__global__ void k_jvp_sum(Problem p, const double* __restrict__ tflux, double* __restrict__ dR) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  double s[NV] = {0, 0, 0, 0, 0};
  for (int f = 0; f < p.nfaces[c]; ++f)
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = s[v] + tflux[(c * MF + f) * NV + v];
#pragma unroll
  for (int v = 0; v < NV; ++v) dR[c * NV + v] = s[v];
}

// ------------------------------------------------------------ wall force
// per cell: sum over its wall faces of (sum_q w_q p_q - PRES) * area * n_x
// (the face points of [n][F][QS] face values: one for MUSCL IORDER 1, the
// quadrature points for WENO/CWENO); with dU != null the tangent of the
// same sum, with adjF != null the adjoint of the face values (jbar * area *
// n_x * w_q * dp/du), else 0.
__global__ void k_force_cell(Problem p, const double* __restrict__ U, const double* __restrict__ dU,
                             const double* __restrict__ tdul, double* __restrict__ fcell, double* __restrict__ adjF,
                             double jbar) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  const int nf = p.nfaces[c];
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const double* dul = (const double*)p.dul;
  double sum = 0.0;
  for (int f = 0; f < nf; ++f) {
    const bool wall = p.neigh[c * MF + f] < 0 && p.bc[c * MF + f] == 4;
    const int ft = p.ftype[c * MF + f], nq = face_nq(p, ft);
    if (adjF)
      for (int q = 0; q < QS; ++q)
#pragma unroll
        for (int v = 0; v < NV; ++v) adjF[((c * MF + f) * QS + q) * NV + v] = 0.0;
    if (!wall) continue;
    const double nx = p.rot[(c * MF + f) * 4 + 0] * p.rot[(c * MF + f) * 4 + 3];
    const double area = p.area[c * MF + f];
    double ssp = 0.0;
    for (int q = 0; q < nq; ++q) {
      const int64_t s = (c * MF + f) * QS + q;
      const double w = face_weight(p, ft, q);
      Dual<NV> u[NV], pr[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        u[v] = Dual<NV>(U[c * NV + v] + dul[s * NV + v]);
        u[v].d[v] = 1.0;
      }
      cons2prim(p.gamma, u, pr);
      if (dU) {
        double t = 0.0;
#pragma unroll
        for (int v = 0; v < NV; ++v) t += pr[4].d[v] * (dU[c * NV + v] + tdul[s * NV + v]);
        sum += w * t * area * nx;
      } else {
        ssp = ssp + (pr[4].v * w);
      }
      if (adjF)
#pragma unroll
        for (int v = 0; v < NV; ++v) adjF[s * NV + v] = jbar * area * nx * w * pr[4].d[v];
    }
    if (!dU) sum += (ssp - p.pres) * area * nx;
  }
  fcell[c] = sum;
}

unsigned blocks_for(int64_t m, int t) { return (unsigned)((m + t - 1) / t); }

}  // namespace

// ====================================================================== host
namespace ucg_host {

void adjoint_release(ucg_engine* e) {
  ucg_engine::DevBuf* all[] = {&e->adj_face,   &e->adj_contrib, &e->adj_rptr,  &e->adj_rsrc,     &e->adj_lam,
                               &e->adj_mu,     &e->adj_pface,   &e->adj_tflux, &e->adj_tdul,     &e->adj_tU,
                               &e->adj_fcell,  &e->adj_traj,    &e->adj_bar,   &e->adj_tmp,      &e->adj_fwd,
                               &e->adjw_face,  &e->adjw_gbar,   &e->adjw_scr,  &e->adjw_self,    &e->adjw_contrib,
                               &e->adjw_rptr,  &e->adjw_rsrc,   &e->adjw_lam,     &e->adjw_mu,
                               &e->adjw_pface, &e->adjw_tmp,    &e->adj_gadj,  &e->adj_tgr,
                               &e->adjw_gpt,   &e->adjw_gvb,    &e->adjw_tfg};
  for (auto* b : all) {
    if (b->p) e->bytes -= (int64_t)b->bytes;
    release(*b);
  }
  e->adj_ready = false;
  e->adjw_ready = false;
}

}  // namespace ucg_host

namespace {

// reverse map and buffers (once per geometry/tables)
int adj_setup(ucg_engine* e) {
  int rc = adj_check(e);
  if (rc) return rc;
  if (e->adj_ready) return UCG_OK;
  const int64_t n = e->n;
  const int IM = e->cfg.imax, W = IM + 1;
  const int slots = 1 + IM + MF;
  if ((int64_t)e->sten1_h.size() != n * W || (int64_t)e->neigh_h.size() != n * MF)
    return fail(e, UCG_ESTATE, "stencils and neighbours of every cell are needed");
  // reverse map: for each target cell, the (cell, slot) pairs pointing at it,
  // ordered by source cell then slot
  std::vector<int64_t> cnt(n + 1, 0);
  // a face neighbour that is also in the stencil shares the stencil slot
  // (k_adj_fwd makes the same choice)
  auto target = [&](int64_t i, int s) -> int64_t {
    if (s == 0) return i;
    if (s <= IM) return e->sten1_h[(size_t)i * W + s];
    const int64_t nb = e->neigh_h[(size_t)i * MF + (s - 1 - IM)];
    for (int k = 1; k <= IM; ++k)
      if (e->sten1_h[(size_t)i * W + k] == nb) return -1;
    return nb;
  };
  for (int64_t i = 0; i < n; ++i)
    for (int s = 0; s < slots; ++s) {
      const int64_t t = target(i, s);
      if (t >= 0 && t < n) ++cnt[t + 1];
    }
  for (int64_t j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
  std::vector<int64_t> src(cnt[n]), pos(cnt.begin(), cnt.end() - 1);
  for (int64_t i = 0; i < n; ++i)
    for (int s = 0; s < slots; ++s) {
      const int64_t t = target(i, s);
      if (t >= 0 && t < n) src[pos[t]++] = s * n + i;
    }
  cudaSetDevice(e->device);
  auto get = [&](ucg_engine::DevBuf& b, size_t bytes) { return alloc(e, b, bytes); };
  rc = get(e->adj_face, (size_t)n * MF * NV * 8);
  rc = rc ? rc : get(e->adj_contrib, (size_t)n * slots * NV * 8);
  rc = rc ? rc : get(e->adj_rptr, (size_t)(n + 1) * 8);
  rc = rc ? rc : get(e->adj_rsrc, (size_t)std::max<int64_t>(1, cnt[n]) * 8);
  rc = rc ? rc : get(e->adj_lam, (size_t)n * NV * 8);
  rc = rc ? rc : get(e->adj_mu, (size_t)n * NV * 8);
  rc = rc ? rc : get(e->adj_pface, (size_t)n * MF * NV * 8);
  rc = rc ? rc : get(e->adj_tflux, (size_t)n * MF * NV * 8);
  rc = rc ? rc : get(e->adj_tdul, (size_t)n * MF * NV * 8);
  rc = rc ? rc : get(e->adj_tU, (size_t)n * NV * 8);
  rc = rc ? rc : get(e->adj_fcell, (size_t)n * 8);
  rc = rc ? rc : get(e->adj_bar, (size_t)4 * n * NV * 8 + 64 * 8);
  rc = rc ? rc : get(e->adj_tmp, (size_t)2 * n * NV * 8);
  rc = rc ? rc : get(e->adj_fwd, (size_t)n * (FWD_D * 8 + FWD_B));
  if (e->cfg.governing == 1) {  // viscous: gradient adjoints per face, gradient tangents per cell
    rc = rc ? rc : get(e->adj_gadj, (size_t)n * MF * 12 * 8);
    rc = rc ? rc : get(e->adj_tgr, (size_t)n * 12 * 8);
  }
  if (rc) return rc;
  CK(cudaMemcpyAsync(e->adj_rptr.p, cnt.data(), (n + 1) * 8, cudaMemcpyHostToDevice, e->stream));
  if (cnt[n]) CK(cudaMemcpyAsync(e->adj_rsrc.p, src.data(), cnt[n] * 8, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemsetAsync(e->adj_face.p, 0, (size_t)n * MF * NV * 8, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  e->adj_ready = true;
  return UCG_OK;
}

// scratch vectors inside adj_bar: 4 state-sized vectors and a few scalars
double* bar_vec(ucg_engine* e, int k) { return (double*)e->adj_bar.p + (size_t)k * e->n * NV; }
double* bar_scal(ucg_engine* e) { return (double*)e->adj_bar.p + (size_t)4 * e->n * NV; }

// mu = (dR/dU)^T lam, psum[0..4] = (dR/dp)^T lam, at state U (device)
FwdStore fwd_store(ucg_engine* e) {
  double* d = (double*)e->adj_fwd.p;
  return FwdStore{d, (int8_t*)(d + (size_t)FWD_D * e->n), e->n};
}

// the reconstruction of U with its intermediates (face values to dul)
int adj_forward(ucg_engine* e, const Problem& p, const double* U) {
  k_adj_fwd<<<blocks_for(e->n, 128), 128, 0, e->stream>>>(p, U, fwd_store(e));
  e->launches++;
  CK(cudaGetLastError());
  return UCG_OK;
}

int vjp_device(ucg_engine* e, const Problem& p, const double* U, const double* lam, double* mu, double* psum) {
  const bool ns = e->cfg.governing == 1;
  int rc = adj_forward(e, p, U);  // face values, records, and the viscous gradients
  if (rc) return rc;
  const int64_t n = e->n;
  const int64_t nplain = e->nown_plain, nbnd = e->nown - nplain;
  if (nplain)
    k_adj_face<<<blocks_for(nplain, 64), 64, 0, e->stream>>>(p, nplain, U, lam, (double*)e->adj_face.p);
  if (nbnd)
    k_adj_face_bnd<<<blocks_for(nbnd * 10, 128), 128, 0, e->stream>>>(p, nplain, U, lam, (double*)e->adj_face.p,
                                                                      (double*)e->adj_pface.p);
  if (ns) {
    k_adj_visc<<<blocks_for(e->nown, 128), 128, 0, e->stream>>>(
        p, nplain, U, lam, (double*)e->adj_face.p, (double*)e->adj_pface.p, (double*)e->adj_gadj.p, nullptr);
    e->launches++;
  }
  k_adj_muscl<<<blocks_for(n, 128), 128, 0, e->stream>>>(p, fwd_store(e), (const double*)e->adj_face.p,
                                                         (double*)e->adj_contrib.p, U,
                                                         ns ? (const double*)e->adj_gadj.p : nullptr);
  k_adj_gather<<<blocks_for(n, 128), 128, 0, e->stream>>>(n, (const int64_t*)e->adj_rptr.p,
                                                          (const int64_t*)e->adj_rsrc.p,
                                                          (const double*)e->adj_contrib.p, mu);
  e->launches += 2 + (nplain > 0) + (nbnd > 0);
  if (nbnd) {
    const int64_t rows = 1024, nb = (nbnd + rows - 1) / rows;
    k_colsum5_part<<<(unsigned)nb, 256, 0, e->stream>>>((const double*)e->adj_pface.p, nbnd, rows,
                                                         (double*)e->adj_tmp.p);
    k_colsum5<<<NV, 256, 0, e->stream>>>((const double*)e->adj_tmp.p, nb, psum);
    e->launches += 2;
  } else {
    CK(cudaMemsetAsync(psum, 0, NV * sizeof(double), e->stream));
  }
  CK(cudaGetLastError());
  return UCG_OK;
}

// dR = (dR/dU) dU + (dR/dp) dp at state U (device); leaves the primal face
// values of U in dul and their tangents in adj_tdul
// recon: run the forward reconstruction (k_muscl) for the face values and
// gradients, which a caller that advances the state with them needs bit for
// bit as the residual makes them; without it k_jvp_muscl writes them from
// its dual numbers' value parts (equal up to rounding).
int jvp_device(ucg_engine* e, const Problem& p, const double* U, const double* dU, const Dp5& dp, double* dR,
               bool recon = false) {
  if (recon) {
    const int rc = launch_recon(e, p, U);
    if (rc) return rc;
  }
  const int64_t n = e->n;
  double* tgr = e->cfg.governing == 1 ? (double*)e->adj_tgr.p : nullptr;
  k_jvp_muscl<<<blocks_for(n, 128), 128, 0, e->stream>>>(p, U, dU, (double*)e->adj_tdul.p, tgr, !recon);
  k_jvp_face<<<blocks_for(e->nown, 128), 128, 0, e->stream>>>(p, U, dU, (const double*)e->adj_tdul.p, dp,
                                                              (double*)e->adj_tflux.p, tgr, nullptr);
  k_jvp_sum<<<blocks_for(n, 256), 256, 0, e->stream>>>(p, (const double*)e->adj_tflux.p, dR);
  e->launches += 3;
  CK(cudaGetLastError());
  return UCG_OK;
}

// J at state U into *out (device); with dU the tangent dJ instead
// COMPUTEFORCE (io.f90:18752-19000) in full, one thread per owned face:
// on a wall face (code 4), SSP = sum_q w_q p_q - PRES and, Navier-Stokes,
// SS = -sum_q mu_q (n . tau_q) w_q from the cell's own face-point velocity
// gradients (ULEFTV: ulv for MUSCL; for WENO fgrad, which on a physical
// boundary face holds the own side's gradient) and SUTHERLAND at the face
// state; columns [6][nown]: SSP S n + SS S, and the pressure moments about
// the cell centre (cen [n][3], or none).  Face values in T (FP32 in the
// mixed form), everything after in FP64.
template <typename T>
__global__ void k_wall_loads(Problem p, const double* __restrict__ U, const double* __restrict__ cen,
                             double* __restrict__ cols) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.nown) return;
  const int32_t code = p.own[i];
  const int64_t c = code >> 3;
  const int f = code & 7;
  double r[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (p.neigh[c * MF + f] < 0 && p.bc[c * MF + f] == 4) {
    const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
    const int ft = p.ftype[c * MF + f], nq = face_nq(p, ft);
    const double* rt = p.rot + (c * MF + f) * 4;
    const double nx = rt[0] * rt[3], ny = rt[1] * rt[3], nz = rt[2];
    const double S = p.area[c * MF + f];
    const T* dul = (const T*)p.dul;
    double ssp = 0.0, ssx = 0.0, ssy = 0.0, ssz = 0.0;
    for (int q = 0; q < nq; ++q) {
      const int64_t s = (c * MF + f) * QS + q;
      double u[NV], pr[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) u[v] = U[c * NV + v] + (double)dul[s * NV + v];
      cons2prim(p.gamma, u, pr);
      const double w = face_weight(p, ft, q);
      ssp = ssp + (pr[4] * w);
      if (p.governing == 1) {
        const double* g = p.fgrad ? p.fgrad + (i * QS + q) * 12 : p.ulv + s * 12;  // rows T, u, v, w
        const double ux = g[3], uy = g[4], uz = g[5], vx = g[6], vy = g[7], vz = g[8];
        const double wx = g[9], wy = g[10], wz = g[11];
        double mu, lam;
        sutherland(p, pr[0], pr[4], &mu, &lam);
        const double txx = (4.0 / 3.0) * ux - (2.0 / 3.0) * vy - (2.0 / 3.0) * wz;
        const double tyy = (4.0 / 3.0) * vy - (2.0 / 3.0) * ux - (2.0 / 3.0) * wz;
        const double tzz = (4.0 / 3.0) * wz - (2.0 / 3.0) * ux - (2.0 / 3.0) * vy;
        const double tyx = uy + vx, tzx = wx + uz, tzy = vz + wy;
        ssx = ssx - ((mu * ((nx * txx) + (ny * tyx) + (nz * tzx))) * w);
        ssy = ssy - ((mu * ((nx * tyx) + (ny * tyy) + (nz * tzy))) * w);
        ssz = ssz - ((mu * ((nx * tzx) + (ny * tzy) + (nz * tzz))) * w);
      }
    }
    ssp = ssp - p.pres;
    r[0] = (ssp * S * nx) + (ssx * S);
    r[1] = (ssp * S * ny) + (ssy * S);
    r[2] = (ssp * S * nz) + (ssz * S);
    if (cen) {
      const double xc = cen[c * 3], yc = cen[c * 3 + 1], zc = cen[c * 3 + 2];
      r[3] = (ssp * S * nz) * yc - (ssp * S * ny) * zc;
      r[4] = (ssp * S * nx) * zc - (ssp * S * nz) * xc;
      r[5] = (ssp * S * ny) * xc - (ssp * S * nx) * yc;
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) cols[k * p.nown + i] = r[k];
}

int force_device(ucg_engine* e, const Problem& p, const double* U, const double* dU, double* out) {
  int rc = launch_recon(e, p, U);
  if (rc) return rc;
  const bool weno = e->cfg.scheme == 3;
  double* tdul = weno ? (double*)e->adjw_face.p : (double*)e->adj_tdul.p;
  if (dU && weno) {  // the tangent face values: dG = least squares of dU, then the WENO tangent
    Problem pt = p;
    pt.gbuf = e->adjw_gbar.p;
    CK(launch_lsq_f64(e->cfg.iorder, pt, dU, e->stream));
    e->launches++;
    if ((rc = launch_weno_tangent(e, p, U, dU, (const double*)e->adjw_gbar.p, tdul))) return rc;
  } else if (dU) {
    k_jvp_muscl<<<blocks_for(e->n, 128), 128, 0, e->stream>>>(p, U, dU, tdul, nullptr, false);
    e->launches++;
  }
  k_force_cell<<<blocks_for(e->n, 128), 128, 0, e->stream>>>(p, U, dU, tdul, (double*)e->adj_fcell.p, nullptr, 0.0);
  k_sum1<<<1, 1024, 0, e->stream>>>((const double*)e->adj_fcell.p, e->n, out);
  e->launches += 2;
  CK(cudaGetLastError());
  return UCG_OK;
}

// dJ/dU at state U into g (device)
int force_vjp_device(ucg_engine* e, const Problem& p, const double* U, double* g) {
  const int64_t n = e->n;
  if (e->cfg.scheme == 3) {  // WENO: the face-value seed through the reconstruction's reverse
    int rc = launch_recon(e, p, U);
    if (rc) return rc;
    double* adjF = (double*)e->adjw_face.p;
    k_force_cell<<<blocks_for(n, 128), 128, 0, e->stream>>>(p, U, nullptr, nullptr, (double*)e->adj_fcell.p, adjF, 1.0);
    e->launches++;
    if ((rc = launch_weno_adjoint(e, p, U, adjF, (double*)e->adjw_gbar.p, (double*)e->adjw_scr.p,
                                  (double*)e->adjw_self.p, (double*)e->adjw_contrib.p)))
      return rc;
    k_adj_gather<<<blocks_for(n, 128), 128, 0, e->stream>>>(n, (const int64_t*)e->adjw_rptr.p,
                                                            (const int64_t*)e->adjw_rsrc.p,
                                                            (const double*)e->adjw_contrib.p, g);
    e->launches++;
    CK(cudaGetLastError());
    return UCG_OK;
  }
  int rc = adj_forward(e, p, U);
  if (rc) return rc;
  k_force_cell<<<blocks_for(n, 128), 128, 0, e->stream>>>(p, U, nullptr, nullptr, (double*)e->adj_fcell.p,
                                                          (double*)e->adj_face.p, 1.0);
  k_adj_muscl<<<blocks_for(n, 128), 128, 0, e->stream>>>(p, fwd_store(e), (const double*)e->adj_face.p,
                                                         (double*)e->adj_contrib.p, U, nullptr);
  k_adj_gather<<<blocks_for(n, 128), 128, 0, e->stream>>>(n, (const int64_t*)e->adj_rptr.p,
                                                          (const int64_t*)e->adj_rsrc.p,
                                                          (const double*)e->adj_contrib.p, g);
  e->launches += 3;
  CK(cudaGetLastError());
  return UCG_OK;
}

// ---------------------------------------------------------------- WENO
// The VJP of the WENO residual: conserved-variable WENO and CWENO, Euler or
// Navier-Stokes, FP64 form (the reverse map of its per-slot contributions).
int adjw_setup(ucg_engine* e) {
  const ucg_config& c = e->cfg;
  if (!(c.scheme == 3 && (c.ees == 0 || c.ees == 5) && c.wenwrt == 1 && (c.governing == 2 || c.governing == 1) &&
        c.precision == UCG_FP64 && c.riemann == 1 && !c.mood))
    return fail(e, UCG_EINVAL,
                "the WENO adjoint covers conserved-variable WENO and CWENO (EES 0 or 5, CWENO with or without WENO-Z), HLLC, Euler or Navier-Stokes, FP64 form, without MOOD");
  if (!ready(e) || !e->have_state) return fail(e, UCG_ESTATE, "geometry, tables and state are needed");
  if (!e->roles.empty()) return fail(e, UCG_EINVAL, "the adjoint covers whole meshes (no partition roles)");
  if (e->adjw_ready) return UCG_OK;
  const int64_t n = e->n, ngrp = (n + 31) / 32;
  const int A = c.admis_max, IM = c.imax, W = IM + 1, ID = c.ideg;
  const bool cw = c.ees == 5;
  const int IM2 = c.imax2;
  // slots: the cell, the central stencil's members, then the others' (CWENO:
  // IMAX2 members each)
  // and one per face: the neighbour that set a bound of the MUSCL fall-back
  const int64_t fslot = cw ? 1 + IM + (int64_t)(A - 1) * IM2 : 1 + (int64_t)A * IM;
  const int64_t slots = fslot + MF;
  cudaSetDevice(e->device);
  // the stencils, back from the device (interleaved over 32-cell groups)
  std::vector<int32_t> st((size_t)ngrp * 32 * A * W);
  CK(cudaMemcpyAsync(st.data(), e->sten.p, st.size() * 4, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  auto target = [&](int64_t i, int64_t s) -> int64_t {
    if (s == 0) return i;
    if (s >= fslot) return e->neigh_h[(size_t)i * MF + (s - fslot)];
    int ll, k;
    if (!cw || s - 1 < IM) {
      ll = (int)((s - 1) / IM);
      k = (int)((s - 1) % IM);
    } else {
      ll = 1 + (int)((s - 1 - IM) / IM2);
      k = (int)((s - 1 - IM) % IM2);
    }
    if (ll >= e->admis_h[i]) return -1;
    return st[(size_t)(((i >> 5) * A * W + ll * W + k + 1) * 32 + (i & 31))];
  };
  std::vector<int64_t> cnt(n + 1, 0);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t s = 0; s < slots; ++s) {
      const int64_t t = target(i, s);
      if (t >= 0 && t < n) ++cnt[t + 1];
    }
  for (int64_t j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
  std::vector<int64_t> src(cnt[n]), pos(cnt.begin(), cnt.end() - 1);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t s = 0; s < slots; ++s) {
      const int64_t t = target(i, s);
      if (t >= 0 && t < n) src[pos[t]++] = s * n + i;
    }
  auto get = [&](ucg_engine::DevBuf& b, size_t bytes) { return alloc(e, b, bytes); };
  int rc = get(e->adjw_face, (size_t)n * MF * e->QS * NV * 8);
  rc = rc ? rc : get(e->adjw_gbar, (size_t)ngrp * 32 * A * ID * NV * 8);
  rc = rc ? rc : get(e->adjw_scr, (size_t)ngrp * 32 * 2 * ID * NV * 8);
  rc = rc ? rc : get(e->adjw_self, (size_t)n * NV * 8);
  rc = rc ? rc : get(e->adjw_contrib, (size_t)n * slots * NV * 8);
  rc = rc ? rc : get(e->adjw_rptr, (size_t)(n + 1) * 8);
  rc = rc ? rc : get(e->adjw_rsrc, (size_t)std::max<int64_t>(1, cnt[n]) * 8);
  rc = rc ? rc : get(e->adjw_lam, (size_t)n * NV * 8);
  rc = rc ? rc : get(e->adjw_mu, (size_t)n * NV * 8 + 64 * 8);
  rc = rc ? rc : get(e->adjw_pface, (size_t)std::max<int64_t>(1, e->nown - e->nown_plain) * NV * 8);
  rc = rc ? rc : get(e->adjw_tmp, (size_t)(std::max<int64_t>(1, e->nown - e->nown_plain) / 1024 + 2) * NV * 8);
  if (c.governing == 1) {  // viscous terms: point-gradient adjoints, coefficient adjoints or tangents
    rc = rc ? rc : get(e->adjw_gpt, (size_t)n * MF * e->QS * 12 * 8);
    rc = rc ? rc : get(e->adjw_gvb, (size_t)n * ID * 4 * 8);
    rc = rc ? rc : get(e->adjw_tfg, (size_t)std::max<int64_t>(1, e->nown) * e->QS * 12 * 8);
  }
  if (rc) return rc;
  CK(cudaMemcpyAsync(e->adjw_rptr.p, cnt.data(), (n + 1) * 8, cudaMemcpyHostToDevice, e->stream));
  if (cnt[n]) CK(cudaMemcpyAsync(e->adjw_rsrc.p, src.data(), cnt[n] * 8, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemsetAsync(e->adjw_face.p, 0, (size_t)n * MF * e->QS * NV * 8, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  e->adjw_ready = true;
  return UCG_OK;
}

// mu = (dR/dU)^T lam, psum = (dR/dp)^T lam for the WENO residual (device)
int weno_vjp_device(ucg_engine* e, const Problem& p, const double* U, const double* lam, double* mu, double* psum) {
  int rc = launch_recon(e, p, U);  // stencil polynomials (gbuf) and face values (dul)
  if (rc) return rc;
  const int64_t n = e->n, nplain = e->nown_plain, nbnd = e->nown - nplain;
  double* adjF = (double*)e->adjw_face.p;
  if (nplain) k_adj_face<<<blocks_for(nplain, 64), 64, 0, e->stream>>>(p, nplain, U, lam, adjF);
  if (nbnd)
    k_adj_face_bnd<<<blocks_for(nbnd * 10, 128), 128, 0, e->stream>>>(p, nplain, U, lam, adjF,
                                                                      (double*)e->adjw_pface.p);
  e->launches += (nplain > 0) + (nbnd > 0);
  const bool ns = e->cfg.governing == 1;
  if (ns) {  // the viscous fluxes at every face point, from the stored face-point gradients
    k_adj_visc<<<blocks_for(e->nown, 128), 128, 0, e->stream>>>(p, nplain, U, lam, adjF, (double*)e->adjw_pface.p,
                                                               (double*)e->adjw_gpt.p, p.fgrad);
    e->launches++;
  }
  if ((rc = launch_weno_adjoint(e, p, U, adjF, (double*)e->adjw_gbar.p, (double*)e->adjw_scr.p,
                                (double*)e->adjw_self.p, (double*)e->adjw_contrib.p)))
    return rc;
  if (ns && (rc = launch_weno_visc_adjoint(e, p, U, (const double*)e->adjw_gpt.p, (double*)e->adjw_gvb.p,
                                           (double*)e->adjw_contrib.p)))
    return rc;
  k_adj_gather<<<blocks_for(n, 128), 128, 0, e->stream>>>(n, (const int64_t*)e->adjw_rptr.p,
                                                          (const int64_t*)e->adjw_rsrc.p,
                                                          (const double*)e->adjw_contrib.p, mu);
  e->launches++;
  if (nbnd) {
    const int64_t rows = 1024, nb = (nbnd + rows - 1) / rows;
    k_colsum5_part<<<(unsigned)nb, 256, 0, e->stream>>>((const double*)e->adjw_pface.p, nbnd, rows,
                                                         (double*)e->adjw_tmp.p);
    k_colsum5<<<NV, 256, 0, e->stream>>>((const double*)e->adjw_tmp.p, nb, psum);
    e->launches += 2;
  } else {
    CK(cudaMemsetAsync(psum, 0, NV * sizeof(double), e->stream));
  }
  CK(cudaGetLastError());
  return UCG_OK;
}

// dR = (dR/dU) dU + (dR/dp) dp for the WENO residual (device)
int weno_jvp_device(ucg_engine* e, const Problem& p, const double* U, const double* dU, const Dp5& dp, double* dR) {
  int rc = launch_recon(e, p, U);  // G (gbuf) and face values (dul)
  if (rc) return rc;
  Problem pt = p;
  pt.gbuf = e->adjw_gbar.p;  // dG = least squares of dU
  CK(launch_lsq_f64(e->cfg.iorder, pt, dU, e->stream));
  e->launches++;
  double* tdul = (double*)e->adjw_face.p;
  double* tflux = (double*)e->adjw_contrib.p;
  if ((rc = launch_weno_tangent(e, p, U, dU, (const double*)e->adjw_gbar.p, tdul))) return rc;
  double* tfg = nullptr;
  if (e->cfg.governing == 1) {
    tfg = (double*)e->adjw_tfg.p;
    if ((rc = launch_weno_visc_tangent(e, p, U, dU, (double*)e->adjw_gvb.p, tfg))) return rc;
  }
  k_jvp_face<<<blocks_for(e->nown, 128), 128, 0, e->stream>>>(p, U, dU, tdul, dp, tflux, nullptr, tfg);
  k_jvp_sum<<<blocks_for(e->n, 256), 256, 0, e->stream>>>(p, tflux, dR);
  e->launches += 2;
  CK(cudaGetLastError());
  return UCG_OK;
}

// ------------------------------------------------ the kinetic-energy objective
// J = sum_c V_c |m_c|^2 / (2 rho_c), the TGV kinetic-energy sum of
// TIME_MARCHING (src/time_p.f90:4145-4198) without its normalisation.
// Per cell: V * KE, or with a tangent dU its derivative V * dKE/dU . dU.
__global__ void k_ke_cell(Problem p, const double* __restrict__ U, const double* __restrict__ dU,
                          double* __restrict__ out) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  const double* u = U + c * NV;
  const double ir = 1.0 / u[0], mm = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
  if (!dU) {
    out[c] = p.vol[c] * (0.5 * mm * ir);
    return;
  }
  const double* d = dU + c * NV;
  out[c] = p.vol[c] * ((-0.5 * mm * ir * ir) * d[0] + (u[1] * d[1] + u[2] * d[2] + u[3] * d[3]) * ir);
}
// g = dJ/dU of the kinetic energy
__global__ void k_ke_grad(Problem p, const double* __restrict__ U, double* __restrict__ g) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  const double* u = U + c * NV;
  const double ir = 1.0 / u[0], mm = u[1] * u[1] + u[2] * u[2] + u[3] * u[3], v = p.vol[c];
  g[c * NV + 0] = v * (-0.5 * mm * ir * ir);
  g[c * NV + 1] = v * (u[1] * ir);
  g[c * NV + 2] = v * (u[2] * ir);
  g[c * NV + 3] = v * (u[3] * ir);
  g[c * NV + 4] = 0.0;
}

// The scheme-specific pieces of the adjoint and tangent runs: the residual
// VJP/JVP (MUSCL or WENO) with their buffers, and the objective J (wall
// force, MUSCL only; kinetic energy, either).
struct RunOps {
  bool weno;
  int obj;
  double* lam;   // scratch vectors the VJP reads and writes
  double* mu;
  double* cell;  // [n] per-cell objective values
};

int run_setup(ucg_engine* e, int obj, RunOps& o) {
  o.weno = e->cfg.scheme == 3;
  o.obj = obj;
  if (obj != UCG_OBJ_FORCE_X && obj != UCG_OBJ_KE) return fail(e, UCG_EINVAL, "unknown objective");
  int rc = o.weno ? adjw_setup(e) : adj_setup(e);
  if (rc) return rc;
  const int64_t n = e->n;
  // four state-sized vectors and a few scalars (bar_vec, bar_scal), and the
  // per-cell objective values
  rc = alloc(e, e->adj_bar, (size_t)4 * n * NV * 8 + 64 * 8);
  rc = rc ? rc : alloc(e, e->adj_fcell, (size_t)n * 8);
  if (rc) return rc;
  o.lam = o.weno ? (double*)e->adjw_lam.p : (double*)e->adj_lam.p;
  o.mu = o.weno ? (double*)e->adjw_mu.p : (double*)e->adj_mu.p;
  o.cell = (double*)e->adj_fcell.p;
  return UCG_OK;
}
int run_vjp(ucg_engine* e, const RunOps& o, const Problem& p, const double* U, const double* lam, double* mu,
            double* psum) {
  return o.weno ? weno_vjp_device(e, p, U, lam, mu, psum) : vjp_device(e, p, U, lam, mu, psum);
}
int run_jvp(ucg_engine* e, const RunOps& o, const Problem& p, const double* U, const double* dU, const Dp5& dp,
            double* dR) {
  return o.weno ? weno_jvp_device(e, p, U, dU, dp, dR) : jvp_device(e, p, U, dU, dp, dR, true);
}
// J (dU null) or dJ/dU . dU at U into out[0]
int run_obj(ucg_engine* e, const RunOps& o, const Problem& p, const double* U, const double* dU, double* out) {
  if (o.obj == UCG_OBJ_FORCE_X) return force_device(e, p, U, dU, out);
  k_ke_cell<<<blocks_for(e->n, 256), 256, 0, e->stream>>>(p, U, dU, o.cell);
  k_sum1<<<1, 1024, 0, e->stream>>>(o.cell, e->n, out);
  e->launches += 2;
  CK(cudaGetLastError());
  return UCG_OK;
}
int run_obj_vjp(ucg_engine* e, const RunOps& o, const Problem& p, const double* U, double* g) {
  if (o.obj == UCG_OBJ_FORCE_X) return force_vjp_device(e, p, U, g);
  k_ke_grad<<<blocks_for(e->n, 256), 256, 0, e->stream>>>(p, U, g);
  e->launches++;
  CK(cudaGetLastError());
  return UCG_OK;
}

// host <-> device; [n][5] per-cell arrays go through the caller's cell order
int copy_in(ucg_engine* e, double* dst, const double* src, size_t count) {
  if (count == (size_t)e->n * NV) return cells_in(e, dst, src);
  CK(cudaMemcpyAsync(dst, src, count * 8, cudaMemcpyHostToDevice, e->stream));
  return UCG_OK;
}
int copy_out(ucg_engine* e, double* dst, const double* src, size_t count) {
  if (count == (size_t)e->n * NV) return cells_out(e, dst, src);
  CK(cudaMemcpyAsync(dst, src, count * 8, cudaMemcpyDeviceToHost, e->stream));
  return UCG_OK;
}

}  // namespace

// =================================================================== ABI
extern "C" {

int ucg_force(ucg_engine* e, double* fx) {
  if (!e || !fx) return fail(e, UCG_EINVAL, "null argument");
  int rc = e->cfg.scheme == 3 ? adjw_setup(e) : adj_setup(e);
  rc = rc ? rc : alloc(e, e->adj_bar, (size_t)4 * e->n * NV * 8 + 64 * 8);
  rc = rc ? rc : alloc(e, e->adj_fcell, (size_t)e->n * 8);
  if (rc) return rc;
  cudaSetDevice(e->device);
  Problem p = make_problem(e);
  double* s = bar_scal(e);
  if ((rc = force_device(e, p, (const double*)e->Un.p, nullptr, s))) return rc;
  if ((rc = copy_out(e, fx, s, 1))) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return UCG_OK;
}

int ucg_force_vjp(ucg_engine* e, double* dJdU) {
  if (!e || !dJdU) return fail(e, UCG_EINVAL, "null argument");
  const bool weno = e->cfg.scheme == 3;
  int rc = weno ? adjw_setup(e) : adj_setup(e);
  rc = rc ? rc : alloc(e, e->adj_fcell, (size_t)e->n * 8);
  if (rc) return rc;
  cudaSetDevice(e->device);
  Problem p = make_problem(e);
  double* g = weno ? (double*)e->adjw_mu.p : (double*)e->adj_mu.p;
  if ((rc = force_vjp_device(e, p, (const double*)e->Un.p, g))) return rc;
  if ((rc = copy_out(e, dJdU, g, (size_t)e->n * NV))) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return UCG_OK;
}

int ucg_wall_loads(ucg_engine* e, const double* centre, double* out) {
  if (!e || !out) return fail(e, UCG_EINVAL, "null argument");
  if (!ready(e) || !e->have_state) return fail(e, UCG_ESTATE, "geometry, tables and state are needed");
  if (e->cfg.mood) return fail(e, UCG_EINVAL, "the wall loads take the plain reconstruction (no MOOD)");
  const int64_t n = e->n, nown = e->nown;
  cudaSetDevice(e->device);
  int rc = alloc(e, e->wl_buf, ((size_t)6 * std::max<int64_t>(nown, 1) + 8 + (size_t)3 * n) * 8);
  if (rc) return rc;
  double* cols = (double*)e->wl_buf.p;
  double* sums = cols + 6 * std::max<int64_t>(nown, 1);
  double* cen = sums + 8;
  if (centre) {  // into the engine's cell order
    if (e->n2o.empty()) {
      CK(cudaMemcpyAsync(cen, centre, (size_t)n * 3 * 8, cudaMemcpyHostToDevice, e->stream));
    } else {
      std::vector<double> h((size_t)n * 3);
      for (int64_t c = 0; c < n; ++c)
        for (int k = 0; k < 3; ++k) h[c * 3 + k] = centre[(size_t)e->n2o[c] * 3 + k];
      CK(cudaMemcpyAsync(cen, h.data(), h.size() * 8, cudaMemcpyHostToDevice, e->stream));
      CK(cudaStreamSynchronize(e->stream));
    }
  }
  Problem p = make_problem(e);
  if ((rc = launch_recon(e, p, (const double*)e->Un.p))) return rc;
  const unsigned nb = blocks_for(std::max<int64_t>(nown, 1), 128);
  if (e->cfg.precision == UCG_FP64)
    k_wall_loads<double><<<nb, 128, 0, e->stream>>>(p, (const double*)e->Un.p, centre ? cen : nullptr, cols);
  else
    k_wall_loads<float><<<nb, 128, 0, e->stream>>>(p, (const double*)e->Un.p, centre ? cen : nullptr, cols);
  for (int k = 0; k < 6; ++k) k_sum1<<<1, 1024, 0, e->stream>>>(cols + k * nown, nown, sums + k);
  e->launches += 7;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, sums, 6 * 8, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return UCG_OK;
}

int ucg_residual_vjp(ucg_engine* e, const double* lambda, double* mu, double* pbar) {
  if (!e || !lambda || !mu) return fail(e, UCG_EINVAL, "null argument");
  if (e->cfg.scheme == 3) {  // WENO
    int rc = adjw_setup(e);
    if (rc) return rc;
    cudaSetDevice(e->device);
    Problem p = make_problem(e);
    const size_t m = (size_t)e->n * NV;
    double* s = (double*)e->adjw_mu.p + m;
    if ((rc = copy_in(e, (double*)e->adjw_lam.p, lambda, m))) return rc;
    if ((rc = weno_vjp_device(e, p, (const double*)e->Un.p, (const double*)e->adjw_lam.p, (double*)e->adjw_mu.p, s)))
      return rc;
    if ((rc = copy_out(e, mu, (const double*)e->adjw_mu.p, m))) return rc;
    if (pbar && (rc = copy_out(e, pbar, s, NV))) return rc;
    CK(cudaStreamSynchronize(e->stream));
    return UCG_OK;
  }
  int rc = adj_setup(e);
  if (rc) return rc;
  cudaSetDevice(e->device);
  Problem p = make_problem(e);
  const size_t m = (size_t)e->n * NV;
  double* s = bar_scal(e);
  if ((rc = copy_in(e, (double*)e->adj_lam.p, lambda, m))) return rc;
  if ((rc = vjp_device(e, p, (const double*)e->Un.p, (const double*)e->adj_lam.p, (double*)e->adj_mu.p, s)))
    return rc;
  if ((rc = copy_out(e, mu, (const double*)e->adj_mu.p, m))) return rc;
  if (pbar && (rc = copy_out(e, pbar, s, NV))) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return UCG_OK;
}

int ucg_residual_jvp(ucg_engine* e, const double* du, const double* dp, double* drhs) {
  if (!e || !du || !drhs) return fail(e, UCG_EINVAL, "null argument");
  if (e->cfg.scheme == 3) {  // WENO
    int rc = adjw_setup(e);
    if (rc) return rc;
    cudaSetDevice(e->device);
    Problem p = make_problem(e);
    const size_t m = (size_t)e->n * NV;
    Dp5 d{};
    if (dp)
      for (int k = 0; k < NV; ++k) d.v[k] = dp[k];
    if ((rc = copy_in(e, (double*)e->adjw_lam.p, du, m))) return rc;
    if ((rc = weno_jvp_device(e, p, (const double*)e->Un.p, (const double*)e->adjw_lam.p, d, (double*)e->adjw_mu.p)))
      return rc;
    if ((rc = copy_out(e, drhs, (const double*)e->adjw_mu.p, m))) return rc;
    CK(cudaStreamSynchronize(e->stream));
    return UCG_OK;
  }
  int rc = adj_setup(e);
  if (rc) return rc;
  cudaSetDevice(e->device);
  Problem p = make_problem(e);
  const size_t m = (size_t)e->n * NV;
  Dp5 d{};
  if (dp)
    for (int k = 0; k < NV; ++k) d.v[k] = dp[k];
  if ((rc = copy_in(e, (double*)e->adj_tU.p, du, m))) return rc;
  if ((rc = jvp_device(e, p, (const double*)e->Un.p, (const double*)e->adj_tU.p, d, (double*)e->adj_mu.p)))
    return rc;
  if ((rc = copy_out(e, drhs, (const double*)e->adj_mu.p, m))) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return UCG_OK;
}

int ucg_time_adjoint(ucg_engine* e, int32_t reps, double* ms) {
  if (!e || !ms || reps < 1) return fail(e, UCG_EINVAL, "bad argument");
  const bool weno = e->cfg.scheme == 3;
  int rc = weno ? adjw_setup(e) : adj_setup(e);
  if (rc) return rc;
  cudaSetDevice(e->device);
  Problem p = make_problem(e);
  const int64_t n = e->n;
  const double* U = (const double*)e->Un.p;
  double* x = weno ? (double*)e->adjw_lam.p : bar_vec(e, 0);
  double* y = weno ? (double*)e->adjw_mu.p : bar_vec(e, 1);
  double* ps = weno ? (double*)e->adjw_mu.p + (size_t)n * NV : bar_scal(e);
  CK(cudaMemsetAsync(x, 0, (size_t)n * NV * 8, e->stream));
  cudaEvent_t ev[4];
  for (auto& t : ev) CK(cudaEventCreate(&t));
  double acc[3] = {0, 0, 0};
  Dp5 d{};
  // r = -1: one untimed pass (first launches load the kernels' modules)
  for (int r = -1; r < reps && !rc; ++r) {
    cudaEventRecord(ev[0], e->stream);
    rc = launch_recon(e, p, U);
    if (!rc) rc = launch_flux(e, p, 0, U, U, nullptr, 0.0);
    cudaEventRecord(ev[1], e->stream);
    if (!rc) rc = weno ? weno_vjp_device(e, p, U, x, y, ps) : vjp_device(e, p, U, x, y, ps);
    cudaEventRecord(ev[2], e->stream);
    if (!rc) rc = weno ? weno_jvp_device(e, p, U, x, d, y) : jvp_device(e, p, U, x, d, y);
    cudaEventRecord(ev[3], e->stream);
    cudaEventSynchronize(ev[3]);
    if (r < 0) continue;
    float t;
    for (int k = 0; k < 3; ++k) {
      cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      acc[k] += t;
    }
  }
  for (auto& t : ev) cudaEventDestroy(t);
  if (rc) return rc;
  for (int k = 0; k < 3; ++k) ms[k] = acc[k] / reps;
  CK(cudaGetLastError());
  return UCG_OK;
}

int ucg_adjoint_run_obj(ucg_engine* e, int32_t objective, int32_t nsteps, double dt, int32_t every, double* J,
                        double* dJdU0, double* dJdp) {
  if (!e || nsteps < 0 || every < 1 || !(dt > 0.0)) return fail(e, UCG_EINVAL, "bad argument");
  RunOps o{};
  int rc = run_setup(e, objective, o);
  if (rc) return rc;
  cudaSetDevice(e->device);
  const int64_t n = e->n;
  const size_t m = (size_t)n * NV, mb = m * 8;
  const int nseg = (nsteps + every - 1) / every;
  const int K = std::min<int>(every, std::max(nsteps, 1));
  // checkpoints [nseg][n][5], stage states of one segment [K][3][n][5], final state
  if ((rc = alloc(e, e->adj_traj, ((size_t)std::max(nseg, 1) + (size_t)3 * K + 1) * mb))) return rc;
  double* ckpt = (double*)e->adj_traj.p;
  double* traj = ckpt + (size_t)std::max(nseg, 1) * m;
  double* fin = traj + (size_t)3 * K * m;
  double* Un = (double*)e->Un.p;
  Problem p = make_problem(e);
  // forward with checkpoints
  for (int s = 0; s < nsteps; ++s) {
    if (s % every == 0) CK(cudaMemcpyAsync(ckpt + (size_t)(s / every) * m, Un, mb, cudaMemcpyDeviceToDevice, e->stream));
    if ((rc = rk3(e, dt, false))) return rc;
  }
  CK(cudaMemcpyAsync(fin, Un, mb, cudaMemcpyDeviceToDevice, e->stream));
  double* sc = bar_scal(e);  // sc[0] J, sc[8..12] pbar accumulator, sc[16..20] partial
  double* pacc = sc + 8;
  double* part = sc + 16;
  if ((rc = run_obj(e, o, p, Un, nullptr, sc))) return rc;
  // terminal adjoint: dJ/dU^N
  double* ub = bar_vec(e, 0);   // adjoint of the current step's output
  double* u0b = bar_vec(e, 1);  // adjoint of its input
  double* u1b = bar_vec(e, 2);
  double* u2b = bar_vec(e, 3);
  double* mu = o.mu;
  double* lam = o.lam;
  if ((rc = run_obj_vjp(e, o, p, Un, ub))) return rc;
  CK(cudaMemsetAsync(pacc, 0, NV * 8, e->stream));
  const unsigned bm = blocks_for((int64_t)m, 256), bv = blocks_for((int64_t)m, 256);
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int s0 = seg * every, s1 = std::min(nsteps, s0 + every);
    CK(cudaMemcpyAsync(Un, ckpt + (size_t)seg * m, mb, cudaMemcpyDeviceToDevice, e->stream));
    for (int s = s0; s < s1; ++s) {
      double* t = traj + (size_t)3 * (s - s0) * m;
      CK(cudaMemcpyAsync(t, Un, mb, cudaMemcpyDeviceToDevice, e->stream));
      if ((rc = rk3(e, dt, false))) return rc;
      CK(cudaMemcpyAsync(t + m, e->Ua.p, mb, cudaMemcpyDeviceToDevice, e->stream));
      CK(cudaMemcpyAsync(t + 2 * m, e->Ub.p, mb, cudaMemcpyDeviceToDevice, e->stream));
    }
    for (int s = s1 - 1; s >= s0; --s) {
      const double* U0 = traj + (size_t)3 * (s - s0) * m;
      const double* U1 = U0 + m;
      const double* U2 = U0 + 2 * m;
      // U3 = 1/3 U0 + 2/3 U2 - 2/3 dt R(U2)/V
      k_over_vol<<<bv, 256, 0, e->stream>>>(p, 1.0, ub, lam);
      if ((rc = run_vjp(e, o, p, U2, lam, mu, part))) return rc;
      k_pacc<<<1, 32, 0, e->stream>>>(-(2.0 / 3.0) * dt, part, pacc);
      CK(cudaMemcpyAsync(u2b, ub, mb, cudaMemcpyDeviceToDevice, e->stream));
      k_axpby<<<bm, 256, 0, e->stream>>>((int64_t)m, -(2.0 / 3.0) * dt, mu, 2.0 / 3.0, u2b);
      CK(cudaMemcpyAsync(u0b, ub, mb, cudaMemcpyDeviceToDevice, e->stream));
      k_axpby<<<bm, 256, 0, e->stream>>>((int64_t)m, 0.0, ub, 1.0 / 3.0, u0b);
      // U2 = 3/4 U0 + 1/4 U1 - 1/4 dt R(U1)/V
      k_over_vol<<<bv, 256, 0, e->stream>>>(p, 1.0, u2b, lam);
      if ((rc = run_vjp(e, o, p, U1, lam, mu, part))) return rc;
      k_pacc<<<1, 32, 0, e->stream>>>(-0.25 * dt, part, pacc);
      CK(cudaMemcpyAsync(u1b, u2b, mb, cudaMemcpyDeviceToDevice, e->stream));
      k_axpby<<<bm, 256, 0, e->stream>>>((int64_t)m, -0.25 * dt, mu, 0.25, u1b);
      k_axpby<<<bm, 256, 0, e->stream>>>((int64_t)m, 0.75, u2b, 1.0, u0b);
      // U1 = U0 - dt R(U0)/V
      k_over_vol<<<bv, 256, 0, e->stream>>>(p, 1.0, u1b, lam);
      if ((rc = run_vjp(e, o, p, U0, lam, mu, part))) return rc;
      k_pacc<<<1, 32, 0, e->stream>>>(-dt, part, pacc);
      k_axpby<<<bm, 256, 0, e->stream>>>((int64_t)m, 1.0, u1b, 1.0, u0b);
      k_axpby<<<bm, 256, 0, e->stream>>>((int64_t)m, -dt, mu, 1.0, u0b);
      CK(cudaMemcpyAsync(ub, u0b, mb, cudaMemcpyDeviceToDevice, e->stream));
      e->launches += 12;
    }
  }
  CK(cudaGetLastError());
  // the handle's state is the final state
  CK(cudaMemcpyAsync(Un, fin, mb, cudaMemcpyDeviceToDevice, e->stream));
  if (J && (rc = copy_out(e, J, sc, 1))) return rc;
  if (dJdU0 && (rc = copy_out(e, dJdU0, ub, m))) return rc;
  if (dJdp && (rc = copy_out(e, dJdp, pacc, NV))) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return UCG_OK;
}

int ucg_adjoint_run(ucg_engine* e, int32_t nsteps, double dt, int32_t every, double* J, double* dJdU0,
                    double* dJdp) {
  return ucg_adjoint_run_obj(e, UCG_OBJ_FORCE_X, nsteps, dt, every, J, dJdU0, dJdp);
}

int ucg_tangent_run_obj(ucg_engine* e, int32_t objective, int32_t nsteps, double dt, const double* dU0,
                        const double* dp, double* J, double* dJ) {
  if (!e || nsteps < 0 || !dU0 || !(dt > 0.0)) return fail(e, UCG_EINVAL, "bad argument");
  RunOps o{};
  int rc = run_setup(e, objective, o);
  if (rc) return rc;
  cudaSetDevice(e->device);
  const int64_t n = e->n;
  const size_t m = (size_t)n * NV, mb = m * 8;
  Dp5 d{};
  if (dp)
    for (int k = 0; k < NV; ++k) d.v[k] = dp[k];
  Problem p = make_problem(e);
  double* Un = (double*)e->Un.p;
  double* t0 = bar_vec(e, 0);  // tangent of the step's input
  double* t1 = bar_vec(e, 1);
  double* t2 = bar_vec(e, 2);
  double* dR = bar_vec(e, 3);
  double* sc = bar_scal(e);
  const unsigned bm = blocks_for((int64_t)m, 256);
  if ((rc = copy_in(e, t0, dU0, m))) return rc;
  // each JVP leaves the face values of its state in the reconstruction
  // buffers, which the stage's flux and update then use
  for (int s = 0; s < nsteps; ++s) {
    // stage 1 at U0 = Un
    if ((rc = run_jvp(e, o, p, Un, t0, d, dR))) return rc;
    if ((rc = launch_flux(e, p, 1, Un, Un, (double*)e->Ua.p, dt))) return rc;
    k_over_vol<<<bm, 256, 0, e->stream>>>(p, -dt, dR, t1);
    k_axpby<<<bm, 256, 0, e->stream>>>((int64_t)m, 1.0, t0, 1.0, t1);
    // stage 2 at U1 = Ua
    if ((rc = run_jvp(e, o, p, (const double*)e->Ua.p, t1, d, dR))) return rc;
    if ((rc = launch_flux(e, p, 2, (const double*)e->Ua.p, Un, (double*)e->Ub.p, dt))) return rc;
    k_over_vol<<<bm, 256, 0, e->stream>>>(p, -0.25 * dt, dR, t2);
    k_axpby<<<bm, 256, 0, e->stream>>>((int64_t)m, 0.75, t0, 1.0, t2);
    k_axpby<<<bm, 256, 0, e->stream>>>((int64_t)m, 0.25, t1, 1.0, t2);
    // stage 3 at U2 = Ub
    if ((rc = run_jvp(e, o, p, (const double*)e->Ub.p, t2, d, dR))) return rc;
    if ((rc = launch_flux(e, p, 3, (const double*)e->Ub.p, Un, Un, dt))) return rc;
    k_over_vol<<<bm, 256, 0, e->stream>>>(p, -(2.0 / 3.0) * dt, dR, t1);
    k_axpby<<<bm, 256, 0, e->stream>>>((int64_t)m, 1.0 / 3.0, t0, 1.0, t1);
    k_axpby<<<bm, 256, 0, e->stream>>>((int64_t)m, 2.0 / 3.0, t2, 1.0, t1);
    CK(cudaMemcpyAsync(t0, t1, mb, cudaMemcpyDeviceToDevice, e->stream));
    e->launches += 9;
  }
  if ((rc = run_obj(e, o, p, Un, nullptr, sc))) return rc;
  if ((rc = run_obj(e, o, p, Un, t0, sc + 1))) return rc;
  CK(cudaGetLastError());
  if (J && (rc = copy_out(e, J, sc, 1))) return rc;
  if (dJ && (rc = copy_out(e, dJ, sc + 1, 1))) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return UCG_OK;
}

int ucg_tangent_run(ucg_engine* e, int32_t nsteps, double dt, const double* dU0, const double* dp, double* J,
                    double* dJ) {
  return ucg_tangent_run_obj(e, UCG_OBJ_FORCE_X, nsteps, dt, dU0, dp, J, dJ);
}

}  // extern "C"
