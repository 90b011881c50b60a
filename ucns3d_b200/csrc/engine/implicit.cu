// Implicit pseudo-time stepping toward a steady state (ucg_implicit_step):
// IMPLICIT_TIMEs (src/time_p.f90:2783-2905) with RELAXATION
// (src/implicit_time.f90:1-778, RELAX = 1, ISCOUN = 1), CALCULATE_JACOBIAN
// (src/implicit_fluxes.f90:12-594, RUNGEKUTTA = 10) and the local time steps
// of CALCULATE_CFLL (src/time_p.f90:193-333).  Per step:
//
//   k_imp_dtl    one thread per cell: DTL = CCFL min_edge / (max|u_i| + c)
//                (+ the viscous term of the Navier-Stokes form)
//   k_imp_jac    one thread per cell: the first-order Jacobian from the cell
//                means, diagonal sum_f (vpp_f / 2) area_f + V / DTL (a
//                multiple of the identity, stored as its inverse) and per
//                face (J(U_R) n / 2 - (vpp / 2) I) area, J of
//                COMPUTE_JACOBIANSE (src/flow_operations.f90:4004-4049)
//                with U_R the neighbour's mean or the boundary ghost
//   k_imp_sweep  one thread per cell: du = D^-1 (-RHS - sum_f O_f du_f),
//                SWEEPS = 10 times
//   k_imp_add    U += du, non-finite corrections raise HEALTH_NONPHYS
//
// The reference's sweep updates IMPDU in place inside an OpenMP loop, so a
// cell reads neighbours of the current or of the previous sweep depending
// on the thread schedule (a serial run is Gauss-Seidel in cell order).
// Here every sweep reads the previous sweep's corrections (block Jacobi),
// which is deterministic; the converged state is the same.  du_f on a
// physical face: inflow (1) 0, outflow (2) and far field (6) the cell's own
// du (the far field's IBFC branch is never taken: BOUNDARYS does not set
// IBFC), symmetry and walls (3, 4) the ghost of du (BOUNDARYS, linear there).
#include <cuda_runtime.h>

#include <cmath>

#include "device.cuh"
#include "engine_internal.h"

using namespace ucg;
using namespace ucg_host;

namespace {

constexpr int NJ = NV * NV;

// COMPUTE_JACOBIANSE without a moving frame: the flux Jacobian of the
// conserved state q along the unit normal n (row-major [5][5]).  Entry
// (5,3) takes gamma - 2 where the others of that row take gamma - 1, as the
// reference writes it.
__device__ __forceinline__ void flux_jacobian(const double* q, double gamma, double nx, double ny, double nz,
                                              double* J) {
  const double a2 = gamma - 1.0, a3 = gamma - 2.0;
  const double oors = 1.0 / q[0];
  const double us = q[1] * oors, vs = q[2] * oors, ws = q[3] * oors, es = q[4] * oors;
  const double phi = 0.5 * a2 * ((us * us) + (vs * vs) + (ws * ws));
  const double a1 = gamma * es - phi;
  const double vvs = nx * us + ny * vs + nz * ws;
  J[0] = 0.0;
  J[1] = nx;
  J[2] = ny;
  J[3] = nz;
  J[4] = 0.0;
  J[5] = nx * phi - us * vvs;
  J[6] = vvs - a3 * nx * us;
  J[7] = ny * us - a2 * nx * vs;
  J[8] = nz * us - a2 * nx * ws;
  J[9] = a2 * nx;
  J[10] = ny * phi - vs * vvs;
  J[11] = nx * vs - a2 * ny * us;
  J[12] = vvs - a3 * ny * vs;
  J[13] = nz * vs - a2 * ny * ws;
  J[14] = a2 * ny;
  J[15] = nz * phi - ws * vvs;
  J[16] = nx * ws - a2 * nz * us;
  J[17] = ny * ws - a2 * nz * vs;
  J[18] = vvs - a3 * nz * ws;
  J[19] = a2 * nz;
  J[20] = vvs * (phi - a1);
  J[21] = nx * a1 - a2 * us * vvs;
  J[22] = ny * a1 - a3 * vs * vvs;
  J[23] = nz * a1 - a2 * ws * vvs;
  J[24] = gamma * vvs;
}

// CALCULATE_CFLL: the local time step of every cell
__global__ void k_imp_dtl(Problem p, const double* __restrict__ U, double ccfl, double* __restrict__ dtl) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  double pr[NV];
  cons2prim(p.gamma, U + c * NV, pr);
  const double agrt = sqrt(pr[4] * p.gamma / pr[0]);
  const double veln = fmax(fmax(fabs(pr[1]), fabs(pr[2])), fabs(pr[3])) + agrt;
  const double me = p.minedge[c];
  if (p.governing == 1) {
    double mu, lam;
    sutherland(p, pr[0], pr[4], &mu, &lam);
    dtl[c] = ccfl * (1.0 / ((fabs(veln) / me) + (0.5 * (lam + mu) / (me * me))));
  } else {
    dtl[c] = ccfl * (me / fabs(veln));
  }
}

// CALCULATE_JACOBIAN from the cell means U: dinv[c] = 1 / diagonal,
// off[c][f] = the face's 5x5 block; dt > 0: the dual-time diagonal
// V (1/DTL + 1.5/dt) + sum_f ... (RUNGEKUTTA 11), else sum_f ... + V/DTL
__global__ void k_imp_jac(Problem p, const double* __restrict__ U, const double* __restrict__ dtl, double dt,
                          double* __restrict__ dinv, double* __restrict__ off) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  double cl[NV], lv[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) cl[v] = U[c * NV + v];
  cons2prim(p.gamma, cl, lv);
  const int nf = p.nfaces[c];
  double diag = 0.0;
  for (int f = 0; f < nf; ++f) {
    double r[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) r[k] = p.rot[(c * MF + f) * 4 + k];
    const double nx = r[0] * r[3], ny = r[1] * r[3], nz = r[2];
    const double area = p.area[c * MF + f];
    const int64_t nb = p.neigh[c * MF + f];
    double cr[NV], rv[NV], clr[NV], crr[NV];
    if (nb >= 0) {
#pragma unroll
      for (int v = 0; v < NV; ++v) cr[v] = U[nb * NV + v];
    } else {
      boundary_ghost(p, p.bc[c * MF + f], r, cl, p.bc_state, cr);
    }
    rot_f(r, cr, crr);
    rot_f(r, cl, clr);
    cons2prim(p.gamma, cr, rv);
    const double as1 = sqrt(lv[4] * p.gamma / lv[0]) + fabs(clr[1] / clr[0]);
    const double as2 = sqrt(rv[4] * p.gamma / rv[0]) + fabs(crr[1] / crr[0]);
    double vpp = fmax(as1, as2);
    if (p.governing == 1) {
      double mul, laml, mur, lamr;
      sutherland(p, lv[0], lv[4], &mul, &laml);
      sutherland(p, rv[0], rv[4], &mur, &lamr);
      double vis = (mul + mur) * 0.5;
      const double rh = 0.5 * (cl[0] + cr[0]), dih = p.dih[c * MF + f];
      vis = fmax((4.0 / (3.0 * rh)) * vis * area / dih, (p.gamma / rh) * vis * area / (dih * p.prandtl));
      vpp = vpp + vis;
    }
    diag = diag + (0.5 * (vpp * 1.0)) * area;
    double J[NJ];
    flux_jacobian(cr, p.gamma, nx, ny, nz, J);
    double* o = off + (c * MF + f) * NJ;
#pragma unroll
    for (int i = 0; i < NV; ++i)
#pragma unroll
      for (int j = 0; j < NV; ++j) o[i * NV + j] = ((0.5 * J[i * NV + j]) - ((0.5 * vpp) * (i == j ? 1.0 : 0.0))) * area;
  }
  if (dt > 0.0) diag = p.vol[c] * ((1.0 / dtl[c]) + (1.5 / dt)) + diag;
  else diag = diag + (p.vol[c] / dtl[c]);
  dinv[c] = 1.0 / diag;
}

// one relaxation sweep: du_new = D^-1 (b - sum_f O_f du_f(du_old)) with
// b = -RHS, or with dual time (U1 the iterate, U2 and U3 the last two
// physical steps, ISCOUN 2) b = -(RHS + V (1.5 U1 - 2 U2 + 0.5 U3) / dt)
__global__ void k_imp_sweep(Problem p, const double* __restrict__ dinv, const double* __restrict__ off,
                            const double* __restrict__ du, double* __restrict__ dn, const double* __restrict__ U1,
                            const double* __restrict__ U2, const double* __restrict__ U3, double dt) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  double b[NV], d0[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    if (U1) {
      const int64_t i = c * NV + v;
      b[v] = -(p.rhs[i] + ((((1.5 * U1[i]) - (2.0 * U2[i]) + (0.5 * U3[i])) / dt) * p.vol[c]));
    } else {
      b[v] = -p.rhs[c * NV + v];
    }
    d0[v] = du[c * NV + v];
  }
  const int nf = p.nfaces[c];
  for (int f = 0; f < nf; ++f) {
    const int64_t nb = p.neigh[c * MF + f];
    double d1[NV];
    if (nb >= 0) {
#pragma unroll
      for (int v = 0; v < NV; ++v) d1[v] = du[nb * NV + v];
    } else {
      const int code = p.bc[c * MF + f];
      if (code == 1) {
#pragma unroll
        for (int v = 0; v < NV; ++v) d1[v] = 0.0;
      } else if (code == 3 || code == 4) {
        double r[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) r[k] = p.rot[(c * MF + f) * 4 + k];
        boundary_ghost(p, code, r, d0, p.bc_state, d1);
      } else {  // 2 outflow, 6 far field
#pragma unroll
        for (int v = 0; v < NV; ++v) d1[v] = d0[v];
      }
    }
    const double* o = off + (c * MF + f) * NJ;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double t = 0.0;
#pragma unroll
      for (int j = 0; j < NV; ++j) t = t + o[i * NV + j] * d1[j];
      b[i] = b[i] - t;
    }
  }
  const double di = dinv[c];
#pragma unroll
  for (int v = 0; v < NV; ++v) dn[c * NV + v] = di * b[v];
}

__global__ void k_imp_add(Problem p, double* __restrict__ U, const double* __restrict__ du) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  bool bad = false;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double d = du[c * NV + v];
    bad = bad || !isfinite(d);
    U[c * NV + v] = U[c * NV + v] + d;
  }
  if (bad) atomicOr(p.health, HEALTH_NONPHYS);
}

// sum over cells of |du|_2 V, in a fixed order: per block a tree sum into
// part[block], then one thread adds the blocks in order
__global__ void __launch_bounds__(256) k_imp_norm_part(Problem p, const double* __restrict__ du,
                                                       double* __restrict__ part) {
  __shared__ double s[256];
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double x = 0.0;
  if (c < p.n) {
    const double* d = du + c * NV;
    x = sqrt((d[0] * d[0]) + (d[1] * d[1]) + (d[2] * d[2]) + (d[3] * d[3]) + (d[4] * d[4])) * p.vol[c];
  }
  s[threadIdx.x] = x;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}
__global__ void k_imp_norm_sum(const double* __restrict__ part, int64_t nb, double* __restrict__ out) {
  double t = 0.0;
  for (int64_t i = 0; i < nb; ++i) t += part[i];
  *out = t;
}

// RHS, local time steps (with local_steps; else those in imp_dtl),
// Jacobian and the sweeps from du = 0; the correction in du[*cur]
int implicit_correction(ucg_engine* e, const Problem& p, double* U, double ccfl, int32_t nsweeps, double dt,
                        const double* U2, const double* U3, int* cur, bool local_steps = true) {
  const int64_t n = e->n;
  const unsigned blocks = (unsigned)((n + 127) / 128);
  double* dtl = (double*)e->imp_dtl.p;
  double* dinv = (double*)e->imp_dinv.p;
  double* off = (double*)e->imp_off.p;
  double* du[2] = {(double*)e->imp_du.p, (double*)e->imp_du.p + n * NV};
  int rc;
  if ((rc = launch_recon(e, p, U))) return rc;
  if ((rc = launch_flux(e, p, 0, U, U, nullptr, 0.0))) return rc;
  if (local_steps) k_imp_dtl<<<blocks, 128, 0, e->stream>>>(p, U, ccfl, dtl);
  k_imp_jac<<<blocks, 128, 0, e->stream>>>(p, U, dtl, dt, dinv, off);
  CK(cudaMemsetAsync(du[0], 0, (size_t)n * NV * 8, e->stream));
  int k = 0;
  for (int32_t sw = 0; sw < nsweeps; ++sw) {
    k_imp_sweep<<<blocks, 128, 0, e->stream>>>(p, dinv, off, du[k], du[k ^ 1], U2 ? U : nullptr, U2, U3, dt);
    k ^= 1;
  }
  e->launches += 2 + nsweeps;
  CK(cudaGetLastError());
  *cur = k;
  return UCG_OK;
}

int implicit_buffers(ucg_engine* e) {
  const int64_t n = e->n;
  int rc = UCG_OK;
  rc = rc ? rc : alloc(e, e->imp_dtl, (size_t)n * 8);
  rc = rc ? rc : alloc(e, e->imp_dinv, (size_t)n * 8);
  rc = rc ? rc : alloc(e, e->imp_off, (size_t)n * MF * NJ * 8);
  rc = rc ? rc : alloc(e, e->imp_du, (size_t)n * NV * 8 * 2);
  return rc;
}

}  // namespace

extern "C" int ucg_implicit_step(ucg_engine* e, double cfl, int32_t nsteps, int32_t nsweeps) {
  if (!e) return UCG_EINVAL;
  if (!(cfl > 0.0) || !std::isfinite(cfl) || nsteps < 0 || nsweeps < 1)
    return fail(e, UCG_EINVAL, "cfl > 0, nsteps >= 0 and nsweeps >= 1 are needed");
  if (!ready(e) || !e->have_state) return fail(e, UCG_ESTATE, "geometry, tables and state are needed");
  if (!e->roles.empty()) return fail(e, UCG_EINVAL, "implicit steps cover whole meshes (no partition roles)");
  cudaSetDevice(e->device);
  int rc = implicit_buffers(e);
  if (rc) return rc;
  Problem p = make_problem(e);
  double* U = (double*)e->Un.p;
  const unsigned blocks = (unsigned)((e->n + 127) / 128);
  for (int32_t s = 0; s < nsteps; ++s) {
    int cur;
    if ((rc = implicit_correction(e, p, U, cfl / 3.0, nsweeps, 0.0, nullptr, nullptr, &cur))) return rc;
    k_imp_add<<<blocks, 128, 0, e->stream>>>(p, U, (double*)e->imp_du.p + cur * e->n * NV);
    e->launches++;
    CK(cudaGetLastError());
  }
  return UCG_OK;
}

// DUAL_TIME (src/time_p.f90:3035-3243, RUNGEKUTTA = 11): one physical step
// dt of BDF2 by inner implicit iterations in pseudo time (local steps at
// `cfl`, formed once from the state at the start of the step, as
// CALCULATE_CFLL runs in the time loop before DUAL_TIME, :4104): the first
// without the time term in the right-hand side (ISCOUN
// 1), the others with it, each adding its correction, until the
// volume-weighted correction norm, relative to its largest value in this
// step, is at most inner_tol or max_inner iterations are done; then
// U^{n-1} <- U^n <- U.  The history starts from the state at the first
// call after ucg_set_state (IT = RESTART).
extern "C" int ucg_dual_time_step(ucg_engine* e, double dt, double cfl, int32_t max_inner, double inner_tol,
                                  int32_t nsweeps, int32_t* inner_iters) {
  if (!e) return UCG_EINVAL;
  if (!(dt > 0.0) || !std::isfinite(dt) || !(cfl > 0.0) || !std::isfinite(cfl) || max_inner < 1 || nsweeps < 1 ||
      !(inner_tol >= 0.0))
    return fail(e, UCG_EINVAL, "dt > 0, cfl > 0, max_inner >= 1, nsweeps >= 1 and inner_tol >= 0 are needed");
  if (!ready(e) || !e->have_state) return fail(e, UCG_ESTATE, "geometry, tables and state are needed");
  if (!e->roles.empty()) return fail(e, UCG_EINVAL, "implicit steps cover whole meshes (no partition roles)");
  cudaSetDevice(e->device);
  const int64_t n = e->n;
  int rc = implicit_buffers(e);
  rc = rc ? rc : alloc(e, e->dual_hist, (size_t)n * NV * 8 * 2);
  const int64_t nblk = (n + 255) / 256;
  rc = rc ? rc : alloc(e, e->dual_part, (size_t)(nblk + 1) * 8);
  if (rc) return rc;
  Problem p = make_problem(e);
  double* U = (double*)e->Un.p;
  double* U2 = (double*)e->dual_hist.p;
  double* U3 = U2 + n * NV;
  double* part = (double*)e->dual_part.p;
  if (!e->dual_ready) {
    CK(cudaMemcpyAsync(U2, U, (size_t)n * NV * 8, cudaMemcpyDeviceToDevice, e->stream));
    CK(cudaMemcpyAsync(U3, U, (size_t)n * NV * 8, cudaMemcpyDeviceToDevice, e->stream));
    e->dual_ready = true;
  }
  const unsigned blocks = (unsigned)((n + 127) / 128);
  k_imp_dtl<<<blocks, 128, 0, e->stream>>>(p, U, cfl / 3.0, (double*)e->imp_dtl.p);
  e->launches++;
  double firsti = 0.0;
  int32_t jj = 0;
  for (jj = 1; jj <= max_inner; ++jj) {
    int cur;
    if ((rc = implicit_correction(e, p, U, cfl / 3.0, nsweeps, dt, jj == 1 ? nullptr : U2, U3, &cur, false)))
      return rc;
    const double* du = (const double*)e->imp_du.p + cur * n * NV;
    k_imp_norm_part<<<(unsigned)nblk, 256, 0, e->stream>>>(p, du, part);
    k_imp_norm_sum<<<1, 1, 0, e->stream>>>(part, nblk, part + nblk);
    k_imp_add<<<blocks, 128, 0, e->stream>>>(p, U, du);
    e->launches += 3;
    double res = 0.0;
    CK(cudaMemcpyAsync(&res, part + nblk, 8, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    res = res / e->totvol;
    if (res > firsti) firsti = res;
    res = res / firsti;
    if (res <= inner_tol) break;
  }
  if (inner_iters) *inner_iters = jj > max_inner ? max_inner : jj;
  CK(cudaMemcpyAsync(U3, U2, (size_t)n * NV * 8, cudaMemcpyDeviceToDevice, e->stream));
  CK(cudaMemcpyAsync(U2, U, (size_t)n * NV * 8, cudaMemcpyDeviceToDevice, e->stream));
  return UCG_OK;
}

namespace {

// RELAXATION_EX (src/time_p.f90:3844-3888): per cell the explicit
// pseudo-time correction du = -(V/dt (1.5 U - 2 U^n + 0.5 U^{n-1}) + RHS)
// dtau, dtau = (DTL/V) / (1 + 1.5 DTL/dt), in the reference's order of
// operations
__global__ void k_dtex_du(Problem p, const double* __restrict__ U, const double* __restrict__ U2,
                          const double* __restrict__ U3, const double* __restrict__ dtl, double dt,
                          double* __restrict__ du) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  const double v = p.vol[c], dt1 = v / dt;
  const double dtau = (dtl[c] / v) * (1.0 / (1.0 + (1.5 * (dtl[c] / dt))));
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    const int64_t i = c * NV + k;
    const double imp = (dt1 * (((1.5 * U[i]) - (2.0 * U2[i])) + (0.5 * U3[i]))) + p.rhs[i];
    du[i] = (-imp) * dtau;
  }
}

// U^{n-1} <- U^n, U^n <- U, U <- 2 U^n - U^{n-1} (DUAL_TIME_EX, :3422-3430)
__global__ void k_dtex_rotate(int64_t m, double* __restrict__ U, double* __restrict__ U2, double* __restrict__ U3) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double u = U[i], u2 = U2[i];
  U3[i] = u2;
  U2[i] = u;
  U[i] = (2.0 * u) - u2;
}

}  // namespace

// DUAL_TIME_EX (src/time_p.f90:3244-3436, RUNGEKUTTA = 12): one physical
// step dt of BDF2 by explicit pseudo-time iterations (RELAXATION_EX; local
// steps at `cfl` formed once from the state at the start of the step), each
// adding its correction, until the volume-weighted correction norm,
// relative to its largest value in this step, is at most inner_tol or
// max_inner iterations are done; then U^{n-1} <- U^n <- U and the state
// becomes 2 U^n - U^{n-1}, the next step's first iterate.  The history is
// the one of ucg_dual_time_step (it starts from the state at the first call
// after ucg_set_state, IT = RESTART).
extern "C" int ucg_dual_time_step_explicit(ucg_engine* e, double dt, double cfl, int32_t max_inner, double inner_tol,
                                           int32_t* inner_iters) {
  if (!e) return UCG_EINVAL;
  if (!(dt > 0.0) || !std::isfinite(dt) || !(cfl > 0.0) || !std::isfinite(cfl) || max_inner < 1 ||
      !(inner_tol >= 0.0))
    return fail(e, UCG_EINVAL, "dt > 0, cfl > 0, max_inner >= 1 and inner_tol >= 0 are needed");
  if (!ready(e) || !e->have_state) return fail(e, UCG_ESTATE, "geometry, tables and state are needed");
  if (!e->roles.empty()) return fail(e, UCG_EINVAL, "dual time steps cover whole meshes (no partition roles)");
  cudaSetDevice(e->device);
  const int64_t n = e->n;
  int rc = implicit_buffers(e);
  rc = rc ? rc : alloc(e, e->dual_hist, (size_t)n * NV * 8 * 2);
  const int64_t nblk = (n + 255) / 256;
  rc = rc ? rc : alloc(e, e->dual_part, (size_t)(nblk + 1) * 8);
  if (rc) return rc;
  Problem p = make_problem(e);
  double* U = (double*)e->Un.p;
  double* U2 = (double*)e->dual_hist.p;
  double* U3 = U2 + n * NV;
  double* part = (double*)e->dual_part.p;
  double* dtl = (double*)e->imp_dtl.p;
  double* du = (double*)e->imp_du.p;
  if (!e->dual_ready) {
    CK(cudaMemcpyAsync(U2, U, (size_t)n * NV * 8, cudaMemcpyDeviceToDevice, e->stream));
    CK(cudaMemcpyAsync(U3, U, (size_t)n * NV * 8, cudaMemcpyDeviceToDevice, e->stream));
    e->dual_ready = true;
  }
  const unsigned blocks = (unsigned)((n + 127) / 128);
  k_imp_dtl<<<blocks, 128, 0, e->stream>>>(p, U, cfl / 3.0, dtl);
  e->launches++;
  double firsti = 0.0;
  int32_t jj = 0;
  for (jj = 1; jj <= max_inner; ++jj) {
    if ((rc = launch_recon(e, p, U))) return rc;
    if ((rc = launch_flux(e, p, 0, U, U, nullptr, 0.0))) return rc;
    k_dtex_du<<<blocks, 128, 0, e->stream>>>(p, U, U2, U3, dtl, dt, du);
    k_imp_norm_part<<<(unsigned)nblk, 256, 0, e->stream>>>(p, du, part);
    k_imp_norm_sum<<<1, 1, 0, e->stream>>>(part, nblk, part + nblk);
    k_imp_add<<<blocks, 128, 0, e->stream>>>(p, U, du);
    e->launches += 4;
    double res = 0.0;
    CK(cudaMemcpyAsync(&res, part + nblk, 8, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    res = res / e->totvol;
    if (res > firsti) firsti = res;
    res = res / firsti;
    if (res <= inner_tol) break;
  }
  if (inner_iters) *inner_iters = jj > max_inner ? max_inner : jj;
  const int64_t m = n * NV;
  k_dtex_rotate<<<(unsigned)((m + 255) / 256), 256, 0, e->stream>>>(m, U, U2, U3);
  e->launches++;
  CK(cudaGetLastError());
  return UCG_OK;
}
