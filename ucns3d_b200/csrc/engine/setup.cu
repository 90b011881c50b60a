// On-device set-up of the reconstruction tables (ucg_build_recon):
// PRESTORE_RECONSTRUCTION3 (src/prestore.f90:167-818) and INDICATORMATRIX
// (src/prestore.f90:1529-1673) as the host set-up library forms them
// (prep.cpp, build_tables): the same tetrahedra, points, weights and
// monomial order (../common/rules.h), the same operations in the same
// order.  This unit is compiled without fused multiply-adds (-fmad=false)
// and the host library without contraction, so every entry is the same
// IEEE double on both sides.
//
//   k_setup_mean   one thread per cell: the basis means (moments of the
//                  cell in its own frame over its volume)
//   k_setup_lsq    one warp per (matrix set, stencil): the moments of the
//                  stencil members (a lane per member), the normal matrix,
//                  Householder QR, R^-1 Q^T and the pseudo-inverse, in
//                  shared memory; every sum runs in the host's order on one
//                  lane, the lanes take different entries
//   k_setup_ind    one warp per matrix set: the smoothness matrices, point
//                  by point as the host accumulates them
// Both table kernels write the FP64 blocks that ucg_upload_recon stages
// (pseudo-inverses at Layout::soff, packed upper triangles), and the
// engine's expansion interleaves them on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../common/rules.h"
#include "engine_internal.h"
#include "expand.cuh"

using namespace ucg;
using namespace ucg_host;

namespace {

constexpr int MD = 34;  // monomials of degree 1..4 (IDEGFREE at IORDER 4)

struct SetupArgs {
  int64_t n;
  const int32_t* shape;   // [n] ISHAPE
  const double* vx;       // [n][8][3]
  const double* cen;      // [n][3]
  const double* vol;      // [n]
  const double* J;        // [n][9] INVCCJAC
  const double* fo;       // [n][3] frame origin
  const double* fdet;     // [n]
  const int32_t* sten;    // [n][A][W]
  const int32_t* admis;   // [n]
  const int64_t* rep;     // [ntab] the first cell of each matrix set
  const double* bm;       // [n][ideg] basis means (k_setup_mean)
  const double* rm;       // moment rule [nrm][4]: three coordinates, weight
  const double* ri;       // smoothness-matrix rule [nri][4]
  double period[3];
  int64_t tstride, istride;
  int A, W, ideg, imax, ideg2, imax2, cw, weno, nrm, nri, vec, i2off;
  int soff[8];
  int mono[MD][3];        // exponents, BASIS_REC order
  int nal, nal2;          // derivatives of INDICATORMATRIX for IORDER and (CWENO) the lower order
  int al[MD][3], al2[MD][3];
  int ntet[5];
  int tet[5][6][4];
  int* err;               // 1: a normal matrix is singular or its inverse not finite
};

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross3(D3 a, D3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 ld3(const double* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ D3 to_local(const double* J, D3 o, D3 x) {
  D3 r = x - o;
  return {J[0] * r.x + J[1] * r.y + J[2] * r.z, J[3] * r.x + J[4] * r.y + J[5] * r.z,
          J[6] * r.x + J[7] * r.y + J[8] * r.z};
}
__device__ __forceinline__ D3 wrap(const SetupArgs& a, D3 d) {
  if (a.period[0] > 0.0) d.x -= a.period[0] * rint(d.x / a.period[0]);
  if (a.period[1] > 0.0) d.y -= a.period[1] * rint(d.y / a.period[1]);
  if (a.period[2] > 0.0) d.z -= a.period[2] * rint(d.z / a.period[2]);
  return d;
}
__device__ __forceinline__ double ipow(double x, int e) {
  double r = 1.0;
  for (int i = 0; i < e; ++i) r *= x;
  return r;
}
// D^alpha of the monomial with exponents e at p
__device__ __forceinline__ double mono_deriv(const int* e, const int* al, D3 p) {
  double c = 1.0;
  int f[3];
  for (int k = 0; k < 3; ++k) {
    if (al[k] > e[k]) return 0.0;
    for (int j = 0; j < al[k]; ++j) c *= (double)(e[k] - j);
    f[k] = e[k] - al[k];
  }
  return c * ipow(p.x, f[0]) * ipow(p.y, f[1]) * ipow(p.z, f[2]);
}

// integral over cell y, moved by T, of each monomial in the frame (J, o):
// per tetrahedron of the cell and per rule point, out[d] += w vol m_d(x)
__device__ void cell_moments(const SetupArgs& a, int64_t y, D3 T, const double* J, D3 o, double (&out)[MD]) {
#pragma unroll
  for (int d = 0; d < MD; ++d) out[d] = 0.0;
  const int sh = a.shape[y];
  for (int k = 0; k < a.ntet[sh]; ++k) {
    D3 p[4];
    for (int j = 0; j < 4; ++j) p[j] = to_local(J, o, ld3(a.vx + (y * 8 + a.tet[sh][k][j]) * 3) + T);
    const double vol = fabs(dot3(p[1] - p[0], cross3(p[2] - p[0], p[3] - p[0])) / 6.0);
    for (int q = 0; q < a.nrm; ++q) {
      const double* r = a.rm + q * 4;
      const D3 x = p[0] + r[0] * (p[1] - p[0]) + r[1] * (p[2] - p[0]) + r[2] * (p[3] - p[0]);
      double px[8], py[8], pz[8];
      px[0] = py[0] = pz[0] = 1.0;
      for (int e = 1; e < 8; ++e) {
        px[e] = px[e - 1] * x.x;
        py[e] = py[e - 1] * x.y;
        pz[e] = pz[e - 1] * x.z;
      }
      const double wv = r[3] * vol;
#pragma unroll
      for (int d = 0; d < MD; ++d)
        if (d < a.ideg) out[d] += wv * (px[a.mono[d][0]] * py[a.mono[d][1]] * pz[a.mono[d][2]]);
    }
  }
}

__global__ void k_setup_mean(SetupArgs a, double* __restrict__ bm) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n) return;
  double mom[MD];
  cell_moments(a, c, D3{0.0, 0.0, 0.0}, a.J + c * 9, ld3(a.fo + c * 3), mom);
  const double vloc = a.vol[c] / fabs(a.fdet[c]);  // VOLUME(1,1)
  for (int d = 0; d < a.ideg; ++d) bm[c * a.ideg + d] = mom[d] / vloc;
}

__host__ __device__ inline size_t lsq_smem_doubles(int imax, int ideg) {
  return (size_t)imax * ideg + imax + 3 * (size_t)ideg * ideg + ideg;
}

// matrix set t0 + blockIdx.x, stencil blockIdx.y; 32 threads
__global__ void __launch_bounds__(32) k_setup_lsq(SetupArgs a, int64_t t0, double* __restrict__ out) {
  extern __shared__ double sm[];
  const int64_t t = t0 + blockIdx.x;
  const int64_t c = a.rep[t];
  const int ll = blockIdx.y, lane = threadIdx.x;
  if (ll >= a.admis[c]) return;  // rows of inadmissible stencils stay zero
  const bool low = a.cw && ll > 0;
  const int nd = low ? a.ideg2 : a.ideg, nk = low ? a.imax2 : a.imax, n = nd;
  double* Am = sm;                          // [nk][nd]
  double* vl = Am + (size_t)a.imax * a.ideg;  // [nk]
  double* N = vl + a.imax;                  // [nd][nd]: normal matrix, then R, then the inverse
  double* Q = N + (size_t)a.ideg * a.ideg;  // [nd][nd]
  double* Ri = Q + (size_t)a.ideg * a.ideg; // [nd][nd]
  double* v = Ri + (size_t)a.ideg * a.ideg; // [nd]
  const double* J = a.J + c * 9;
  const D3 o = ld3(a.fo + c * 3), cc = ld3(a.cen + c * 3);
  const double absdet = fabs(a.fdet[c]);
  // ---- rows of the least-squares matrix: moments of each member minus
  // its volume times the cell's basis means
  for (int k = lane; k < nk; k += 32) {
    const int64_t y = a.sten[(c * a.A + ll) * a.W + k + 1];
    const D3 d = ld3(a.cen + y * 3) - cc;
    const D3 T = wrap(a, d) - d;
    double mom[MD];
    cell_moments(a, y, T, J, o, mom);
    const double vloc = a.vol[y] / absdet;  // ILOX_VOLUME
    vl[k] = vloc;
#pragma unroll
    for (int e = 0; e < MD; ++e)
      if (e < nd) Am[k * nd + e] = mom[e] - vloc * a.bm[c * a.ideg + e];
  }
  __syncthreads();
  // ---- normal matrix
  for (int i = lane; i < n * n; i += 32) {
    const int r = i / n, s = i - r * n;
    double acc = 0.0;
    for (int k = 0; k < nk; ++k) acc += Am[k * nd + r] * Am[k * nd + s];
    N[i] = acc;
  }
  for (int i = lane; i < n * n; i += 32) Q[i] = (i / n == i % n) ? 1.0 : 0.0;
  __syncthreads();
  // ---- Householder QR of N (columns and rows of Q split over the lanes)
  for (int k = 0; k < n - 1; ++k) {
    __syncthreads();  // the previous step's reads of v are done
    double nrm = 0.0;
    for (int i = k; i < n; ++i) nrm += N[i * n + k] * N[i * n + k];
    nrm = sqrt(nrm);
    if (nrm == 0.0) continue;
    const double alpha = N[k * n + k] > 0 ? -nrm : nrm;
    for (int i = lane; i < n; i += 32) v[i] = i < k ? 0.0 : (i == k ? N[i * n + k] - alpha : N[i * n + k]);
    __syncthreads();
    double vn = 0.0;
    for (int i = k; i < n; ++i) vn += v[i] * v[i];
    if (vn == 0.0) continue;
    for (int j = lane; j < n; j += 32) {
      double s = 0.0;
      for (int i = k; i < n; ++i) s += v[i] * N[i * n + j];
      s = 2.0 * s / vn;
      for (int i = k; i < n; ++i) N[i * n + j] -= s * v[i];
    }
    for (int i = lane; i < n; i += 32) {
      double s = 0.0;
      for (int j = k; j < n; ++j) s += Q[i * n + j] * v[j];
      s = 2.0 * s / vn;
      for (int j = k; j < n; ++j) Q[i * n + j] -= s * v[j];
    }
    __syncthreads();
  }
  // ---- R^-1, row by row from the last
  __syncthreads();
  for (int i = lane; i < n * n; i += 32) Ri[i] = 0.0;
  __syncthreads();
  for (int i = n - 1; i >= 0; --i) {
    const double rii = N[i * n + i];
    if (rii == 0.0) {
      if (lane == 0) atomicOr(a.err, 1);
      return;
    }
    if (lane == 0) Ri[i * n + i] = 1.0 / rii;
    for (int j = i + 1 + lane; j < n; j += 32) {
      double s = 0.0;
      for (int k = i + 1; k <= j; ++k) s += N[i * n + k] * Ri[k * n + j];
      Ri[i * n + j] = -s / rii;
    }
    __syncthreads();
  }
  // ---- inverse R^-1 Q^T (into N)
  for (int i = lane; i < n * n; i += 32) {
    const int r = i / n, s = i - r * n;
    double acc = 0.0;
    for (int k = r; k < n; ++k) acc += Ri[r * n + k] * Q[s * n + k];
    N[i] = acc;
    if (!isfinite(acc)) atomicOr(a.err, 1);
  }
  __syncthreads();
  // ---- pseudo-inverse rows, column-scaled by the member volumes
  double* o_t = out + (t - t0) * a.tstride + a.soff[ll];
  for (int i = lane; i < nk * nd; i += 32) {
    const int k = i / nd, d = i - k * nd;
    double acc = 0.0;
    for (int e = 0; e < nd; ++e) acc += N[d * nd + e] * Am[k * nd + e];
    o_t[i] = acc * vl[k];
  }
}

// smoothness matrix of order (al, nal) over n monomials of cell c, packed
// as ucg_upload_recon packs it (upper triangle, off-diagonal S_de + S_ed,
// rows padded to a.vec) at dst
__device__ void indicator(const SetupArgs& a, int64_t c, int n, const int (*al)[3], int nal, double* D, double* S,
                          double* dst) {
  const int lane = threadIdx.x;
  const double* J = a.J + c * 9;
  const D3 o = ld3(a.fo + c * 3);
  for (int i = lane; i < n * n; i += 32) S[i] = 0.0;
  __syncthreads();
  const int sh = a.shape[c];
  for (int k = 0; k < a.ntet[sh]; ++k) {
    D3 p[4];
    for (int j = 0; j < 4; ++j) p[j] = to_local(J, o, ld3(a.vx + (c * 8 + a.tet[sh][k][j]) * 3));
    const double vol = fabs(dot3(p[1] - p[0], cross3(p[2] - p[0], p[3] - p[0])) / 6.0);
    for (int q = 0; q < a.nri; ++q) {
      const double* r = a.ri + q * 4;
      const D3 x = p[0] + r[0] * (p[1] - p[0]) + r[1] * (p[2] - p[0]) + r[2] * (p[3] - p[0]);
      for (int i = lane; i < nal * n; i += 32) {
        const int g = i / n, d = i - g * n;
        D[i] = mono_deriv(a.mono[d], al[g], x);
      }
      __syncthreads();
      const double wv = r[3] * vol;
      for (int i = lane; i < n * n; i += 32) {
        const int r1 = i / n, r2 = i - r1 * n;
        double sacc = 0.0;
        for (int g = 0; g < nal; ++g) sacc += D[g * n + r1] * D[g * n + r2];
        S[i] += wv * sacc;
      }
      __syncthreads();
    }
  }
  if (lane == 0) {
    int j = 0;
    for (int d = 0; d < n; ++d) {
      for (int k = d; k < n; ++k) dst[j + k - d] = k == d ? S[d * n + d] : S[d * n + k] + S[k * n + d];
      j += (n - d + a.vec - 1) / a.vec * a.vec;
    }
  }
  __syncthreads();
}

// matrix set t0 + blockIdx.x; 32 threads
__global__ void __launch_bounds__(32) k_setup_ind(SetupArgs a, int64_t t0, double* __restrict__ out) {
  __shared__ double D[MD * MD], S[MD * MD];
  const int64_t t = t0 + blockIdx.x;
  const int64_t c = a.rep[t];
  double* dst = out + (t - t0) * a.istride;
  indicator(a, c, a.ideg, a.al, a.nal, D, S, dst);
  if (a.cw) indicator(a, c, a.ideg2, a.al2, a.nal2, D, S, dst + a.i2off);
}

template <typename T>
int upload_vec(ucg_engine* e, DevBuf& b, const T* src, size_t count) {
  int rc = alloc(e, b, count * sizeof(T));
  if (rc) return rc;
  CK(cudaMemcpyAsync(b.p, src, count * sizeof(T), cudaMemcpyHostToDevice, e->stream));
  return UCG_OK;
}

void free_all(ucg_engine* e, std::vector<DevBuf*> bufs) {
  for (DevBuf* b : bufs) {
    if (b->p) {
      cudaFree(b->p);
      e->bytes -= (int64_t)b->bytes;
    }
    b->p = nullptr;
    b->bytes = 0;
  }
}

}  // namespace

int ucg_build_recon(ucg_engine* e, const ucg_shapes* s, const ucg_recon* r) {
  if (!e || !s || !r) return fail(e, UCG_EINVAL, "null argument");
  const ucg_config& c = e->cfg;
  const int64_t n = e->n;
  if (s->ncells != n || r->first != 0 || r->count != n)
    return fail(e, UCG_EINVAL, "ucg_build_recon takes every cell (first 0, count n)");
  if (!s->shape || !s->vertices || !s->centre || !s->volume || !s->frame || !s->frame_origin || !s->frame_det ||
      !r->stencil)
    return fail(e, UCG_EINVAL, "a shape array or the stencils are NULL");
  if (!e->have_geometry) return fail(e, UCG_ESTATE, "upload the geometry before building the tables");
  if (c.ideg > MD || c.admis_max > 8) return fail(e, UCG_EINVAL, "unsupported sizes");
  for (int64_t i = 0; i < n; ++i)
    if (s->shape[i] < 1 || s->shape[i] > 4) return fail(e, UCG_EINVAL, "shape code out of range at cell " + std::to_string(i));
  for (int k = 0; k < 3; ++k)
    if (!(s->period[k] >= 0.0) || !std::isfinite(s->period[k])) return fail(e, UCG_EINVAL, "bad period");
  const int64_t ntab = r->table_id ? r->ntables : n;
  std::vector<int64_t> rep((size_t)std::max<int64_t>(ntab, 0), -1);
  if (r->table_id) {
    if (ntab <= 0) return fail(e, UCG_EINVAL, "ntables must be positive with table_id");
    for (int64_t i = 0; i < n; ++i) {
      const int32_t t = r->table_id[i];
      if (t < 0 || t >= ntab) return fail(e, UCG_EINVAL, "table_id out of range");
      if (rep[t] < 0) rep[t] = i;
    }
    for (int64_t t = 0; t < ntab; ++t)
      if (rep[t] < 0) return fail(e, UCG_EINVAL, "a matrix set no cell uses");
  } else {
    for (int64_t i = 0; i < n; ++i) rep[i] = i;
  }
  cudaSetDevice(e->device);
  DevBuf rowbuf;
  const int32_t* d_rowmap = nullptr;
  int rc = upload_stencils(e, 0, n, r->stencil, rowbuf, &d_rowmap);
  if (rc) {
    release(rowbuf);
    return rc;
  }
  // ---- arguments: shapes, stencils and ADMIS in the caller's order
  const int A = c.admis_max, W = c.imax + 1;
  SetupArgs a{};
  a.n = n;
  a.A = A;
  a.W = W;
  a.ideg = c.ideg;
  a.imax = c.imax;
  a.ideg2 = c.ideg2;
  a.imax2 = c.imax2;
  a.cw = c.ees == 5;
  a.weno = c.scheme == 3;
  a.vec = e->mixed ? 4 : 2;
  a.tstride = e->layout.tstride;
  a.istride = e->layout.istride;
  a.i2off = e->layout.i2off;
  for (int k = 0; k < 8; ++k) a.soff[k] = e->layout.soff[k];
  for (int k = 0; k < 3; ++k) a.period[k] = s->period[k];
  const std::vector<ucrules::Mono> mono = ucrules::monomials(c.iorder);
  for (size_t d = 0; d < mono.size() && d < (size_t)MD; ++d)
    for (int k = 0; k < 3; ++k) a.mono[d][k] = mono[d].e[k];
  // INDICATORMATRIX: every derivative of orders 1..order, in the monomials' order
  const int order2 = c.ideg2 == 9 ? 2 : 1;
  const std::vector<ucrules::Mono> al = ucrules::monomials(c.iorder), al2 = ucrules::monomials(order2);
  a.nal = (int)al.size();
  a.nal2 = a.cw ? (int)al2.size() : 0;
  for (int g = 0; g < a.nal; ++g)
    for (int k = 0; k < 3; ++k) a.al[g][k] = al[g].e[k];
  for (int g = 0; g < a.nal2; ++g)
    for (int k = 0; k < 3; ++k) a.al2[g][k] = al2[g].e[k];
  for (int sh = 1; sh <= 4; ++sh) {
    const ucrules::Topo& tp = ucrules::topo(sh);
    a.ntet[sh] = tp.ntet;
    for (int k = 0; k < tp.ntet; ++k)
      for (int j = 0; j < 4; ++j) a.tet[sh][k][j] = tp.tet[k][j];
  }
  // the host set-up's rules: moments and smoothness matrices
  auto flat = [](const ucrules::TetRule& R) {
    std::vector<double> f(R.w.size() * 4);
    for (size_t q = 0; q < R.w.size(); ++q) {
      for (int k = 0; k < 3; ++k) f[q * 4 + k] = R.p[q][k];
      f[q * 4 + 3] = R.w[q];
    }
    return f;
  };
  const std::vector<double> rmf = flat(ucrules::tet_rule(std::max(2, (c.iorder + 4) / 2)));
  const std::vector<double> rif = flat(ucrules::tet_rule(std::max(2, (2 * c.iorder + 2) / 2 + 1)));
  a.nrm = (int)(rmf.size() / 4);
  a.nri = (int)(rif.size() / 4);
  std::vector<int32_t> admis_c((size_t)n);
  for (int64_t i = 0; i < n; ++i) admis_c[i] = e->admis_h[e->o2n.empty() ? i : e->o2n[i]];
  DevBuf b_shape, b_vx, b_cen, b_vol, b_J, b_fo, b_fd, b_sten, b_adm, b_rep, b_bm, b_rm, b_ri, b_err;
  std::vector<DevBuf*> tmp = {&b_shape, &b_vx, &b_cen, &b_vol, &b_J, &b_fo, &b_fd, &b_sten, &b_adm, &b_rep,
                              &b_bm, &b_rm, &b_ri, &b_err};
  auto bail = [&](int code) {
    free_all(e, tmp);
    release(rowbuf);
    return code;
  };
  if ((rc = upload_vec(e, b_shape, s->shape, n)) || (rc = upload_vec(e, b_vx, s->vertices, n * 24)) ||
      (rc = upload_vec(e, b_cen, s->centre, n * 3)) || (rc = upload_vec(e, b_vol, s->volume, n)) ||
      (rc = upload_vec(e, b_J, s->frame, n * 9)) || (rc = upload_vec(e, b_fo, s->frame_origin, n * 3)) ||
      (rc = upload_vec(e, b_fd, s->frame_det, n)) || (rc = upload_vec(e, b_sten, r->stencil, (size_t)n * A * W)) ||
      (rc = upload_vec(e, b_adm, admis_c.data(), n)) || (rc = upload_vec(e, b_rep, rep.data(), ntab)) ||
      (rc = upload_vec(e, b_rm, rmf.data(), rmf.size())) || (rc = upload_vec(e, b_ri, rif.data(), rif.size())) ||
      (rc = alloc(e, b_bm, (size_t)n * c.ideg * 8)) || (rc = alloc(e, b_err, 4)))
    return bail(rc);
  if (cudaMemsetAsync(b_err.p, 0, 4, e->stream) != cudaSuccess) return bail(cuda_fail(e, cudaGetLastError(), "memset"));
  a.shape = (const int32_t*)b_shape.p;
  a.vx = (const double*)b_vx.p;
  a.cen = (const double*)b_cen.p;
  a.vol = (const double*)b_vol.p;
  a.J = (const double*)b_J.p;
  a.fo = (const double*)b_fo.p;
  a.fdet = (const double*)b_fd.p;
  a.sten = (const int32_t*)b_sten.p;
  a.admis = (const int32_t*)b_adm.p;
  a.rep = (const int64_t*)b_rep.p;
  a.bm = (const double*)b_bm.p;
  a.rm = (const double*)b_rm.p;
  a.ri = (const double*)b_ri.p;
  a.err = (int*)b_err.p;
  // ---- basis means of every cell, into the engine's interleaved copy
  k_setup_mean<<<(unsigned)((n + 127) / 128), 128, 0, e->stream>>>(a, (double*)b_bm.p);
  e->launches++;
  {
    const int64_t total = n * c.ideg;
    const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, 148 * 64);
    if (e->mixed)
      k_expand_il<float, double, 1><<<blocks, 256, 0, e->stream>>>((float*)e->bmean.p, (const double*)b_bm.p, nullptr, 0,
                                                                  n, c.ideg, 0, n, d_rowmap, n);
    else
      k_expand_il<double, double, 1><<<blocks, 256, 0, e->stream>>>((double*)e->bmean.p, (const double*)b_bm.p, nullptr,
                                                                   0, n, c.ideg, 0, n, d_rowmap, n);
    e->launches++;
  }
  if (cudaGetLastError() != cudaSuccess) return bail(cuda_fail(e, cudaErrorLaunchFailure, "k_setup_mean"));
  // ---- matrix sets, staged and expanded like uploaded ones
  const size_t lsq_smem = lsq_smem_doubles(c.imax, c.ideg) * 8;
  if (cudaFuncSetAttribute(k_setup_lsq, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsq_smem) != cudaSuccess)
    return bail(cuda_fail(e, cudaGetLastError(), "cudaFuncSetAttribute"));
  DevBuf tidbuf;
  if (r->table_id) {
    if ((rc = upload_vec(e, tidbuf, r->table_id, n))) return bail(rc);
    tmp.push_back(&tidbuf);
  }
  rc = expand_tables(e, 0, n, ntab, (const int32_t*)tidbuf.p, d_rowmap,
                     [&](int which, int64_t t0, int64_t t1, double* dev) {
                       const int64_t len = which == 0 ? a.tstride : a.istride;
                       CK(cudaMemsetAsync(dev, 0, (size_t)(t1 - t0) * len * 8, e->stream));
                       if (which == 0)
                         k_setup_lsq<<<dim3((unsigned)(t1 - t0), (unsigned)A), 32, lsq_smem, e->stream>>>(a, t0, dev);
                       else
                         k_setup_ind<<<(unsigned)(t1 - t0), 32, 0, e->stream>>>(a, t0, dev);
                       e->launches++;
                       CK(cudaGetLastError());
                       return (int)UCG_OK;
                     });
  if (rc) return bail(rc);
  int err = 0;
  if (cudaMemcpy(&err, b_err.p, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return bail(cuda_fail(e, cudaGetLastError(), "cudaMemcpy"));
  bail(UCG_OK);
  if (err) return fail(e, UCG_EINVAL, "singular least-squares normal matrix");
  mark_recon(e, 0, n);
  return UCG_OK;
}
