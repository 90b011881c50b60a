// Reconstruction for WENO / CWENO / high-order MUSCL in two kernels.
//
// k_lsq      LEAST_SQUARES (src/gradients.f90:253-497): one lane per cell.
//            Tables are interleaved over groups of 32 cells, so every table
//            load of a warp is one contiguous 128/256-byte row; each gathered
//            difference U_k - U_i is reused across DH rows held in registers.
//            Output: the stencil polynomials G[ll][d][v], interleaved.
// k_wpost    CP_RECONSTRUCTION (src/reconstruct_p.f90:920-1250), CHECKSOL,
//            MUSCL fall-back, CHECKSOLX (3126-3406): a block reconstructs
//            `cpc` cells cooperatively in shared memory.
#pragma once

#include "device.cuh"

namespace ucg {

// Tuning of k_lsq (compile-time): rows of G held in registers per pass for
// IORDER 4/3 in FP32/FP64, software pipelining of the index/state chain,
// minimum resident blocks per SM for the register budget.
#ifndef UCG_LSQ_ROWS_P4F
#define UCG_LSQ_ROWS_P4F 17
#endif
#ifndef UCG_LSQ_ROWS_P4D
#define UCG_LSQ_ROWS_P4D 12
#endif
#ifndef UCG_LSQ_ROWS_P3F
#define UCG_LSQ_ROWS_P3F 19
#endif
#ifndef UCG_LSQ_ROWS_P3D
#define UCG_LSQ_ROWS_P3D 10
#endif
#ifndef UCG_LSQ_PIPE
#define UCG_LSQ_PIPE 0
#endif
#ifndef UCG_LSQ_MINB
#define UCG_LSQ_MINB 1
#endif
// 1: k_lsq_bulk (tables streamed through shared memory), 0: k_lsq
#ifndef UCG_LSQ_BULK
#define UCG_LSQ_BULK 1
#endif

// rows of G held in registers per pass
template <int P, typename T>
struct LsqRows {
  static constexpr int ID = Deg<P>::ideg;
  static constexpr int value = P == 4   ? (sizeof(T) == 4 ? UCG_LSQ_ROWS_P4F : UCG_LSQ_ROWS_P4D)
                               : P == 3 ? (sizeof(T) == 4 ? UCG_LSQ_ROWS_P3F : UCG_LSQ_ROWS_P3D)
                                        : ID;
};

template <int P, typename T>
__global__ void __launch_bounds__(128, UCG_LSQ_MINB) k_lsq(Problem p, const double* __restrict__ U) {
  constexpr int ID = Deg<P>::ideg;
  constexpr int DH = LsqRows<P, T>::value;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int A = p.admis_max, W = p.imax + 1;
  const bool cw = p.ees == 5;
  const int64_t grp = c >> 5;
  const int lane = (int)(c & 31);
  const bool live = c < p.n;
  const int adm = live ? p.admis[c] : 0;
  double u0[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u0[v] = live ? U[c * NV + v] : 0.0;
  const T* Mi = (const T*)p.invmat + grp * p.tstride * 32 + lane;
  const int32_t* Si = p.sten + grp * (int64_t)(A * W) * 32 + lane;
  T* Gi = (T*)p.gbuf + grp * (int64_t)(A * ID * NV) * 32 + lane;
  for (int ll = 0; ll < A; ++ll) {
    const bool low = cw && ll > 0;
    const int nk = low ? p.imax2 : p.imax, nd = low ? p.ideg2 : ID;
    const bool act = ll < adm;
    for (int d0 = 0; d0 < nd; d0 += DH) {
      T acc[DH][NV];
#pragma unroll
      for (int j = 0; j < DH; ++j)
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[j][v] = T(0);
      if (act) {
        const T* M = Mi + (int64_t)(p.soff[ll] + d0) * 32;
        const int32_t* S = Si + (ll * W + 1) * 32;
#if UCG_LSQ_PIPE
        // software pipeline of the dependent chain index -> state -> FMA:
        // indices two rows ahead, neighbour state one row ahead
        int y1 = nk > 1 ? S[32] : 0;
        double ua[NV];
        {
          const double* uy = U + (int64_t)S[0] * NV;
#pragma unroll
          for (int v = 0; v < NV; ++v) ua[v] = uy[v];
        }
        for (int k = 0; k < nk; ++k) {
          const int y2 = k + 2 < nk ? S[(k + 2) * 32] : 0;
          double ub[NV];
          const double* un = U + (int64_t)y1 * NV;
#pragma unroll
          for (int v = 0; v < NV; ++v) ub[v] = k + 1 < nk ? un[v] : 0.0;
          T du[NV];
#pragma unroll
          for (int v = 0; v < NV; ++v) du[v] = T(ua[v] - u0[v]);
          const T* Mk = M + (int64_t)k * nd * 32;
#pragma unroll
          for (int j = 0; j < DH; ++j)
            if (d0 + j < nd) {
              T m = Mk[j * 32];
#pragma unroll
              for (int v = 0; v < NV; ++v) acc[j][v] += m * du[v];
            }
#pragma unroll
          for (int v = 0; v < NV; ++v) ua[v] = ub[v];
          y1 = y2;
        }
      }
#else
#pragma unroll 2
        for (int k = 0; k < nk; ++k) {
          const double* uy = U + (int64_t)S[k * 32] * NV;
          T du[NV];
#pragma unroll
          for (int v = 0; v < NV; ++v) du[v] = T(uy[v] - u0[v]);
          const T* Mk = M + (int64_t)k * nd * 32;
#pragma unroll
          for (int j = 0; j < DH; ++j)
            if (d0 + j < nd) {
              T m = Mk[j * 32];
#pragma unroll
              for (int v = 0; v < NV; ++v) acc[j][v] += m * du[v];
            }
        }
      }
#endif
      if (live)
#pragma unroll
        for (int j = 0; j < DH; ++j)
          if (d0 + j < nd)
#pragma unroll
            for (int v = 0; v < NV; ++v) Gi[(int64_t)((ll * ID + d0 + j) * NV + v) * 32] = acc[j][v];
    }
  }
}

// ------------------------------------------------------------- k_lsq_bulk
// The same product G = invmat * (U_k - U_i) with the pseudo-inverse rows
// streamed through shared memory.  Each warp owns one 32-cell group; lane 0
// keeps `stages` chunks of bulk copies in flight (table rows and stencil
// indices), so the DRAM requests outstanding per SM do not depend on the
// register budget.  A chunk is KR stencil rows x dc columns [d0, d0+dc) of
// stencil ll; LsqBulk<P,T>::DH columns are accumulated in registers over all
// rows of a stencil.  The neighbour states of chunk i+1 are gathered while
// chunk i is multiplied.  No block-wide barrier: warps run independently.
template <int P, typename T>
struct LsqBulk {
  static constexpr int ID = Deg<P>::ideg;
  // columns per pass: 170 accumulator registers at most
  static constexpr int DH = sizeof(T) == 4 ? (ID <= 34 ? ID : 34) : (ID <= 17 ? ID : (ID + 1) / 2);
  static constexpr int KR = 2;  // stencil rows per chunk
  static constexpr int stage_bytes = KR * DH * 32 * (int)sizeof(T) + KR * 128;
};

struct LsqBulkPlan {
  int nw;      // warps (32-cell groups) per block
  int stages;  // chunks in flight per warp
  int total;   // dynamic shared memory per block
};

template <int P, typename T>
LsqBulkPlan lsq_bulk_plan(int nw) {
  constexpr int sb = LsqBulk<P, T>::stage_bytes;
  int st = 36 * 1024 / sb;
  st = st < 3 ? 3 : (st > 16 ? 16 : st);
  return LsqBulkPlan{nw, st, nw * st * (sb + 8)};
}

struct LsqChunk {
  int ll, d0, k0;
};

template <int P, typename T>
__global__ void __launch_bounds__(96, 2) k_lsq_bulk(Problem p, const double* __restrict__ U, LsqBulkPlan pl) {
  using B = LsqBulk<P, T>;
  constexpr int ID = B::ID, DH = B::DH, KR = B::KR, SB = B::stage_bytes;
  extern __shared__ __align__(128) unsigned char smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t grp = (int64_t)blockIdx.x * pl.nw + w;
  if (grp * 32 >= p.n) return;  // warp-uniform
  const int S = pl.stages;
  unsigned char* stage0 = smem + (size_t)w * S * SB;
  uint64_t* bar = (uint64_t*)(smem + (size_t)pl.nw * S * SB) + w * S;
  const int A = p.admis_max, W = p.imax + 1;
  const bool cw = p.ees == 5;
  const int64_t c = grp * 32 + lane;
  const bool live = c < p.n;
  const int adm = live ? p.admis[c] : 0;
  const int amax = __reduce_max_sync(0xffffffffu, adm);  // stencils any lane of the group uses
  const T* Mg = (const T*)p.invmat + grp * p.tstride * 32;
  const int32_t* Sg = p.sten + grp * (int64_t)(A * W) * 32;
  T* Gi = (T*)p.gbuf + grp * (int64_t)(A * ID * NV) * 32 + lane;
  auto nk_of = [&](int ll) { return cw && ll > 0 ? p.imax2 : p.imax; };
  auto nd_of = [&](int ll) { return cw && ll > 0 ? p.ideg2 : ID; };
  auto next = [&](LsqChunk& q) {
    q.k0 += KR;
    if (q.k0 >= nk_of(q.ll)) {
      q.k0 = 0;
      q.d0 += DH;
      if (q.d0 >= nd_of(q.ll)) {
        q.d0 = 0;
        ++q.ll;
      }
    }
  };
  // lane 0: copy chunk q into stage s
  auto issue = [&](const LsqChunk& q, int s) {
    const int nk = nk_of(q.ll), nd = nd_of(q.ll);
    const int kc = min(KR, nk - q.k0), dc = min(DH, nd - q.d0);
    unsigned char* st = stage0 + (size_t)s * SB;
    T* tab = (T*)st;
    int32_t* idx = (int32_t*)(st + KR * DH * 32 * sizeof(T));
    const T* M = Mg + (int64_t)p.soff[q.ll] * 32;
    mbar_expect_tx(&bar[s], (unsigned)(kc * dc * 32 * sizeof(T) + kc * 128));
    if (dc == nd) {
      bulk_g2s(tab, M + (int64_t)q.k0 * nd * 32, (unsigned)(kc * nd * 32 * sizeof(T)), &bar[s]);
    } else {
      for (int r = 0; r < kc; ++r)
        bulk_g2s(tab + r * dc * 32, M + ((int64_t)(q.k0 + r) * nd + q.d0) * 32, (unsigned)(dc * 32 * sizeof(T)),
                 &bar[s]);
    }
    bulk_g2s(idx, Sg + (int64_t)(q.ll * W + 1 + q.k0) * 32, (unsigned)(kc * 128), &bar[s]);
  };
  if (lane == 0)
    for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
  mbar_fence_init();
  __syncwarp();

  double u0[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u0[v] = live ? U[c * NV + v] : 0.0;

  // chunk indices: waited < issued; chunk i lives in stage i % S
  int64_t issued = 0, waited = 0;
  LsqChunk prod{0, 0, 0};
  for (int s = 0; s < S && prod.ll < amax; ++s) {
    if (lane == 0) issue(prod, s);
    next(prod);
    ++issued;
  }
  bool ok = true;
  auto wait_chunk = [&](int64_t i) {
    const bool r = __all_sync(0xffffffffu, mbar_wait(&bar[i % S], (unsigned)((i / S) & 1)));
    ok = ok && r;
    if (r) waited = i + 1;
  };

  LsqChunk cur{0, 0, 0};
  double un[KR][NV];  // neighbour states of the current chunk
  // gather the rows of chunk q (its indices are in stage s)
  auto gather = [&](const LsqChunk& q, int s) {
    const int kc = min(KR, nk_of(q.ll) - q.k0);
    const bool act = q.ll < adm;
    const int32_t* idx = (const int32_t*)(stage0 + (size_t)s * SB + KR * DH * 32 * sizeof(T));
#pragma unroll
    for (int r = 0; r < KR; ++r) {
      const bool on = act && r < kc;
      const int y = on ? idx[r * 32 + lane] : 0;
#pragma unroll
      for (int v = 0; v < NV; ++v) un[r][v] = on ? U[(int64_t)y * NV + v] : 0.0;
    }
  };
  if (issued > 0) {
    wait_chunk(0);
    if (ok) gather(cur, 0);
  }
  T acc[DH][NV];
#pragma unroll
  for (int j = 0; j < DH; ++j)
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[j][v] = T(0);

  for (int64_t i = 0; ok && cur.ll < amax; ++i) {
    const int s = (int)(i % S);
    const int nk = nk_of(cur.ll), nd = nd_of(cur.ll);
    const int kc = min(KR, nk - cur.k0), dc = min(DH, nd - cur.d0);
    const bool act = cur.ll < adm;
    T du[KR][NV];
#pragma unroll
    for (int r = 0; r < KR; ++r)
#pragma unroll
      for (int v = 0; v < NV; ++v) du[r][v] = T(un[r][v] - u0[v]);
    // start the gathers of the next chunk
    LsqChunk nx = cur;
    next(nx);
    if (nx.ll < amax) {
      wait_chunk(i + 1);
      if (!ok) break;
      gather(nx, (int)((i + 1) % S));
    }
    const T* tab = (const T*)(stage0 + (size_t)s * SB);
    if (act) {
#pragma unroll
      for (int r = 0; r < KR; ++r)
        if (r < kc) {
#pragma unroll
          for (int j = 0; j < DH; ++j)
            if (j < dc) {
              const T m = tab[(r * dc + j) * 32 + lane];
#pragma unroll
              for (int v = 0; v < NV; ++v) acc[j][v] += m * du[r][v];
            }
        }
    }
    if (cur.k0 + kc >= nk) {  // last rows of this column pass: write G
      if (live)
#pragma unroll
        for (int j = 0; j < DH; ++j)
          if (j < dc)
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              Gi[(int64_t)((cur.ll * ID + cur.d0 + j) * NV + v) * 32] = acc[j][v];
              acc[j][v] = T(0);
            }
    }
    // stage s is free again: refill it with chunk i + S
    __syncwarp();
    if (prod.ll < amax) {
      if (lane == 0) {
        fence_proxy_async();
        issue(prod, s);
      }
      next(prod);
      ++issued;
    }
    cur = nx;
  }
  if (!ok) {
    // record the timeout and let the copies in flight land before leaving
    if (lane == 0) atomicOr(p.health, HEALTH_TIMEOUT);
    for (int64_t i = waited; i < issued; ++i) mbar_wait(&bar[i % S], (unsigned)((i / S) & 1));
    return;
  }
  // stencils no lane of the group uses
  if (live)
    for (int ll = amax; ll < A; ++ll)
      for (int j = 0; j < nd_of(ll); ++j)
#pragma unroll
        for (int v = 0; v < NV; ++v) Gi[(int64_t)((ll * ID + j) * NV + v) * 32] = T(0);
}

}  // namespace ucg

namespace ucg {

struct WPPlan {
  int cpc;
  int o_G, o_g1, o_S, o_tmp, o_gh, o_w, o_dul, o_u0, o_bnd, o_slope, o_flag, total;
};

template <typename T>
inline WPPlan wpost_plan(int cpc, int A, int ID, int ID2, int QS, bool cw, int istride) {
  WPPlan w{};
  w.cpc = cpc;
  const int s = (int)sizeof(T);
  int off = 0;
  auto take = [&](int bytes) {
    int o = off;
    off += (bytes + 15) / 16 * 16;
    return o;
  };
  w.o_G = take(cpc * A * ID * NV * s);
  w.o_g1 = take(cw ? cpc * ID * NV * s : 0);
  w.o_S = take(cpc * istride * s);
  int tmp = cpc * A * ID * NV * s, psi = cpc * MF * QS * NV * 8;
  w.o_tmp = take(tmp > psi ? tmp : psi);  // indicator partials, later the limiter values
  w.o_gh = take(cpc * ID * NV * s);
  w.o_w = take(cpc * A * NV * 8);
  w.o_dul = take(cpc * MF * QS * NV * s);
  w.o_u0 = take(cpc * NV * 8);
  w.o_bnd = take(cpc * 2 * NV * 8);
  w.o_slope = take(cpc * NV * 8);
  w.o_flag = take(cpc * 2 * 4);
  w.total = off;
  return w;
}

template <int P, typename T>
__global__ void __launch_bounds__(256) k_wpost(Problem p, const double* __restrict__ U, WPPlan w) {
  constexpr int ID = Deg<P>::ideg;
  const int A = p.admis_max;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const bool cw = p.ees == 5;
  const bool weno = p.scheme == 3;
  const int ID2 = p.ideg2;
  const int cpc = w.cpc, tid = threadIdx.x, NT = blockDim.x;
  const int64_t c0 = (int64_t)blockIdx.x * cpc;
  const int nc = (int)((p.n - c0) < cpc ? (p.n - c0) : cpc);
  extern __shared__ __align__(16) unsigned char sm[];
  T* s_G = (T*)(sm + w.o_G);
  T* s_g1 = (T*)(sm + w.o_g1);
  T* s_S = (T*)(sm + w.o_S);
  T* s_tmp = (T*)(sm + w.o_tmp);
  double* s_psi = (double*)(sm + w.o_tmp);
  T* s_gh = (T*)(sm + w.o_gh);
  double* s_w = (double*)(sm + w.o_w);
  T* s_dul = (T*)(sm + w.o_dul);
  double* s_u0 = (double*)(sm + w.o_u0);
  double* s_bnd = (double*)(sm + w.o_bnd);
  double* s_slope = (double*)(sm + w.o_slope);
  int* s_flag = (int*)(sm + w.o_flag);

  const int GS = A * ID * NV;
  const T* Gi = (const T*)p.gbuf;
  for (int i = tid; i < nc * NV; i += NT) s_u0[i] = U[c0 * NV + i];
  for (int i = tid; i < nc * 2; i += NT) s_flag[i] = 0;
  // stencil polynomials: consecutive threads read consecutive cells (lanes)
  for (int i = tid; i < nc * GS; i += NT) {
    int r = i / nc, cl = i - r * nc;
    int64_t c = c0 + cl;
    s_G[cl * GS + r] = Gi[((c >> 5) * GS + r) * 32 + (c & 31)];
  }
  if (weno) {
    const T* IND = (const T*)p.ind + c0 * p.istride;
    for (int i = tid; i < nc * (int)p.istride; i += NT) s_S[i] = IND[i];
  }
  __syncthreads();

  if (weno) {
    if (cw) {  // central polynomial with the low-order stencils removed (reconstruct_p.f90:956-965)
      for (int i = tid; i < nc * ID * NV; i += NT) {
        int cl = i / (ID * NV), r = i - cl * ID * NV, d = r / NV, v = r - d * NV;
        int adm = p.admis[c0 + cl];
        const double lc1 = 1.0 - 1.0 / p.lwci;
        const double lk = adm > 1 ? (1.0 - lc1) / (adm - 1) : 0.0;
        T g3 = T(0);
        if (d < ID2)
          for (int ll = 1; ll < adm; ++ll) g3 = g3 + T(lk) * s_G[cl * GS + (ll * ID + d) * NV + v];
        s_g1[i] = T(1.0 / lc1) * (s_G[cl * GS + d * NV + v] - g3);
      }
      __syncthreads();
    }
    // IS = g^T S g: thread (cell, ll, e) forms (S g)_e g_e for the five variables
    for (int i = tid; i < nc * A * ID; i += NT) {
      int cl = i / (A * ID), r = i - cl * A * ID, ll = r / ID, e = r - ll * ID;
      bool low = cw && ll > 0;
      int nd = low ? ID2 : ID;
      T t[NV] = {T(0), T(0), T(0), T(0), T(0)};
      if (ll < p.admis[c0 + cl] && e < nd) {
        const T* S = s_S + cl * (int)p.istride + (low ? p.i2off : 0);
        const T* g = (cw && ll == 0) ? s_g1 + cl * ID * NV : s_G + cl * GS + ll * ID * NV;
        T acc[NV] = {T(0), T(0), T(0), T(0), T(0)};
        for (int d = 0; d < nd; ++d) {
          T sde = S[d * nd + e];
#pragma unroll
          for (int v = 0; v < NV; ++v) acc[v] += sde * g[d * NV + v];
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) t[v] = g[e * NV + v] * acc[v];
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) s_tmp[(size_t)i * NV + v] = t[v];
    }
    __syncthreads();
    for (int i = tid; i < nc * A * NV; i += NT) {
      int cl = i / (A * NV), r = i - cl * A * NV, ll = r / NV, v = r - ll * NV;
      int nd = (cw && ll > 0) ? ID2 : ID;
      T is = T(0);
      for (int e = 0; e < nd; ++e) is += s_tmp[((size_t)(cl * A + ll) * ID + e) * NV + v];
      s_w[i] = (double)is;
    }
    __syncthreads();
    // nonlinear weights in FP64 ((10E-12)^4 underflows FP32)
    for (int i = tid; i < nc * NV; i += NT) {
      int cl = i / NV, v = i - cl * NV;
      int adm = p.admis[c0 + cl];
      double* ws = s_w + cl * A * NV;
      double lam0, lamk;
      if (cw) {
        lam0 = 1.0 - 1.0 / p.lwci;
        lamk = adm > 1 ? (1.0 - lam0) / (adm - 1) : 0.0;
      } else {
        lam0 = p.lwci;
        lamk = 1.0;
      }
      double tau = 0.0, sum = 0.0;
      if (cw && p.wenoz) {
        for (int ll = 0; ll < adm; ++ll) tau += fabs(ws[v] - ws[ll * NV + v]);
        tau = tau / (adm - 1);
      }
      for (int ll = 0; ll < adm; ++ll) {
        double e = p.weno_eps + ws[ll * NV + v];
        double lam = ll == 0 ? lam0 : lamk, wt;
        if (cw && p.wenoz) {
          double q = tau / e;
          q = q * q;
          wt = lam * (1.0 + q * q);
        } else {
          double e2 = e * e;
          wt = lam / (e2 * e2);
        }
        ws[ll * NV + v] = wt;
        sum += wt;
      }
      for (int ll = 0; ll < adm; ++ll) ws[ll * NV + v] = ws[ll * NV + v] / sum;
    }
    __syncthreads();
    // combined polynomial
    for (int i = tid; i < nc * ID * NV; i += NT) {
      int cl = i / (ID * NV), r = i - cl * ID * NV, d = r / NV, v = r - d * NV;
      int adm = p.admis[c0 + cl];
      const double* ws = s_w + cl * A * NV;
      const T* g0 = cw ? s_g1 + cl * ID * NV : s_G + cl * GS;
      T acc = T(ws[v]) * g0[d * NV + v];
      for (int ll = 1; ll < adm; ++ll)
        if (!cw || d < ID2) acc += T(ws[ll * NV + v]) * s_G[cl * GS + (ll * ID + d) * NV + v];
      s_gh[i] = acc;
    }
    __syncthreads();
  }

  // ---- face values and CHECKSOL
  const T* QPa = (const T*)p.qpts;
  const T* BMa = (const T*)p.bmean;
  const int FQ = MF * QS;
  for (int i = tid; i < nc * FQ; i += NT) {
    int cl = i / FQ, j = i - cl * FQ, f = j / QS, q = j - f * QS;
    int64_t c = c0 + cl;
    T* o = s_dul + (size_t)i * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = T(0);
    if (f >= p.nfaces[c] || q >= face_nq(p, p.ftype[c * MF + f])) continue;
    if (!weno || !p.full[c]) {  // MUSCL everywhere / CHECKSOL: FULL = 0 -> REDUCE
      s_flag[cl * 2] = 1;
      continue;
    }
    const T* xi = QPa + ((size_t)c * FQ + j) * 3;
    T b[ID];
    monomials<P, T>(xi[0], xi[1], xi[2], b);
#pragma unroll
    for (int d = 0; d < ID; ++d) b[d] -= BMa[c * ID + d];
    const T* gh = s_gh + cl * ID * NV;
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
    if (jump_bad(p.gamma, pm, uf, 0.85)) s_flag[cl * 2] = 1;
  }
  __syncthreads();
  const int any = __syncthreads_or((tid < nc) ? s_flag[tid * 2] : 0);
  if (any) {
    // ---- MUSCL with the central stencil polynomial on flagged cells
    for (int i = tid; i < nc * NV; i += NT) {
      int cl = i / NV, v = i - cl * NV;
      if (!s_flag[cl * 2]) continue;
      int64_t c = c0 + cl;
      double u0 = s_u0[i], mn = u0, mx = u0;
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
    for (int i = tid; i < nc * FQ; i += NT) {
      int cl = i / FQ, j = i - cl * FQ, f = j / QS, q = j - f * QS;
      if (!s_flag[cl * 2]) continue;
      int64_t c = c0 + cl;
      double* ps = s_psi + (size_t)i * NV;
      if (f >= p.nfaces[c] || q >= face_nq(p, p.ftype[c * MF + f])) {
#pragma unroll
        for (int v = 0; v < NV; ++v) ps[v] = TOLBIG;
        continue;
      }
      const T* xi = QPa + ((size_t)c * FQ + j) * 3;
      T b[ID];
      monomials<P, T>(xi[0], xi[1], xi[2], b);
#pragma unroll
      for (int d = 0; d < ID; ++d) b[d] -= BMa[c * ID + d];
      const T* g0 = s_G + cl * GS;
      const double e3 = p.kappa_ven * p.minedge[c];
      const double epsi2 = e3 * e3 * e3;
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
    for (int i = tid; i < nc * NV; i += NT) {
      int cl = i / NV, v = i - cl * NV;
      if (!s_flag[cl * 2]) continue;
      double mn = TOLBIG;
      for (int j = 0; j < FQ; ++j) mn = fmin(mn, s_psi[((size_t)cl * FQ + j) * NV + v]);
      s_slope[i] = mn;
    }
    __syncthreads();
    for (int i = tid; i < nc * FQ * NV; i += NT) {
      int cl = i / (FQ * NV);
      if (!s_flag[cl * 2]) continue;
      s_dul[i] = T((double)s_dul[i] * s_slope[cl * NV + i % NV]);
    }
    __syncthreads();
  }

  // ---- CHECKSOLX: first order where a face value jumps by 95 %
  for (int i = tid; i < nc * FQ; i += NT) {
    int cl = i / FQ, j = i - cl * FQ, f = j / QS, q = j - f * QS;
    int64_t c = c0 + cl;
    if (f >= p.nfaces[c] || q >= face_nq(p, p.ftype[c * MF + f])) continue;
    double uf[NV], pm[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uf[v] = s_u0[cl * NV + v] + (double)s_dul[(size_t)i * NV + v];
    cons2prim(p.gamma, s_u0 + cl * NV, pm);
    if (jump_bad(p.gamma, pm, uf, 0.95)) s_flag[cl * 2 + 1] = 1;
  }
  __syncthreads();
  T* out = (T*)p.dul + c0 * FQ * NV;
  for (int i = tid; i < nc * FQ * NV; i += NT) {
    int cl = i / (FQ * NV);
    out[i] = s_flag[cl * 2 + 1] ? T(0) : s_dul[i];
  }
}

}  // namespace ucg
