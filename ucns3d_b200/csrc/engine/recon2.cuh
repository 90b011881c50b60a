// WENO / CWENO / high-order MUSCL reconstruction, one thread block per cell,
// with the cell's pseudo-inverse streamed into shared memory by 1-D bulk
// asynchronous copies (two ring slots, mbarrier completion, no multicast).
//
// Per cell, in the order of ARBITRARY_ORDER (src/reconstruct_p.f90:2954):
//   LEAST_SQUARES      G[ll] = invmat[ll] . (U_k - U_i)      gradients.f90:253-497
//   CP_RECONSTRUCTION  IS = g^T S g, weights, face values    reconstruct_p.f90:920-1250
//   CHECKSOL -> MUSCL on flagged cells -> CHECKSOLX          reconstruct_p.f90:3126, 2286, 3245
#pragma once

#include "device.cuh"

namespace ucg {

constexpr int W2_THREADS = 256;
constexpr int W2_MAXITEM = 16;

// Host-computed description of the stream of table chunks and of the
// shared-memory carve-up (offsets in bytes).
struct W2Plan {
  int nch[8];      // chunks of slice ll (1 or 2)
  int rc[8];       // rows per chunk of slice ll (last chunk: the rest)
  int slot_bytes;  // one ring slot
  int kp;          // row partitions of the LSQ product
  int db;          // rows of G per thread (d block)
  int o_bar, o_slot, o_S, o_du, o_part, o_G, o_g1, o_gh, o_w, o_dul, o_psi, o_u0, o_bnd, o_slope, o_flag,
      o_sten, total;
};

template <typename T>
inline W2Plan w2_plan(int A, int IM, int ID, int IM2, int ID2, int QS, bool cw, const int* sbytes, int ibytes) {
  W2Plan w{};
  const int s = (int)sizeof(T);
  int slot = 0;
  for (int ll = 0; ll < A; ++ll) {
    bool low = cw && ll > 0;
    int nk = low ? IM2 : IM, nd = low ? ID2 : ID;
    int rb = nd * s;
    int g = 16;
    for (int x = rb; x % 2 == 0 && g > 1; x /= 2) g /= 2;  // rows per 16-byte granule
    if (sbytes[ll] <= 16 * 1024 || nk < 2 * g) {
      w.nch[ll] = 1;
      w.rc[ll] = nk;
      slot = slot > sbytes[ll] ? slot : sbytes[ll];
    } else {
      int rc = (nk + 1) / 2;
      rc = (rc + g - 1) / g * g;
      w.nch[ll] = 2;
      w.rc[ll] = rc;
      int b0 = rc * rb, b1 = sbytes[ll] - b0;
      slot = slot > b0 ? slot : b0;
      slot = slot > b1 ? slot : b1;
    }
  }
  w.slot_bytes = (slot + 127) / 128 * 128;
  w.db = ID >= 19 ? 4 : 3;
  int ndb = (ID + w.db - 1) / w.db;
  w.kp = W2_THREADS / ndb;
  if (w.kp > 16) w.kp = 16;
  if (w.kp > IM) w.kp = IM;
  int off = 0;
  auto take = [&](int bytes) {
    int o = off;
    off += (bytes + 127) / 128 * 128;
    return o;
  };
  const int NVv = 5, MFv = 6;
  w.o_bar = take(4 * 8);
  w.o_slot = take(2 * w.slot_bytes);
  w.o_S = take(ibytes);
  w.o_du = take(A * IM * NVv * s);
  int part = w.kp * ndb * w.db * NVv * s, psi = MFv * QS * NVv * 8, tmp = A * ID * NVv * s;
  if (psi > part) part = psi;
  if (tmp > part) part = tmp;
  w.o_part = take(part);
  w.o_psi = w.o_part;  // partial sums are dead once G is formed
  w.o_G = take(A * ID * NVv * s);
  w.o_g1 = take(cw ? ID * NVv * s : 0);
  w.o_gh = take(ID * NVv * s);
  w.o_w = take(A * NVv * 8);
  w.o_dul = take(MFv * QS * NVv * s);
  w.o_u0 = take(NVv * 8);
  w.o_bnd = take(2 * NVv * 8);
  w.o_slope = take(NVv * 8);
  w.o_flag = take(2 * 4);
  w.o_sten = take(A * (IM + 1) * 4);
  w.total = off;
  return w;
}

}  // namespace ucg

namespace ucg {

template <int P, typename T>
__global__ void __launch_bounds__(W2_THREADS, 2) k_weno2(Problem p, const double* __restrict__ U, W2Plan w) {
  constexpr int ID = Deg<P>::ideg;
  const int A = p.admis_max, IM = p.imax, W = IM + 1;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const bool cw = p.ees == 5;
  const bool weno = p.scheme == 3;
  const int ID2 = p.ideg2, IM2 = p.imax2;
  const int tid = threadIdx.x;
  const int64_t c = blockIdx.x;
  extern __shared__ __align__(128) unsigned char sm[];
  uint64_t* bar = (uint64_t*)(sm + w.o_bar);  // [0],[1] ring slots, [2] smoothness block
  T* s_S = (T*)(sm + w.o_S);
  T* s_du = (T*)(sm + w.o_du);
  T* s_part = (T*)(sm + w.o_part);
  double* s_psi = (double*)(sm + w.o_psi);
  T* s_G = (T*)(sm + w.o_G);
  T* s_g1 = (T*)(sm + w.o_g1);
  T* s_gh = (T*)(sm + w.o_gh);
  double* s_w = (double*)(sm + w.o_w);
  T* s_dul = (T*)(sm + w.o_dul);
  double* s_u0 = (double*)(sm + w.o_u0);
  double* s_bnd = (double*)(sm + w.o_bnd);
  double* s_slope = (double*)(sm + w.o_slope);
  int* s_flag = (int*)(sm + w.o_flag);
  int32_t* s_sten = (int32_t*)(sm + w.o_sten);

  const int adm = p.admis[c];
  const char* tab = (const char*)p.invmat + (size_t)c * p.tstride * sizeof(T);
  // stream items: (slice, chunk) in order
  int it_ll[W2_MAXITEM], it_r0[W2_MAXITEM], it_r1[W2_MAXITEM];
  int nitem = 0;
  for (int ll = 0; ll < adm; ++ll) {
    int nk = (cw && ll > 0) ? IM2 : IM;
    for (int j = 0; j < w.nch[ll]; ++j) {
      it_ll[nitem] = ll;
      it_r0[nitem] = j * w.rc[ll];
      it_r1[nitem] = (j + 1 == w.nch[ll]) ? nk : (j + 1) * w.rc[ll];
      ++nitem;
    }
  }
  auto item_src = [&](int it, unsigned& bytes) -> const char* {
    int ll = it_ll[it];
    int nd = (cw && ll > 0) ? ID2 : ID;
    int rb = nd * (int)sizeof(T);
    int off = it_r0[it] * rb;
    bytes = (it_r1[it] == ((cw && ll > 0) ? IM2 : IM)) ? (unsigned)(p.sbytes[ll] - off) : (unsigned)((it_r1[it] - it_r0[it]) * rb);
    return tab + (size_t)p.soff[ll] * sizeof(T) + off;
  };
  auto issue = [&](int it) {
    unsigned bytes;
    const char* src = item_src(it, bytes);
    int slot = it & 1;
    mbar_expect_tx(&bar[slot], bytes);
    bulk_g2s(sm + w.o_slot + slot * w.slot_bytes, src, bytes, &bar[slot]);
  };
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0) {
    if (weno) {
      mbar_expect_tx(&bar[2], (unsigned)p.ibytes);
      bulk_g2s(s_S, (const char*)p.ind + (size_t)c * p.istride * sizeof(T), (unsigned)p.ibytes, &bar[2]);
    }
    if (nitem > 0) issue(0);
    if (nitem > 1) issue(1);
  }
  // own state and stencil indices
  if (tid < NV) s_u0[tid] = U[c * NV + tid];
  for (int i = tid; i < A * W; i += W2_THREADS) s_sten[i] = p.sten[c * A * W + i];
  if (tid < 2) s_flag[tid] = 0;
  __syncthreads();
  // gather U_k - U_i for every stencil cell (FP64 difference, rounded to T)
  for (int i = tid; i < adm * IM; i += W2_THREADS) {
    int ll = i / IM, k = i - ll * IM;
    int nk = (cw && ll > 0) ? IM2 : IM;
    T* o = s_du + (size_t)i * NV;
    if (k < nk) {
      const double* uy = U + (int64_t)s_sten[ll * W + k + 1] * NV;
#pragma unroll
      for (int v = 0; v < NV; ++v) o[v] = T(uy[v] - s_u0[v]);
    }
  }
  __syncthreads();

  // ---- least squares, slice by slice as the chunks arrive
  bool ok = true;
  const int DB = w.db, KP = w.kp;
  for (int it = 0; it < nitem; ++it) {
    const int ll = it_ll[it];
    const bool low = cw && ll > 0;
    const int nd = low ? ID2 : ID;
    const int ndb = (nd + DB - 1) / DB;
    const int slot = it & 1;
    if (!mbar_wait(&bar[slot], (it >> 1) & 1)) ok = false;
    const T* M = (const T*)(sm + w.o_slot + slot * w.slot_bytes) - it_r0[it] * nd;  // row-indexed
    const int db = tid % ndb, kp = tid / ndb;
    const bool first_chunk = it == 0 || it_ll[it - 1] != ll;
    const bool last_chunk = it + 1 == nitem || it_ll[it + 1] != ll;
    if (kp < KP) {
      T acc[4][NV];
      // partial sums of this slice live in s_part between chunks
      if (first_chunk) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int v = 0; v < NV; ++v) acc[j][v] = T(0);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int v = 0; v < NV; ++v)
            acc[j][v] = j < DB ? s_part[((size_t)kp * ndb * DB + db * DB + j) * NV + v] : T(0);
      }
      const T* du = s_du + (size_t)ll * IM * NV;
      for (int k = it_r0[it] + kp; k < it_r1[it]; k += KP) {
        T dv[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) dv[v] = du[k * NV + v];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          int d = db * DB + j;
          if (j < DB && d < nd) {
            T m = M[k * nd + d];
#pragma unroll
            for (int v = 0; v < NV; ++v) acc[j][v] += m * dv[v];
          }
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j < DB)
#pragma unroll
          for (int v = 0; v < NV; ++v) s_part[((size_t)kp * ndb * DB + db * DB + j) * NV + v] = acc[j][v];
    }
    __syncthreads();  // slot consumed, partials written
    if (tid == 0 && it + 2 < nitem) {
      fence_proxy_async();
      issue(it + 2);
    }
    if (last_chunk) {
      // G[ll][d][v] = sum over row partitions, in partition order
      const int npart = KP < ((low ? IM2 : IM)) ? KP : (low ? IM2 : IM);
      for (int i = tid; i < ID * NV; i += W2_THREADS) {
        int d = i / NV, v = i - d * NV;
        T s = T(0);
        if (d < nd)
          for (int q = 0; q < npart; ++q) s += s_part[((size_t)q * ndb * DB + d) * NV + v];
        s_G[((size_t)ll * ID + d) * NV + v] = s;
      }
      __syncthreads();
    }
  }
  if (!ok) atomicOr(p.health, HEALTH_TIMEOUT);

  T* s_tmp = s_part;  // [A][ID][NV] scratch for the indicator reduction
  if (weno) {
    if (!mbar_wait(&bar[2], 0)) atomicOr(p.health, HEALTH_TIMEOUT);
    // CWENO: central polynomial with the low-order stencils removed (reconstruct_p.f90:956-965)
    if (cw) {
      const double lc1 = 1.0 - 1.0 / p.lwci;
      const double lk = adm > 1 ? (1.0 - lc1) / (adm - 1) : 0.0;
      for (int i = tid; i < ID * NV; i += W2_THREADS) {
        int d = i / NV, v = i - d * NV;
        T g3 = T(0);
        if (d < ID2)
          for (int ll = 1; ll < adm; ++ll) g3 = g3 + T(lk) * s_G[((size_t)ll * ID + d) * NV + v];
        s_g1[i] = T(1.0 / lc1) * (s_G[(size_t)d * NV + v] - g3);
      }
      __syncthreads();
    }
    // IS = g^T S g: thread (ll, e) forms (S g)_e g_e for the five variables
    for (int i = tid; i < adm * ID; i += W2_THREADS) {
      int ll = i / ID, e = i - ll * ID;
      bool low = cw && ll > 0;
      int nd = low ? ID2 : ID;
      T t[NV] = {T(0), T(0), T(0), T(0), T(0)};
      if (e < nd) {
        const T* S = low ? s_S + p.i2off : s_S;
        const T* g = (cw && ll == 0) ? s_g1 : s_G + (size_t)ll * ID * NV;
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
    for (int i = tid; i < adm * NV; i += W2_THREADS) {
      int ll = i / NV, v = i - ll * NV;
      int nd = (cw && ll > 0) ? ID2 : ID;
      T is = T(0);
      for (int e = 0; e < nd; ++e) is += s_tmp[((size_t)ll * ID + e) * NV + v];
      s_w[ll * NV + v] = (double)is;
    }
    __syncthreads();
    // nonlinear weights in FP64 ((10E-12)^4 underflows FP32)
    if (tid < NV) {
      const int v = tid;
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
        for (int ll = 0; ll < adm; ++ll) tau += fabs(s_w[v] - s_w[ll * NV + v]);
        tau = tau / (adm - 1);
      }
      for (int ll = 0; ll < adm; ++ll) {
        double e = p.weno_eps + s_w[ll * NV + v];
        double lam = ll == 0 ? lam0 : lamk, wt;
        if (cw && p.wenoz) {
          double q = tau / e;
          q = q * q;
          wt = lam * (1.0 + q * q);
        } else {
          double e2 = e * e;
          wt = lam / (e2 * e2);
        }
        s_w[ll * NV + v] = wt;
        sum += wt;
      }
      for (int ll = 0; ll < adm; ++ll) s_w[ll * NV + v] = s_w[ll * NV + v] / sum;
    }
    __syncthreads();
    // combined polynomial
    for (int i = tid; i < ID * NV; i += W2_THREADS) {
      int d = i / NV, v = i - d * NV;
      const T* g0 = cw ? s_g1 : s_G;
      T acc = T(s_w[v]) * g0[d * NV + v];
      for (int ll = 1; ll < adm; ++ll)
        if (!cw || d < ID2) acc += T(s_w[ll * NV + v]) * s_G[((size_t)ll * ID + d) * NV + v];
      s_gh[i] = acc;
    }
    __syncthreads();
  }

  // ---- face values and CHECKSOL
  const T* QP = (const T*)p.qpts + (size_t)c * MF * QS * 3;
  const T* BM = (const T*)p.bmean + (size_t)c * ID;
  const int nfc = p.nfaces[c];
  const bool full = p.full[c] != 0;
  for (int i = tid; i < MF * QS; i += W2_THREADS) {
    int f = i / QS, q = i - f * QS;
    T* o = s_dul + (size_t)i * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = T(0);
    if (f >= nfc || q >= face_nq(p, p.ftype[c * MF + f])) continue;
    if (!weno || !full) {  // MUSCL everywhere / CHECKSOL: FULL = 0 -> REDUCE
      s_flag[0] = 1;
      continue;
    }
    T b[ID];
    monomials<P, T>(QP[i * 3 + 0], QP[i * 3 + 1], QP[i * 3 + 2], b);
#pragma unroll
    for (int d = 0; d < ID; ++d) b[d] -= BM[d];
    double uf[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      T res = T(0);
#pragma unroll
      for (int d = 0; d < ID; ++d) res += b[d] * s_gh[d * NV + v];
      o[v] = res;
      uf[v] = s_u0[v] + (double)res;
    }
    double pm[NV];
    cons2prim(p.gamma, s_u0, pm);
    if (jump_bad(p.gamma, pm, uf, 0.85)) s_flag[0] = 1;
  }
  __syncthreads();

  // ---- MUSCL with the central stencil polynomial on flagged cells
  if (s_flag[0]) {
    if (tid < NV) {
      const int v = tid;
      double u0 = s_u0[v], mn = u0, mx = u0;
      for (int f = 0; f < nfc; ++f) {
        int64_t nb = p.neigh[c * MF + f];
        if (nb < 0) continue;
        double un = U[nb * NV + v];
        mn = fmin(mn, un);
        mx = fmax(mx, un);
      }
      s_bnd[v] = mn - u0;
      s_bnd[NV + v] = mx - u0;
    }
    __syncthreads();
    const double e3 = p.kappa_ven * p.minedge[c];
    const double epsi2 = e3 * e3 * e3;
    for (int i = tid; i < MF * QS; i += W2_THREADS) {
      int f = i / QS, q = i - f * QS;
      double* ps = s_psi + (size_t)i * NV;
      if (f >= nfc || q >= face_nq(p, p.ftype[c * MF + f])) {
#pragma unroll
        for (int v = 0; v < NV; ++v) ps[v] = TOLBIG;
        continue;
      }
      T b[ID];
      monomials<P, T>(QP[i * 3 + 0], QP[i * 3 + 1], QP[i * 3 + 2], b);
#pragma unroll
      for (int d = 0; d < ID; ++d) b[d] -= BM[d];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        T res = T(0);
#pragma unroll
        for (int d = 0; d < ID; ++d) res += b[d] * s_G[d * NV + v];
        double dd = (s_u0[v] + (double)res) - s_u0[v];
        s_dul[(size_t)i * NV + v] = T(dd);
        ps[v] = venkat(dd, s_bnd[v], s_bnd[NV + v], epsi2);
      }
    }
    __syncthreads();
    if (tid < NV) {
      double mn = TOLBIG;
      for (int j = 0; j < MF * QS; ++j) mn = fmin(mn, s_psi[(size_t)j * NV + tid]);
      s_slope[tid] = mn;
    }
    __syncthreads();
    for (int i = tid; i < MF * QS * NV; i += W2_THREADS)
      s_dul[i] = T((double)s_dul[i] * s_slope[i % NV]);
    __syncthreads();
  }

  // ---- CHECKSOLX: first order where a face value jumps by 95 %
  for (int i = tid; i < MF * QS; i += W2_THREADS) {
    int f = i / QS, q = i - f * QS;
    if (f >= nfc || q >= face_nq(p, p.ftype[c * MF + f])) continue;
    double uf[NV], pm[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uf[v] = s_u0[v] + (double)s_dul[(size_t)i * NV + v];
    cons2prim(p.gamma, s_u0, pm);
    if (jump_bad(p.gamma, pm, uf, 0.95)) s_flag[1] = 1;
  }
  __syncthreads();
  T* out = (T*)p.dul + (size_t)c * MF * QS * NV;
  const bool first = s_flag[1] != 0;
  for (int i = tid; i < MF * QS * NV; i += W2_THREADS) out[i] = first ? T(0) : s_dul[i];
}

}  // namespace ucg
