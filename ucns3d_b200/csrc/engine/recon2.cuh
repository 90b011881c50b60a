// Reconstruction for WENO / CWENO / high-order MUSCL in two kernels.
//
// k_lsq      LEAST_SQUARES (src/gradients.f90:253-497): one lane per cell.
//            Tables are interleaved over groups of 32 cells, so every table
//            load of a warp is one contiguous 128/256-byte row; each gathered
//            difference U_k - U_i is reused across DH rows held in registers.
//            Output: the stencil polynomials G[ll][d][v], interleaved.
// k_wpost    CP_RECONSTRUCTION (src/reconstruct_p.f90:920-1250), CHECKSOL,
//            MUSCL fall-back, CHECKSOLX (3126-3406): one lane per cell, no
//            block barriers; smoothness indicators as packed quadratic forms.
#pragma once

#include "device.cuh"

namespace ucg {

// rows of G held in registers per pass (accumulators: DH x 5 values of T)
template <int P, typename T>
struct LsqRows {
  static constexpr int ID = Deg<P>::ideg;
  static constexpr int value = P == 4 ? (sizeof(T) == 4 ? 34 : 17) : P == 3 ? (sizeof(T) == 4 ? 19 : 10) : ID;
};

// The conserved state in 48-byte records (five values and a zero), formed
// once per stage: k_lsq<P, T, true> gathers each stencil member with three
// aligned 16-byte loads instead of five 8-byte loads.
template <int P, typename T>
__global__ void k_pad_state(Problem p, const double* __restrict__ U) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  const double* u = U + c * NV;
  double2* o = (double2*)(p.upad + c * 6);
  o[0] = make_double2(u[0], u[1]);
  o[1] = make_double2(u[2], u[3]);
  o[2] = make_double2(u[4], 0.0);
}

// PAD: stencil members gathered from p.upad (the engine's stage), else from U
// (also used on tangent states by the discrete adjoint).
// FP32 at IORDER 3: four blocks per SM (128 registers instead of 160), at
// IORDER 2 five (instead of four at 126): the gather of the stencil members
// is latency-bound, and more warps in flight made the 2.1 M-cell CWENO4
// step 6 % faster (61.1 -> 57.3 ms on one box) and the 82,944-tet WENO3
// step 3 % (1.094 -> 1.063 ms); the same values bit for bit.  Five blocks
// at IORDER 3 (102 registers) made the CWENO4 step slower (56.0 -> 58.0 ms).
template <int P, typename T, bool PAD = false>
__global__ void __launch_bounds__(128, sizeof(T) != 4 ? 1 : P == 3 ? 4 : P == 2 ? 5 : 1)
    k_lsq(Problem p, const double* __restrict__ U) {
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
#pragma unroll 2
        for (int k = 0; k < nk; ++k) {
          T du[NV];
          if (PAD) {
            const double2* q = (const double2*)(p.upad + (int64_t)S[k * 32] * 6);
            const double2 a = q[0], b = q[1], e = q[2];
            const double uy[NV] = {a.x, a.y, b.x, b.y, e.x};
#pragma unroll
            for (int v = 0; v < NV; ++v) du[v] = T(uy[v] - u0[v]);
          } else {
            const double* uy = U + (int64_t)S[k * 32] * NV;
#pragma unroll
            for (int v = 0; v < NV; ++v) du[v] = T(uy[v] - u0[v]);
          }
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
      if (live)
#pragma unroll
        for (int j = 0; j < DH; ++j)
          if (d0 + j < nd)
#pragma unroll
            for (int v = 0; v < NV; ++v) Gi[(int64_t)((ll * ID + d0 + j) * NV + v) * 32] = acc[j][v];
    }
  }
}

// k_lsq with the pseudo-inverse rows streamed through shared memory by bulk
// copies.  Each warp owns one 32-cell group and a ring of NSTG stages; a
// stage holds the rows [d0, d0 + DH) of one stencil member for the 32 cells
// (DH * 32 table elements, contiguous in the interleaved layout), copied by
// cp.async.bulk and completed on the stage's mbarrier.  Lane 0 refills a
// stage as soon as the warp has consumed it, so NSTG - 1 members are in
// flight while the warp multiplies the current one; the gathered neighbour
// state of the next member is loaded one member ahead.  Same products and
// accumulation order as k_lsq, so G is the same bit for bit.  A wait that
// gives up (after Problem::lsq_wait polls) sets HEALTH_TIMEOUT, drains the
// copies in flight (each wait bounded by LSQ_WAIT, whatever lsq_wait is) and
// leaves the group.  Opt-in (Problem::lsq_bulk): on B200 it takes 7.2 ms
// against k_lsq's 5.8 ms for the mixed WENO5 64^3 stage, at 3, 4 or 6
// stages alike, because k_lsq is bound by the per-member gather of the
// neighbour states and the issue rate of 8 warps per SM, not by the latency
// of its coalesced table loads.
template <int P, typename T>
__host__ __device__ constexpr int lsq_stage_elems() {
  return LsqRows<P, T>::value * 32;
}
template <int P, typename T, int NSTG>
__host__ __device__ constexpr size_t lsq_tma_smem() {
  return (size_t)4 * NSTG * lsq_stage_elems<P, T>() * sizeof(T) + (size_t)4 * NSTG * sizeof(uint64_t);
}

// polls of one stage wait (about 20 ms; a stage normally lands in microseconds)
constexpr long LSQ_WAIT = 1L << 16;

template <int P, typename T, int NSTG>
__global__ void __launch_bounds__(128) k_lsq_tma(Problem p, const double* __restrict__ U) {
  constexpr int ID = Deg<P>::ideg;
  constexpr int DH = LsqRows<P, T>::value;
  constexpr int CH = lsq_stage_elems<P, T>();
  extern __shared__ __align__(128) unsigned char lsq_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* ring = (T*)lsq_smem + warp * NSTG * CH;
  uint64_t* bar = (uint64_t*)((T*)lsq_smem + 4 * NSTG * CH) + warp * NSTG;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t grp = c >> 5;
  if (grp * 32 >= p.n) return;  // the whole warp: no cell of this group exists
  const bool live = c < p.n;
  const int A = p.admis_max, W = p.imax + 1;
  const bool cw = p.ees == 5;
  const int adm = live ? p.admis[c] : 0;
  const int admw = __reduce_max_sync(0xffffffffu, adm);
  double u0[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u0[v] = live ? U[c * NV + v] : 0.0;
  const T* Mg = (const T*)p.invmat + grp * p.tstride * 32;  // the group's tables
  const int32_t* Si = p.sten + grp * (int64_t)(A * W) * 32 + lane;
  T* Gi = (T*)p.gbuf + grp * (int64_t)(A * ID * NV) * 32 + lane;
  if (lane == 0) {
    for (int s = 0; s < NSTG; ++s) mbar_init(&bar[s], 1);
    mbar_fence_init();
  }
  __syncwarp();
  // copy cursor: the next (stencil, row pass, member) to copy, tracked by
  // every lane (warp-uniform); lane 0 issues the copies
  int ill = 0, id0 = 0, ik = 0;
  auto n_k = [&](int ll) { return cw && ll > 0 ? p.imax2 : p.imax; };
  auto n_d = [&](int ll) { return cw && ll > 0 ? p.ideg2 : ID; };
  auto copy_next = [&](int slot) {
    const int nd = n_d(ill);
    if (lane == 0) {
      const int rows = nd - id0 < DH ? nd - id0 : DH;
      const unsigned bytes = (unsigned)(rows * 32 * sizeof(T));
      fence_proxy_async();
      mbar_expect_tx(&bar[slot], bytes);
      bulk_g2s(ring + slot * CH, Mg + (int64_t)(p.soff[ill] + id0 + ik * nd) * 32, bytes, &bar[slot]);
    }
    if (++ik == n_k(ill)) {
      ik = 0;
      id0 += DH;
      if (id0 >= nd) {
        id0 = 0;
        ++ill;
      }
    }
  };
  int issued = 0;
  for (; issued < NSTG && ill < admw; ++issued) copy_next(issued);
  int t = 0;  // members consumed
  bool ok = true;
  const long wait = p.lsq_wait < 0 ? LSQ_WAIT : p.lsq_wait;
  for (int ll = 0; ll < admw && ok; ++ll) {
    const int nk = n_k(ll), nd = n_d(ll);
    const bool act = ll < adm;
    const int32_t* S = Si + (ll * W + 1) * 32;
    for (int d0 = 0; d0 < nd && ok; d0 += DH) {
      T acc[DH][NV];
#pragma unroll
      for (int j = 0; j < DH; ++j)
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[j][v] = T(0);
      double un[NV] = {0, 0, 0, 0, 0};  // state of member k, loaded one member ahead
      if (act) {
        const double* uy = U + (int64_t)S[0] * NV;
#pragma unroll
        for (int v = 0; v < NV; ++v) un[v] = uy[v];
      }
      for (int k = 0; k < nk; ++k) {
        T du[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) du[v] = T(un[v] - u0[v]);
        if (act && k + 1 < nk) {
          const double* uy = U + (int64_t)S[(k + 1) * 32] * NV;
#pragma unroll
          for (int v = 0; v < NV; ++v) un[v] = uy[v];
        }
        const int slot = t % NSTG;
        if (!__all_sync(0xffffffffu, mbar_wait(&bar[slot], (unsigned)(t / NSTG) & 1u, wait))) {
          ok = false;
          break;
        }
        if (act) {
          const T* Mk = ring + slot * CH + lane;
#pragma unroll
          for (int j = 0; j < DH; ++j)
            if (d0 + j < nd) {
              const T m = Mk[j * 32];
#pragma unroll
              for (int v = 0; v < NV; ++v) acc[j][v] += m * du[v];
            }
        }
        __syncwarp();
        ++t;
        if (ill < admw) {  // refill the stage just consumed
          copy_next(slot);
          ++issued;
        }
      }
      if (ok && live)
#pragma unroll
        for (int j = 0; j < DH; ++j)
          if (d0 + j < nd)
#pragma unroll
            for (int v = 0; v < NV; ++v) Gi[(int64_t)((ll * ID + d0 + j) * NV + v) * 32] = acc[j][v];
    }
  }
  if (!ok) {
    if (lane == 0) atomicOr(p.health, HEALTH_TIMEOUT);
    for (; t < issued; ++t) mbar_wait(&bar[t % NSTG], (unsigned)(t / NSTG) & 1u, LSQ_WAIT);
  }
}

// ------------------------------------------------------------- k_wpost
// Smoothness matrices are packed upper triangles, interleaved over 32-cell
// groups like the pseudo-inverses: entry (d, e >= d) of cell c is element
// tri(d, e) = d*nd - d*(d-1)/2 + (e - d) of the cell's block, and an
// off-diagonal entry holds S_de + S_ed, so that
//   g^T S g = sum_d g_d * sum_{e >= d} P_de g_e
// is the full quadratic form of INDICATORMATRIX (src/prestore.f90:1529-1673)
// with half the loads and multiplies.

// variables per register pass of each phase: indicators (IS), combined
// polynomial + face values (FACE), MUSCL fall-back (FALL); the polynomial
// of a pass ([ID] x variables) stays in registers.  Measured on the 64^3
// WENO5 stage (B200): FP32 FACE 5 takes 1.95 ms against 2.75 ms for 3 and
// 3.17 ms for 2 (one read of the polynomials, CHECKSOL in registers); FP64
// IS 3 / FACE 3 takes 6.50 ms against 6.95 ms for 2 / 2, 8.11 ms for IS 1
// and 7.46 ms for FACE 5 (spills).
#ifndef UCG_WV_IS_F
#define UCG_WV_IS_F 5
#endif
#ifndef UCG_WV_FACE_F
#define UCG_WV_FACE_F 5
#endif
#ifndef UCG_WV_FALL_F
#define UCG_WV_FALL_F 1
#endif
#ifndef UCG_WV_IS_D
#define UCG_WV_IS_D 3
#endif
#ifndef UCG_WV_FACE_D
#define UCG_WV_FACE_D 3
#endif
#ifndef UCG_WV_FALL_D
#define UCG_WV_FALL_D 1
#endif
#ifndef UCG_WV_CHAR_F
#define UCG_WV_CHAR_F 5
#endif
#ifndef UCG_WV_CHAR_D
#define UCG_WV_CHAR_D 3
#endif
template <typename T>
struct WVars {
  static constexpr int is = sizeof(T) == 4 ? UCG_WV_IS_F : UCG_WV_IS_D;
  static constexpr int face = sizeof(T) == 4 ? UCG_WV_FACE_F : UCG_WV_FACE_D;
  static constexpr int fall = sizeof(T) == 4 ? UCG_WV_FALL_F : UCG_WV_FALL_D;
  static constexpr int chr = sizeof(T) == 4 ? UCG_WV_CHAR_F : UCG_WV_CHAR_D;
};

// is[k] += sum_d g[d][k] * sum_{e>=d} P_de g[e][k] over d, e < nd <= NMAX.
// P: the cell's packed triangle, vector-interleaved (rows padded to VEC);
// entries past nd in a row's last vector are zero, and so is g[e] for e >= nd.
template <int NMAX, int VG, typename T>
__device__ __forceinline__ void quad_form(const T* __restrict__ P, const T (&g)[NMAX][VG], int nd, T (&is)[VG]) {
  constexpr int VEC = Vec<T>::N;
  int rs = 0;  // first vector of row d
#pragma unroll
  for (int d = 0; d < NMAX; ++d) {
    if (d < nd) {
      T t[VG];
#pragma unroll
      for (int k = 0; k < VG; ++k) t[k] = T(0);
#pragma unroll
      for (int q = 0; q < (NMAX - d + VEC - 1) / VEC; ++q)
        if (d + q * VEC < nd) {
          T s[VEC];
          ldv(P + (int64_t)(rs + q) * 32 * VEC, s);
#pragma unroll
          for (int i = 0; i < VEC; ++i)
            if (d + q * VEC + i < NMAX)
#pragma unroll
              for (int k = 0; k < VG; ++k) t[k] += s[i] * g[d + q * VEC + i][k];
        }
      rs += (nd - d + VEC - 1) / VEC;
#pragma unroll
      for (int k = 0; k < VG; ++k) is[k] += g[d][k] * t[k];
      // keep the loads of one row together: without this fence the
      // compiler hoists the whole triangle and spills it
      asm volatile("" ::: "memory");
    }
  }
}

// A[u][w] += sum_d g[d][u] * sum_{e>=d} P_de g[e][w] over d, e < nd (P the
// packed triangle as in quad_form); sym(A) = g^T S g for every pair of
// columns, A[u][u] the quadratic form of column u.
template <int NMAX, int VG, typename T>
__device__ __forceinline__ void sym_form(const T* __restrict__ P, const T (&g)[NMAX][VG], int nd, T (&A)[VG][VG]) {
  constexpr int VEC = Vec<T>::N;
  int rs = 0;
#pragma unroll
  for (int d = 0; d < NMAX; ++d) {
    if (d < nd) {
      T t[VG];
#pragma unroll
      for (int k = 0; k < VG; ++k) t[k] = T(0);
#pragma unroll
      for (int q = 0; q < (NMAX - d + VEC - 1) / VEC; ++q)
        if (d + q * VEC < nd) {
          T s[VEC];
          ldv(P + (int64_t)(rs + q) * 32 * VEC, s);
#pragma unroll
          for (int i = 0; i < VEC; ++i)
            if (d + q * VEC + i < NMAX)
#pragma unroll
              for (int k = 0; k < VG; ++k) t[k] += s[i] * g[d + q * VEC + i][k];
        }
      rs += (nd - d + VEC - 1) / VEC;
#pragma unroll
      for (int u = 0; u < VG; ++u)
#pragma unroll
        for (int w = 0; w < VG; ++w) A[u][w] += g[d][u] * t[w];
      asm volatile("" ::: "memory");
    }
  }
}

// Smoothness indicators IS[ll][v] = g^T S g of every stencil polynomial,
// one block per 32-cell group with one warp per stencil: lane i of warp ll
// takes stencil ll of cell i of the group.  The warps of a block read the
// same packed triangles (the cells' INDICATOR, prestore.f90:1529-1673) at
// about the same time, so each triangle comes from DRAM once and is reused
// from L1/L2 by the other stencils, instead of once per stencil as when one
// lane runs all the stencils of its cell.  Output: p.isb, FP64, interleaved
// over 32-cell groups ((group * A + ll) * NV + v) * 32 + lane; cells that
// take the MUSCL fall-back outright (not FULL) are skipped, except under
// MOOD, where every cell is reconstructed.
template <int P, typename T>
__global__ void __launch_bounds__(224) k_wis(Problem p) {
  constexpr int ID = Deg<P>::ideg;
  constexpr int VEC = Vec<T>::N;
  constexpr int L2 = ID < 9 ? ID : 9;
  constexpr int VI = WVars<T>::is;
  const int lane = threadIdx.x & 31, ll = threadIdx.x >> 5;
  const int64_t grp = blockIdx.x, c = grp * 32 + lane;
  if (c >= p.n || (!p.mprev && !p.full[c])) return;
  const int adm = p.admis[c];
  if (ll >= adm) return;
  const int A = p.admis_max, ID2 = p.ideg2;
  const bool cw = p.ees == 5, low = cw && ll > 0;
  const T* Gc = (const T*)p.gbuf + grp * (int64_t)(A * ID * NV) * 32 + lane;
  auto G = [&](int l, int d, int v) -> T { return Gc[(int64_t)((l * ID + d) * NV + v) * 32]; };
  const double lc1 = 1.0 - 1.0 / p.lwci;
  const double lk = adm > 1 ? (1.0 - lc1) / (adm - 1) : 0.0;
  const T* Pc = (const T*)p.ind + grp * p.istride * 32 + lane * VEC;
  double* out = p.isb + (grp * A + ll) * (int64_t)NV * 32 + lane;
  for (int v0 = 0; v0 < NV; v0 += VI) {
    T is[VI];
#pragma unroll
    for (int k = 0; k < VI; ++k) is[k] = T(0);
    if (low) {
      T g[L2][VI];
#pragma unroll
      for (int d = 0; d < L2; ++d)
#pragma unroll
        for (int k = 0; k < VI; ++k) g[d][k] = (v0 + k < NV && d < ID2) ? G(ll, d, v0 + k) : T(0);
      quad_form<L2, VI>(Pc + (int64_t)(p.i2off / VEC) * 32 * VEC, g, ID2, is);
    } else {
      T g[ID][VI];
#pragma unroll
      for (int d = 0; d < ID; ++d)
#pragma unroll
        for (int k = 0; k < VI; ++k) g[d][k] = (v0 + k < NV) ? G(ll, d, v0 + k) : T(0);
      if (ll == 0 && cw) {  // the CWENO central polynomial with the lower-order stencils removed
        T g3[L2][VI];
#pragma unroll
        for (int d = 0; d < L2; ++d)
#pragma unroll
          for (int k = 0; k < VI; ++k) g3[d][k] = T(0);
        for (int l2 = 1; l2 < adm; ++l2)
#pragma unroll
          for (int d = 0; d < L2; ++d)
#pragma unroll
            for (int k = 0; k < VI; ++k)
              if (v0 + k < NV && d < ID2) g3[d][k] = g3[d][k] + T(lk) * G(l2, d, v0 + k);
#pragma unroll
        for (int d = 0; d < ID; ++d)
#pragma unroll
          for (int k = 0; k < VI; ++k)
            if (v0 + k < NV) g[d][k] = T(1.0 / lc1) * (g[d][k] - (d < L2 ? g3[d][k] : T(0)));
      }
      quad_form<ID, VI>(Pc, g, ID, is);
    }
#pragma unroll
    for (int k = 0; k < VI; ++k)
      if (v0 + k < NV) out[(int64_t)(v0 + k) * 32] = (double)is[k];
  }
}

// k_wface (conserved-variable WENO, IORDER 4, indicators from k_wis): the
// nonlinear weights, the combined polynomial and its face values, one block
// per 32-cell group with one warp per conserved variable (lane i: cell i of
// the group).  A thread holds one variable's combined polynomial (ID
// coefficients) instead of all five, so the block runs at several times
// k_wpost's occupancy.  The group's face points are staged in shared memory
// once (the five warps evaluate at the same points); the values of one face
// go through shared memory, [cell][point][variable] with an odd row stride
// (no bank conflicts), from where the block tests CHECKSOL (0.85) and stores
// them as one contiguous run per cell.  Cells that fail CHECKSOL, or are not
// FULL, are marked in p.wflag for k_wpost<..., FB> (the MUSCL fall-back).
// Weights, combination and face values take k_wpost's operations in
// k_wpost's order.  Under MOOD the cells that are not FULL are reconstructed
// too (over their admissible stencils) and marked.
template <int P, typename T>
__global__ void __launch_bounds__(32 * NV) k_wface(Problem p, const double* __restrict__ U) {
  constexpr int ID = Deg<P>::ideg;
  constexpr int L2 = ID < 9 ? ID : 9;
  constexpr int MA = 7;  // stencils per cell at most
  extern __shared__ __align__(16) unsigned char wf_smem[];
  __shared__ int s_flag[32];
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const int FQ = MF * QS;
  const int RS = (QS * NV) | 1;  // row stride of a cell in s_o
  T* s_x = (T*)wf_smem;          // [FQ * 3][32]: the group's face points, as in p.qpts
  T* s_o = s_x + FQ * 3 * 32;    // [32][RS]: the values of one face
  const int tid = threadIdx.x, lane = tid & 31, v = tid >> 5;
  const int64_t grp = blockIdx.x, c = grp * 32 + lane;
  {
    const T* xg = (const T*)p.qpts + grp * (int64_t)FQ * 3 * 32;
    for (int i = tid; i < FQ * 3 * 32; i += 32 * NV) s_x[i] = __ldcs(xg + i);
  }
  const bool cell = c < p.n;
  const bool full = cell && p.full[c];
  const bool live = cell && (full || p.mprev);
  const int A = p.admis_max;
  const int adm = live ? p.admis[c] : 0;
  const bool cw = p.ees == 5;
  const int ID2 = p.ideg2;
  const double lc1 = 1.0 - 1.0 / p.lwci;
  const double lk = adm > 1 ? (1.0 - lc1) / (adm - 1) : 0.0;
  if (tid < 32) s_flag[tid] = full ? 0 : 1;
  // ---- weights of variable v (WENOWEIGHTS, FP64)
  double w[MA];
  {
    const double* is = p.isb + grp * (int64_t)A * NV * 32 + lane + v * 32;
    const double lam0 = cw ? lc1 : p.lwci, lamk = cw ? lk : 1.0;
    double tau = 0.0, sum = 0.0;
    if (cw && p.wenoz) {
#pragma unroll
      for (int l = 0; l < MA; ++l)
        if (l < adm) tau += fabs(is[0] - is[(int64_t)l * NV * 32]);
      tau = tau / (adm - 1);
    }
#pragma unroll
    for (int l = 0; l < MA; ++l) {
      w[l] = 0.0;
      if (l < adm) {
        const double e = p.weno_eps + is[(int64_t)l * NV * 32];
        const double lam = l == 0 ? lam0 : lamk;
        double wt;
        if (cw && p.wenoz) {
          double q = tau / e;
          q = q * q;
          wt = lam * (1.0 + q * q);
        } else {
          const double e2 = e * e;
          wt = lam / (e2 * e2);
        }
        w[l] = wt;
        sum += wt;
      }
    }
#pragma unroll
    for (int l = 0; l < MA; ++l) w[l] = w[l] / sum;
  }
  // ---- combined polynomial of variable v (CWENO: the central stencil with
  // the lower-order ones removed, reconstruct_p.f90:956-965)
  const T* Gc = (const T*)p.gbuf + grp * (int64_t)(A * ID * NV) * 32 + v * 32 + lane;
  auto G = [&](int l, int d) -> T { return Gc[(int64_t)((l * ID + d) * NV) * 32]; };
  T gh[ID];
#pragma unroll
  for (int d = 0; d < ID; ++d) gh[d] = live ? G(0, d) : T(0);
  if (live && cw) {
    T g3[L2];
#pragma unroll
    for (int d = 0; d < L2; ++d) g3[d] = T(0);
    for (int l2 = 1; l2 < adm; ++l2)
#pragma unroll
      for (int d = 0; d < L2; ++d)
        if (d < ID2) g3[d] = g3[d] + T(lk) * G(l2, d);
#pragma unroll
    for (int d = 0; d < ID; ++d) gh[d] = T(1.0 / lc1) * (gh[d] - (d < L2 ? g3[d] : T(0)));
  }
  if (live) {
    const T w0 = T(w[0]);
#pragma unroll
    for (int d = 0; d < ID; ++d) gh[d] = w0 * gh[d];
    // every stencil row of the table is in the buffer (l < A), so the loads
    // need no guard on adm and can all be in flight; rows past adm add 0 * 0
#pragma unroll
    for (int l = 1; l < MA; ++l)
      if (l < A) {
        const bool on = l < adm;
        const T wl = on ? T(w[l]) : T(0);
#pragma unroll
        for (int d = 0; d < ID; ++d)
          if (!cw || d < ID2) {
            const T gv = G(l, d);
            gh[d] += wl * (on ? gv : T(0));
          }
      }
  }
  T cb = T(0);
  {
    const T* bmv = (const T*)p.bmean + grp * (int64_t)ID * 32 + lane;
#pragma unroll
    for (int d = 0; d < ID; ++d) cb += bmv[d * 32] * gh[d];
  }
  // ---- face values, CHECKSOL and the stores, face by face
  __syncthreads();  // s_x
  const T* xq = s_x + lane;
  const int nf = cell ? p.nfaces[c] : 0;
  double u0[NV], pm[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) u0[k] = cell ? U[c * NV + k] : 1.0;
  cons2prim(p.gamma, u0, pm);
  bool flag = false;
  T* out = (T*)p.dul + grp * 32 * (int64_t)FQ * NV;
  const int ncl = p.n - grp * 32 < 32 ? (int)(p.n - grp * 32) : 32;  // cells of this group
  for (int f = 0; f < MF; ++f) {
    T* so = s_o;
    if (f) __syncthreads();  // the stores of face f - 1 have read s_o
    const int nq = live && f < nf ? face_nq(p, p.ftype[c * MF + f]) : 0;
    for (int q = 0; q < QS; ++q) {
      T r = T(0);
      if (q < nq) {
        const T* xi = xq + (int64_t)(f * QS + q) * 3 * 32;
        T m[ID];
        monomials<P, T>(xi[0], xi[32], xi[64], m);
#pragma unroll
        for (int d = 0; d < ID; ++d) r += m[d] * gh[d];
        r = r - cb;
      }
      so[lane * RS + q * NV + v] = r;
    }
    __syncthreads();
    // CHECKSOL: warp v takes the points v, v + NV, ... of its lane's cell
    for (int q = v; q < nq; q += NV) {
      double uf[NV];
#pragma unroll
      for (int k = 0; k < NV; ++k) uf[k] = u0[k] + (double)so[lane * RS + q * NV + k];
      flag = flag || jump_bad(p.gamma, pm, uf, 0.85);
    }
    // the group's values of face f: one run of QS * NV per cell, warp v
    // storing the cells v, v + NV, ...
    for (int cl = v; cl < ncl; cl += NV)
      for (int r = lane; r < QS * NV; r += 32) out[(int64_t)cl * FQ * NV + f * QS * NV + r] = so[cl * RS + r];
  }
  if (flag) atomicOr(&s_flag[lane], 1);
  __syncthreads();
  if (tid < ncl) p.wflag[grp * 32 + tid] = (int8_t)s_flag[tid];
}

// k_wpost: one lane per cell, no block barriers.  Indicators and weights of
// CP_RECONSTRUCTION (src/reconstruct_p.f90:920-1250), the combined
// polynomial, its face values and CHECKSOL; flagged cells (and every cell of
// high-order MUSCL) take the central stencil polynomial limited by
// Venkatakrishnan, then CHECKSOLX (3126-3406).  Output: dul [n][F][QS][5],
// face value minus cell mean, 0 in unused slots.  A face value is
// sum_d m_d(x) g_d - sum_d mean(m_d) g_d: the second sum is formed once per
// polynomial instead of subtracting the basis means at every face point.
// ISB: the indicators come from k_wis (p.isb) instead of being formed here.
// FB: only the cells that k_wface marked in p.wflag, straight to the MUSCL
// fall-back (the others return at once).  MU (with FB): the first MOOD
// cascade, MUSCL on the cells of p.mmus without CHECKSOLX (MUSCL of
// MOOD_OPERATOR_2, mood.f90:353).
// Under MOOD (p.mprev) every cell is reconstructed; a reduced cell (CHECKSOL,
// or not FULL) takes the MUSCL fall-back only if the last MOOD pass
// recomputed it (RECALC, reconstruct_p.f90:2306-2315), else it keeps its
// WENO values and only CHECKSOLX; the reduced flags go to p.wflag.
// Three blocks of 128 per SM where that measured faster than the two that
// the kernel's registers otherwise allow: IORDER 2 (WENO3 tets, 82,944
// cells: 1.109 -> 1.083 ms per step mixed, 1.585 -> 1.540 FP64) and IORDER 3
// in FP32 (2.1 M-cell CWENO4 Navier-Stokes: 52.7 -> 51.2 ms; in FP64 the
// bound made the 647 k-cell step 31.8 -> 33.8 ms, so FP64 keeps two; four
// blocks in FP32 made it 56.0 -> 57.6 ms on another box).
template <int P, typename T, bool CH = false, bool ISB = false, bool FB = false, bool MU = false>
__global__ void __launch_bounds__(CH ? 64 : 128, !CH && (P == 2 || (P == 3 && sizeof(T) == 4)) ? 3 : 1)
    k_wpost(Problem p, const double* __restrict__ U) {
  constexpr int ID = Deg<P>::ideg;
  constexpr int VEC = Vec<T>::N;
  constexpr int L2 = ID < 9 ? ID : 9;  // CWENO lower order: IDEGFREE2 3 or 9 (grid_p.f90:6145-6160)
  constexpr int VI = WVars<T>::is, VH = WVars<T>::face, VF = WVars<T>::fall;
  // variables per pass of the characteristic face polynomial (its 5x5 FP64
  // combination matrices beside the polynomial).  Every pass reads all the
  // stencil polynomials again for each face, so fewer variables per pass
  // remove the spills (FP32: 978 bytes at 5, 16 at 2, none at 1) but cost
  // more: 64^3 WENO5 reconstruction 17.2 ms at 5, 21.1 at 3, 25.3 at 2,
  // 36.8 at 1 (FP32); FP64 52.6 ms at 3, 61.6 at 2, 78.5 at 1.
  constexpr int VC = WVars<T>::chr;
  constexpr int BT = CH ? 64 : 128;    // threads per block
  __shared__ double s_w[7 * NV * BT];  // per thread, [ll][v]: indicators, then weights
  __shared__ double s_e[CH ? 50 * BT : 1];  // per thread: left then right eigenvectors (characteristic form)
  const int tid = threadIdx.x;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + tid;
  if (c >= p.n) return;
  const int A = p.admis_max;
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const int FQ = MF * QS;
  const bool cw = p.ees == 5, weno = p.scheme == 3;
  const int ID2 = p.ideg2;
  const int adm = p.admis[c];
  const int nf = p.nfaces[c];
  const int64_t grp = c >> 5;
  const int lane = (int)(c & 31);
  // stencil polynomials G[ll][d][v], interleaved like the tables
  const T* Gc = (const T*)p.gbuf + grp * (int64_t)(A * ID * NV) * 32 + lane;
  auto G = [&](int ll, int d, int v) -> T { return Gc[(int64_t)((ll * ID + d) * NV + v) * 32]; };
  double u0[NV], pm[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u0[v] = U[c * NV + v];
  cons2prim(p.gamma, u0, pm);
  const T* xq = (const T*)p.qpts + grp * (int64_t)FQ * 3 * 32 + lane;  // interleaved
  const T* bmv = (const T*)p.bmean + grp * (int64_t)ID * 32 + lane;    // interleaved
  T* out = (T*)p.dul + c * FQ * NV;
  double* sw = s_w + tid;  // sw[(ll * NV + v) * BT]
  const double lc1 = 1.0 - 1.0 / p.lwci;
  const double lk = adm > 1 ? (1.0 - lc1) / (adm - 1) : 0.0;
  auto nq_of = [&](int f) { return f < nf ? face_nq(p, p.ftype[c * MF + f]) : 0; };
  // monomials at face point (f, q)
  auto mono = [&](int f, int q, T (&m)[ID]) {
    const T* xi = xq + (int64_t)(f * QS + q) * 3 * 32;
    monomials<P, T>(__ldcs(xi), __ldcs(xi + 32), __ldcs(xi + 64), m);
  };
  // g[d][k] = G(ll, d, v0 + k) for d < ndl, else 0
  auto load_poly = [&](int ll, int v0, auto& g, int ndl) {
    constexpr int ND = sizeof(g) / sizeof(g[0]);
    constexpr int VV = sizeof(g[0]) / sizeof(T);
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
      for (int k = 0; k < VV; ++k) g[d][k] = (v0 + k < NV && d < ndl) ? G(ll, d, v0 + k) : T(0);
  };
  // central stencil polynomial for variables v0, v0+1, ... (as many as g
  // holds); with `rem`, the CWENO form with the low-order stencils removed
  // (reconstruct_p.f90:956-965)
  auto load_g0 = [&](int v0, auto& g, bool rem) {
    constexpr int VV = sizeof(g[0]) / sizeof(T);
    load_poly(0, v0, g, ID);
    if (rem) {
      T g3[L2][VV];
#pragma unroll
      for (int d = 0; d < L2; ++d)
#pragma unroll
        for (int k = 0; k < VV; ++k) g3[d][k] = T(0);
      for (int l2 = 1; l2 < adm; ++l2)
#pragma unroll
        for (int d = 0; d < L2; ++d)
#pragma unroll
          for (int k = 0; k < VV; ++k)
            if (v0 + k < NV && d < ID2) g3[d][k] = g3[d][k] + T(lk) * G(l2, d, v0 + k);
#pragma unroll
      for (int d = 0; d < ID; ++d)
#pragma unroll
        for (int k = 0; k < VV; ++k)
          if (v0 + k < NV) g[d][k] = T(1.0 / lc1) * (g[d][k] - (d < L2 ? g3[d][k] : T(0)));
    }
  };
  // sum_d mean(m_d) g[d][k]
  auto mean_term = [&](const auto& g, auto& cb) {
    constexpr int VV = sizeof(g[0]) / sizeof(T);
#pragma unroll
    for (int k = 0; k < VV; ++k) cb[k] = T(0);
#pragma unroll
    for (int d = 0; d < ID; ++d) {
      const T b = bmv[d * 32];
#pragma unroll
      for (int k = 0; k < VV; ++k) cb[k] += b * g[d][k];
    }
  };

  // nonlinear weights in FP64 ((10E-12)^4 underflows FP32): sw holds the
  // indicators [ll][v] on entry and the weights on exit
  auto weights = [&]() {
    for (int v = 0; v < NV; ++v) {
      const double lam0 = cw ? lc1 : p.lwci, lamk = cw ? lk : 1.0;
      double tau = 0.0, sum = 0.0;
      if (cw && p.wenoz) {
        for (int ll = 0; ll < adm; ++ll) tau += fabs(sw[v * BT] - sw[(ll * NV + v) * BT]);
        tau = tau / (adm - 1);
      }
      for (int ll = 0; ll < adm; ++ll) {
        const double e = p.weno_eps + sw[(ll * NV + v) * BT];
        const double lam = ll == 0 ? lam0 : lamk;
        double wt;
        if (cw && p.wenoz) {
          double q = tau / e;
          q = q * q;
          wt = lam * (1.0 + q * q);
        } else {
          const double e2 = e * e;
          wt = lam / (e2 * e2);
        }
        sw[(ll * NV + v) * BT] = wt;
        sum += wt;
      }
      for (int ll = 0; ll < adm; ++ll) sw[(ll * NV + v) * BT] = sw[(ll * NV + v) * BT] / sum;
    }
  };
  const bool md = p.mprev != nullptr;
  if (FB && !(MU ? p.mmus[c] : p.wflag[c])) return;
  bool fall = FB || !weno || (!md && !p.full[c]);  // CHECKSOL: FULL = 0 -> REDUCE
  if (!CH && !fall && ISB) {
    // ---- smoothness indicators from k_wis
    const double* is = p.isb + grp * (int64_t)A * NV * 32 + lane;
    for (int ll = 0; ll < adm; ++ll)
#pragma unroll
      for (int v = 0; v < NV; ++v) sw[(ll * NV + v) * BT] = is[(int64_t)(ll * NV + v) * 32];
  } else if (!CH && !ISB && !fall) {
    // ---- smoothness indicators g^T S g per stencil and variable
    const T* Pc = (const T*)p.ind + grp * p.istride * 32 + lane * VEC;
    for (int ll = 0; ll < adm; ++ll) {
      const bool low = cw && ll > 0;
      for (int v0 = 0; v0 < NV; v0 += VI) {
        T is[VI];
#pragma unroll
        for (int k = 0; k < VI; ++k) is[k] = T(0);
        if (low) {
          T g[L2][VI];
          load_poly(ll, v0, g, ID2);
          quad_form<L2, VI>(Pc + (int64_t)(p.i2off / VEC) * 32 * VEC, g, ID2, is);
        } else {
          T g[ID][VI];
          if (ll == 0) load_g0(v0, g, cw);
          else load_poly(ll, v0, g, ID);
          quad_form<ID, VI>(Pc, g, ID, is);
        }
#pragma unroll
        for (int k = 0; k < VI; ++k)
          if (v0 + k < NV) sw[(ll * NV + v0 + k) * BT] = (double)is[k];
      }
    }
  }
  if (!CH && !fall) {
    weights();
    // ---- combined polynomial, face values, CHECKSOL (threshold 0.85)
    bool flag = false;
    for (int v0 = 0; v0 < NV; v0 += VH) {
      T gh[ID][VH];
      load_g0(v0, gh, cw);
#pragma unroll
      for (int k = 0; k < VH; ++k) {
        const T w0 = v0 + k < NV ? T(sw[(v0 + k) * BT]) : T(0);
#pragma unroll
        for (int d = 0; d < ID; ++d) gh[d][k] = w0 * gh[d][k];
      }
      for (int ll = 1; ll < adm; ++ll) {
        T wl[VH];
#pragma unroll
        for (int k = 0; k < VH; ++k) wl[k] = v0 + k < NV ? T(sw[(ll * NV + v0 + k) * BT]) : T(0);
#pragma unroll
        for (int d = 0; d < ID; ++d)
          if (!cw || d < ID2)
#pragma unroll
            for (int k = 0; k < VH; ++k)
              if (v0 + k < NV) gh[d][k] += wl[k] * G(ll, d, v0 + k);
      }
      T cb[VH];
      mean_term(gh, cb);
      for (int f = 0; f < MF; ++f) {
        const int nq = nq_of(f);
        for (int q = 0; q < QS; ++q) {
          T* o = out + (f * QS + q) * NV;
          if (q >= nq) {
#pragma unroll
            for (int k = 0; k < VH; ++k)
              if (v0 + k < NV) o[v0 + k] = T(0);
            continue;
          }
          T m[ID];
          mono(f, q, m);
          T res[VH];
#pragma unroll
          for (int k = 0; k < VH; ++k) {
            T r = T(0);
#pragma unroll
            for (int d = 0; d < ID; ++d) r += m[d] * gh[d][k];
            res[k] = r - cb[k];
            if (v0 + k < NV) o[v0 + k] = res[k];
          }
          if (VH == NV) {
            double uf[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) uf[v] = u0[v] + (double)res[v % VH];
            flag = flag || jump_bad(p.gamma, pm, uf, 0.85);
          }
        }
      }
    }
    if (VH < NV) {  // CHECKSOL on the stored face values
      for (int f = 0; f < nf; ++f) {
        const int nq = nq_of(f);
        for (int q = 0; q < nq; ++q) {
          const T* o = out + (f * QS + q) * NV;
          double uf[NV];
#pragma unroll
          for (int v = 0; v < NV; ++v) uf[v] = u0[v] + (double)o[v];
          flag = flag || jump_bad(p.gamma, pm, uf, 0.85);
        }
      }
    }
    fall = flag;
  }
  if (CH && !fall) {
    // ---- CHARACTERISTIC_RECONSTRUCTION (src/reconstruct_p.f90:497-758), per
    // face: eigenvectors at the average of the cell mean and the face
    // neighbour's mean (or the boundary ghost of the cell mean), both in the
    // face frame; stencil polynomials projected on the left eigenvectors
    // (global-frame conserved variables, as the reference projects them);
    // indicators and weights per characteristic variable; the face's
    // polynomial back-projected.  The indicator of the projection W = G EL^T
    // is EL_k^T (G^T S G) EL_k, so G^T S G is formed once per stencil and
    // each face only applies its eigenvectors.  With M_ll = ER diag(w_ll) EL the combined
    // conserved polynomial is sum_ll M_ll G_ll (rows d >= 1) and its mean
    // sum_ll M_ll u0, formed in FP64.
    const T* Pc = (const T*)p.ind + grp * p.istride * 32 + lane * VEC;
    double* EL = s_e + tid;            // EL[(k * NV + v) * BT]
    double* ER = s_e + 25 * BT + tid;  // ER[(v * NV + k) * BT]
    // stencil polynomial row d of variable u (CWENO: the central one with the
    // lower-order stencils removed, reconstruct_p.f90:1723-1737; g3 holds
    // sum_l2 lk * G(l2) for the rows d < IDEGFREE2)
    auto Gp = [&](int ll, int d, int u, const T (&g3)[L2][NV]) -> T {
      if (!(cw && ll == 0)) return G(ll, d, u);
      return T(1.0 / lc1) * (G(0, d, u) - (d < L2 ? g3[d][u] : T(0)));
    };
    auto lower_sum = [&](T (&g3)[L2][NV]) {
#pragma unroll
      for (int d = 0; d < L2; ++d)
#pragma unroll
        for (int u = 0; u < NV; ++u) g3[d][u] = T(0);
      if (!cw) return;
      for (int l2 = 1; l2 < adm; ++l2)
#pragma unroll
        for (int d = 0; d < L2; ++d)
          if (d < ID2)
#pragma unroll
            for (int u = 0; u < NV; ++u) g3[d][u] = g3[d][u] + T(lk) * G(l2, d, u);
    };
    // Q_l = G_l^T S G_l (symmetric 5x5, upper triangle row by row) once per
    // cell: the face-independent part of the characteristic indicators
    double* Qc = p.qbuf + grp * (int64_t)(A * 15) * 32 + lane;
#pragma unroll 1
    for (int ll = 0; ll < adm; ++ll) {
      const bool low = cw && ll > 0;
      T g3[L2][NV];
      lower_sum(g3);
      auto store = [&](int u, int w, double x) {
        Qc[(int64_t)(ll * 15 + (u * (2 * NV - u + 1)) / 2 + (w - u)) * 32] = x;
      };
      auto forms = [&](auto& g, const T* Pl, int nd) {
        constexpr int ND = sizeof(g) / sizeof(g[0]);
        constexpr int VG = sizeof(g[0]) / sizeof(T);
        if constexpr (VG == NV) {  // all five variables at once
#pragma unroll
          for (int d = 0; d < ND; ++d)
#pragma unroll
            for (int u = 0; u < NV; ++u) g[d][u] = d < nd ? Gp(ll, d, u, g3) : T(0);
          T a[NV][NV];
#pragma unroll
          for (int u = 0; u < NV; ++u)
#pragma unroll
            for (int w = 0; w < NV; ++w) a[u][w] = T(0);
          sym_form<ND, NV>(Pl, g, nd, a);
#pragma unroll
          for (int u = 0; u < NV; ++u)
#pragma unroll
            for (int w = u; w < NV; ++w) store(u, w, u == w ? (double)a[u][u] : 0.5 * ((double)a[u][w] + (double)a[w][u]));
        } else {  // pairs of variables
#pragma unroll 1
          for (int u = 0; u < NV; ++u)
#pragma unroll 1
            for (int w = u; w < NV; ++w) {
#pragma unroll
              for (int d = 0; d < ND; ++d) {
                g[d][0] = d < nd ? Gp(ll, d, u, g3) : T(0);
                g[d][1] = d < nd ? Gp(ll, d, w, g3) : T(0);
              }
              T a[2][2] = {{T(0), T(0)}, {T(0), T(0)}};
              sym_form<ND, 2>(Pl, g, nd, a);
              store(u, w, u == w ? (double)a[0][0] : 0.5 * ((double)a[0][1] + (double)a[1][0]));
            }
        }
      };
      constexpr int QV = sizeof(T) == 4 ? NV : 2;
      if (low) {
        T g[L2][QV];
        forms(g, Pc + (int64_t)(p.i2off / VEC) * 32 * VEC, ID2);
      } else {
        T g[ID][QV];
        forms(g, Pc, ID);
      }
    }
    bool flag = false;
    for (int f = 0; f < nf; ++f) {
      double r[4], ur[NV];
#pragma unroll
      for (int k = 0; k < 4; ++k) r[k] = p.rot[(c * MF + f) * 4 + k];
      const int64_t nb = p.neigh[c * MF + f];
      if (nb >= 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) ur[v] = U[nb * NV + v];
      } else {
        boundary_ghost(p, p.bc[c * MF + f], r, u0, ur);
      }
      {
        double rl[NV], rr[NV];
        rot_f(r, u0, rl);
        rot_f(r, ur, rr);
        char_eigenvectors(p.gamma, rl, rr, EL, ER, BT);
      }
      // indicators of the projected polynomials: IS_l[k] = EL_k^T Q_l EL_k
#pragma unroll 1
      for (int ll = 0; ll < adm; ++ll) {
        double q[15];
#pragma unroll
        for (int j = 0; j < 15; ++j) q[j] = Qc[(int64_t)(ll * 15 + j) * 32];
#pragma unroll 1
        for (int k = 0; k < NV; ++k) {
          double l[NV];
#pragma unroll
          for (int u = 0; u < NV; ++u) l[u] = EL[(k * NV + u) * BT];
          double is = 0.0;
          int j = 0;
#pragma unroll
          for (int u = 0; u < NV; ++u)
#pragma unroll
            for (int w = u; w < NV; ++w, ++j) is += (u == w ? 1.0 : 2.0) * l[u] * l[w] * q[j];
          sw[(ll * NV + k) * BT] = is;
        }
      }
      weights();
      // the face's polynomial in conserved variables, VC at a time
      const int nq = face_nq(p, p.ftype[c * MF + f]);
#pragma unroll 1
      for (int v0 = 0; v0 < NV; v0 += VC) {
        T gh[ID][VC];
        double f0[VC];
#pragma unroll
        for (int k = 0; k < VC; ++k) {
          f0[k] = 0.0;
#pragma unroll
          for (int d = 0; d < ID; ++d) gh[d][k] = T(0);
        }
#pragma unroll 1
        for (int ll = 0; ll < adm; ++ll) {
          const int nd = cw && ll > 0 ? ID2 : ID;
          T g3[L2][NV];
          if (ll == 0) lower_sum(g3);
          double M[VC][NV];
#pragma unroll
          for (int k = 0; k < VC; ++k)
#pragma unroll
            for (int u = 0; u < NV; ++u) {
              double a = 0.0;
              if (v0 + k < NV)
#pragma unroll
                for (int j = 0; j < NV; ++j)
                  a += ER[((v0 + k) * NV + j) * BT] * sw[(ll * NV + j) * BT] * EL[(j * NV + u) * BT];
              M[k][u] = a;
            }
#pragma unroll
          for (int k = 0; k < VC; ++k)
#pragma unroll
            for (int u = 0; u < NV; ++u) f0[k] += M[k][u] * u0[u];
#pragma unroll
          for (int d = 0; d < ID; ++d)
            if (d < nd) {
              T gu[NV];
#pragma unroll
              for (int u = 0; u < NV; ++u) gu[u] = Gp(ll, d, u, g3);
#pragma unroll
              for (int k = 0; k < VC; ++k)
#pragma unroll
                for (int u = 0; u < NV; ++u) gh[d][k] += T(M[k][u]) * gu[u];
            }
        }
        T cb[VC];
        mean_term(gh, cb);
        for (int q = 0; q < QS; ++q) {
          T* o = out + (f * QS + q) * NV;
          if (q >= nq) {
#pragma unroll
            for (int k = 0; k < VC; ++k)
              if (v0 + k < NV) o[v0 + k] = T(0);
            continue;
          }
          T m[ID];
          mono(f, q, m);
#pragma unroll
          for (int k = 0; k < VC; ++k) {
            T rsum = T(0);
#pragma unroll
            for (int d = 0; d < ID; ++d) rsum += m[d] * gh[d][k];
            if (v0 + k < NV) o[v0 + k] = T((f0[k] - u0[v0 + k]) + (double)(rsum - cb[k]));
          }
        }
      }
      // CHECKSOL on this face's stored values
      for (int q = 0; q < nq; ++q) {
        const T* o = out + (f * QS + q) * NV;
        double uf[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) uf[v] = u0[v] + (double)o[v];
        flag = flag || jump_bad(p.gamma, pm, uf, 0.85);
      }
    }
    for (int f = nf; f < MF; ++f)
      for (int q = 0; q < QS; ++q)
#pragma unroll
        for (int v = 0; v < NV; ++v) out[(f * QS + q) * NV + v] = T(0);
    fall = flag;
  }
  // CHECKSOLX (threshold 0.95) cannot fire where the 0.85 test passed on the
  // same face values
  bool mus = fall, chkx = fall;
  if (md && !FB && weno) {  // MOOD: the fall-back only where RECALC
    const bool reduce = fall || !p.full[c];
    p.wflag[c] = reduce ? 1 : 0;
    mus = reduce && p.mprev[c];
    chkx = reduce;
  } else if (md && FB && !MU) {
    mus = p.mprev[c];
  }
  if (MU) chkx = false;
  if (!mus && !chkx) return;

  if (mus) {
    // ---- MUSCL with the central stencil polynomial (FIND_BOUNDS + Venkatakrishnan)
    double lo[NV], hi[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) lo[v] = hi[v] = u0[v];
    for (int f = 0; f < nf; ++f) {
      const int64_t nb = p.neigh[c * MF + f];
      if (nb < 0) continue;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double un = U[nb * NV + v];
        lo[v] = fmin(lo[v], un);
        hi[v] = fmax(hi[v], un);
      }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      lo[v] -= u0[v];
      hi[v] -= u0[v];
    }
    const double e3 = p.kappa_ven * p.minedge[c];
    const double epsi2 = e3 * e3 * e3;
    for (int v0 = 0; v0 < NV; v0 += VF) {
      T g0[ID][VF];
      load_poly(0, v0, g0, ID);
      T cb[VF];
      mean_term(g0, cb);
      double slope[VF];
#pragma unroll
      for (int k = 0; k < VF; ++k) slope[k] = TOLBIG;
      for (int pass = 0; pass < 2; ++pass) {
        for (int f = 0; f < MF; ++f) {
          const int nq = nq_of(f);
          for (int q = 0; q < QS; ++q) {
            T* o = out + (f * QS + q) * NV;
            if (q >= nq) {
              if (pass == 1)
#pragma unroll
                for (int k = 0; k < VF; ++k)
                  if (v0 + k < NV) o[v0 + k] = T(0);
              continue;
            }
            T m[ID];
            mono(f, q, m);
#pragma unroll
            for (int k = 0; k < VF; ++k) {
              const int v = v0 + k;
              if (v >= NV) continue;
              T r = T(0);
#pragma unroll
              for (int d = 0; d < ID; ++d) r += m[d] * g0[d][k];
              r = r - cb[k];
              const double dd = (u0[v] + (double)r) - u0[v];
              if (pass == 0) slope[k] = fmin(slope[k], slope_limiter(p.limiter, dd, lo[v], hi[v], epsi2));
              else o[v] = T((double)T(dd) * slope[k]);
            }
          }
        }
      }
    }
  }
  if (!chkx) return;
  // ---- CHECKSOLX: first order where a face value jumps by 95 %
  bool bad = false;
  for (int f = 0; f < nf; ++f) {
    const int nq = nq_of(f);
    for (int q = 0; q < nq; ++q) {
      const T* o = out + (f * QS + q) * NV;
      double uf[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) uf[v] = u0[v] + (double)o[v];
      bad = bad || jump_bad(p.gamma, pm, uf, 0.95);
    }
  }
  if (bad)
    for (int i = 0; i < FQ * NV; ++i) out[i] = T(0);
}

// ======================================================================
// Viscous gradients for WENO/CWENO + Navier-Stokes: LSQ on (T,u,v,w) with
// stencil 1 (gradients.f90:502-706), then face gradients (SOLUTIONTRIAV2).
// ======================================================================
// One lane per cell: each stencil member's primitive state is formed once
// and its differences (T, u, v, w) are accumulated for VP variables per pass
// (all four when the FP64 accumulators fit), reading the interleaved table
// rows of stencil 1 with coalesced loads.  Same products and order per
// (row, variable) as one thread per variable.
// T = p / (rho R), u, v, w of every cell, formed once per stage: the viscous
// least squares then gathers 32-byte records (two 16-byte loads, no
// division) instead of forming them from the conserved state per member.
template <int P, typename T>
__global__ void k_visc_prim(Problem p, const double* __restrict__ U) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  double pm[NV];
  cons2prim(p.gamma, U + c * NV, pm);
  double2* o = (double2*)(p.prim + c * 4);
  o[0] = make_double2(pm[4] / (pm[0] * p.r_gas), pm[1]);
  o[1] = make_double2(pm[2], pm[3]);
}

// Accumulated in the table precision T: FP64 in the FP64 form; in the mixed
// form FP32 on the differences of (T, u, v, w) from the cell's own, like
// the stencil least squares of the conserved variables (all four variables
// in one pass there).
template <int P, typename T>
__global__ void __launch_bounds__(128) k_visc_lsq(Problem p, const double* __restrict__ U) {
  constexpr int ID = Deg<P>::ideg;
  constexpr int VP = sizeof(T) == 4 || ID * 4 <= 80 ? 4 : 2;  // variables per pass
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= p.n) return;
  const int IM = p.imax, W = IM + 1;
  double pm[NV];
  cons2prim(p.gamma, U + c * NV, pm);
  const double s0[4] = {pm[4] / (pm[0] * p.r_gas), pm[1], pm[2], pm[3]};
  const int64_t grp = c >> 5;
  const int lane = (int)(c & 31);
  const int32_t* st = p.sten + grp * (int64_t)p.admis_max * W * 32 + lane;
  const T* M = (const T*)p.invmat + (grp * p.tstride + p.soff[0]) * 32 + lane;
  T* gv = (T*)p.gv;
#pragma unroll 1
  for (int v0 = 0; v0 < 4; v0 += VP) {
    T acc[ID][VP];
#pragma unroll
    for (int d = 0; d < ID; ++d)
#pragma unroll
      for (int j = 0; j < VP; ++j) acc[d][j] = T(0);
    for (int k = 0; k < IM; ++k) {
      const double2* q = (const double2*)(p.prim + (int64_t)st[(k + 1) * 32] * 4);
      const double2 qa = q[0], qb = q[1];
      const double sy[4] = {qa.x, qa.y, qb.x, qb.y};
      T ds[VP];
#pragma unroll
      for (int j = 0; j < VP; ++j) ds[j] = T(sy[v0 + j] - s0[v0 + j]);
#pragma unroll
      for (int d = 0; d < ID; ++d) {
        const T m = M[(k * ID + d) * 32];
#pragma unroll
        for (int j = 0; j < VP; ++j) acc[d][j] += m * ds[j];
      }
    }
    // 16-byte stores: a row's four FP32 values, or FP64 pairs (VP even;
    // rows are 16- and 32-byte aligned)
#pragma unroll
    for (int d = 0; d < ID; ++d) {
      if constexpr (sizeof(T) == 4) {
        *(float4*)(gv + (c * ID + d) * 4) = make_float4(acc[d][0], acc[d][1], acc[d][2], acc[d][3]);
      } else {
#pragma unroll
        for (int j = 0; j < VP; j += 2)
          *(double2*)(gv + (c * ID + d) * 4 + v0 + j) = make_double2(acc[d][j], acc[d][j + 1]);
      }
    }
  }
}

// Face-point gradients of T, u, v, w for the viscous flux, one thread per
// (owned face, point): SOLUTIONTRIAV2 (reconstruct_p.f90:2358) on
// both sides of the face at the paired points, and their average, the only
// form CALCULATE_FLUXESHI_DIFFUSIVE uses (flux_p.f90:1614-1779), written
// once per face point to p.fgrad [nown][QS][12] (half the bytes of one
// record per cell face and point, read back once instead of twice).
// evaluated in T (FP32 in the mixed form, from the FP32 coefficients and
// reference-frame points)
template <int P, typename T>
__device__ __forceinline__ void visc_point_grad(const Problem& p, int64_t c, int f, int q, int QS, T* out) {
  constexpr int ID = Deg<P>::ideg;
  const T* xi = (const T*)p.qpts + ((c >> 5) * MF * QS * 3 + (f * QS + q) * 3) * 32 + (c & 31);
  T dx[ID], dy[ID], dz[ID];
  dmonomials<P, T>(xi[0], xi[32], xi[64], dx, dy, dz);
  const double* J = p.jinv + c * 9;
  const T* gv = (const T*)p.gv + c * ID * 4;
  if constexpr (sizeof(T) == 4) {
    // FP32: a coefficient row's four variables in one 16-byte load (the
    // scalar loads kept k_visc_facegrad at 80 % of L1 throughput; 2.1 M-cell
    // CWENO4: 52.7 -> 51.8 ms per step); each variable's sum still runs over
    // the rows in order, so the values are the same bit for bit
    T gl[4][3];
#pragma unroll
    for (int var = 0; var < 4; ++var) gl[var][0] = gl[var][1] = gl[var][2] = T(0);
#pragma unroll
    for (int d = 0; d < ID; ++d) {
      const float4 a = *(const float4*)(gv + d * 4);
      const T g[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
      for (int var = 0; var < 4; ++var) {
        gl[var][0] += g[var] * dx[d];
        gl[var][1] += g[var] * dy[d];
        gl[var][2] += g[var] * dz[d];
      }
    }
#pragma unroll
    for (int var = 0; var < 4; ++var)
#pragma unroll
      for (int k = 0; k < 3; ++k)
        out[var * 3 + k] = T(J[0 * 3 + k]) * gl[var][0] + T(J[1 * 3 + k]) * gl[var][1] + T(J[2 * 3 + k]) * gl[var][2];
  } else {
#pragma unroll
    for (int var = 0; var < 4; ++var) {
      T gl[3] = {T(0), T(0), T(0)};
#pragma unroll
      for (int d = 0; d < ID; ++d) {
        const T g = gv[d * 4 + var];
        gl[0] += g * dx[d];
        gl[1] += g * dy[d];
        gl[2] += g * dz[d];
      }
#pragma unroll
      for (int k = 0; k < 3; ++k)
        out[var * 3 + k] = T(J[0 * 3 + k]) * gl[0] + T(J[1 * 3 + k]) * gl[1] + T(J[2 * 3 + k]) * gl[2];
    }
  }
}

template <int P, typename T>
__global__ void k_visc_facegrad(Problem p) {
  const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = t / QS;
  const int q = (int)(t - i * QS);
  if (i >= p.nown) return;
  const int32_t code = p.own[i];
  const int64_t c = code >> 3;
  const int f = code & 7;
  const int64_t nb = p.neigh[c * MF + f];
  if (q >= face_nq(p, p.ftype[c * MF + f])) return;
  T gl[12], gr[12];
  visc_point_grad<P, T>(p, c, f, q, QS, gl);
  if (nb >= 0) {
    visc_point_grad<P, T>(p, nb, p.nface[c * MF + f], p.qperm[(c * MF + f) * QS + q], QS, gr);
  } else {  // physical boundary: the ghost side takes the cell's own gradient
#pragma unroll
    for (int k = 0; k < 12; ++k) gr[k] = gl[k];
  }
  double2* o = (double2*)(p.fgrad + (i * QS + q) * 12);
#pragma unroll
  for (int k = 0; k < 6; ++k)
    o[k] = make_double2((double)((gl[2 * k] + gr[2 * k]) / T(2)), (double)((gl[2 * k + 1] + gr[2 * k + 1]) / T(2)));
}

// Characteristic-variable post-processing (k_wpost<P, T, true>), 64 threads
// per block for its shared eigenvectors.  Instantiated only in
// recon_char_*.cu (explicit instantiations), which nvcc compiles in parallel
// with the other reconstruction units.
template <int P, typename T>
cudaError_t launch_wpost_char(const Problem& p, const double* U, cudaStream_t st) {
  k_wpost<P, T, true><<<(unsigned)((p.n + 63) / 64), 64, 0, st>>>(p, U);
  return cudaGetLastError();
}
#ifndef UCG_RECON_CHAR_TU
extern template cudaError_t launch_wpost_char<1, float>(const Problem&, const double*, cudaStream_t);
extern template cudaError_t launch_wpost_char<2, float>(const Problem&, const double*, cudaStream_t);
extern template cudaError_t launch_wpost_char<3, float>(const Problem&, const double*, cudaStream_t);
extern template cudaError_t launch_wpost_char<4, float>(const Problem&, const double*, cudaStream_t);
extern template cudaError_t launch_wpost_char<1, double>(const Problem&, const double*, cudaStream_t);
extern template cudaError_t launch_wpost_char<2, double>(const Problem&, const double*, cudaStream_t);
extern template cudaError_t launch_wpost_char<3, double>(const Problem&, const double*, cudaStream_t);
extern template cudaError_t launch_wpost_char<4, double>(const Problem&, const double*, cudaStream_t);
#endif

// One reconstruction: stencil polynomials, WENO post-processing and, for
// Navier-Stokes, the viscous LSQ and face gradients.  Instantiated per
// precision and order in recon_*.cu, which nvcc compiles in parallel.
// `mark`, if not null, is recorded between k_lsq and k_wpost (kernel timing).
template <int P, typename T>
cudaError_t launch_weno_t(const Problem& p, const double* U, bool ns, int QS, cudaStream_t st, int64_t* launches,
                          cudaEvent_t mark) {
  const unsigned b = (unsigned)((p.n + 127) / 128);
  // the per-cell records that the stencils gather cover every cell, also
  // those past the reconstructed prefix of a partition (p.n < p.nall)
  Problem pa = p;
  pa.n = p.nall > p.n ? p.nall : p.n;
  if (p.mmus) {  // the first MOOD cascade: MUSCL of the selected cells from this stage's G
    k_wpost<P, T, false, false, true, true><<<b, 128, 0, st>>>(p, U);
    ++*launches;
    return cudaGetLastError();
  }
  if (p.lsq_bulk) {  // opt-in: tables staged through shared memory (UCG_LSQ_BULK=1)
    constexpr int NSTG = 4;
    constexpr size_t smem = lsq_tma_smem<P, T, NSTG>();
    cudaFuncSetAttribute(k_lsq_tma<P, T, NSTG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_lsq_tma<P, T, NSTG><<<b, 128, smem, st>>>(p, U);
  } else if (P == 3) {
    // padded records: 6.9 -> 4.7 ms per stage for CWENO4 at 2.1 M cells; on
    // B200 the vector gather doubled k_lsq's time at IORDER 4 (255
    // registers: it breaks the load schedule) and made IORDER 2 slower by a
    // third, so those keep five 8-byte loads
    k_pad_state<P, T><<<(unsigned)((pa.n + 255) / 256), 256, 0, st>>>(pa, U);
    k_lsq<P, T, (P == 3)><<<b, 128, 0, st>>>(p, U);
    ++*launches;
  } else {
    k_lsq<P, T><<<b, 128, 0, st>>>(p, U);
  }
  if (mark) cudaEventRecord(mark, st);
  if (p.wenwrt == 2) {
    const cudaError_t e = launch_wpost_char<P, T>(p, U, st);
    if (e != cudaSuccess) return e;
  } else {
    // indicators in their own kernel at IORDER 4, where the cell's packed
    // triangle (595 entries) no longer stays in L1 between the stencils of
    // one lane (64^3 WENO5: FP64 stage 17.2 -> 15.5 ms, mixed 7.80 -> 7.67 ms);
    // at IORDER 2-3 the triangle is small and the extra kernel costs more
    // than it saves (2.1 M-cell CWENO4: 17.3 -> 19.6 ms)
    bool done = false;
    if constexpr (P == 4) {
      if (p.wface && p.isb && p.scheme == 3) {
        const int QS = p.nq_quad > p.nq_tri ? p.nq_quad : p.nq_tri;
        const size_t smem = ((size_t)MF * QS * 3 + ((QS * NV) | 1)) * 32 * sizeof(T);
        cudaFuncSetAttribute(k_wface<P, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_wis<P, T><<<(unsigned)((p.n + 31) / 32), 32 * p.admis_max, 0, st>>>(p);
        k_wface<P, T><<<(unsigned)((p.n + 31) / 32), 32 * NV, smem, st>>>(p, U);
        k_wpost<P, T, false, false, true><<<b, 128, 0, st>>>(p, U);
        *launches += 2;
        done = true;
      }
    }
    if constexpr (P == 4) {
      if (!done && p.isb && p.scheme == 3) {
        k_wis<P, T><<<(unsigned)((p.n + 31) / 32), 32 * p.admis_max, 0, st>>>(p);
        k_wpost<P, T, false, true><<<b, 128, 0, st>>>(p, U);
        ++*launches;
        done = true;
      }
    }
    if (!done) k_wpost<P, T><<<b, 128, 0, st>>>(p, U);
  }
  *launches += 2;
  if (ns) {
    k_visc_prim<P, T><<<(unsigned)((pa.n + 255) / 256), 256, 0, st>>>(pa, U);
    k_visc_lsq<P, T><<<(unsigned)((p.n + 127) / 128), 128, 0, st>>>(p, U);
    *launches += 2;
    const int64_t nfp = p.nown * QS;
    k_visc_facegrad<P, T><<<(unsigned)((nfp + 127) / 128), 128, 0, st>>>(p);
    *launches += 1;
  }
  return cudaGetLastError();
}

// precision-specific entry points (recon_f32.cu + recon_f32_p4.cu, recon_f64.cu +
// recon_f64_p4.cu; characteristic post-processing in recon_char*.cu);
// iorder 1..4, anything else returns cudaErrorInvalidValue
cudaError_t launch_weno_f32(int iorder, const Problem& p, const double* U, bool ns, int QS, cudaStream_t st,
                            int64_t* launches, cudaEvent_t mark);
cudaError_t launch_weno_f32_p4(const Problem& p, const double* U, bool ns, int QS, cudaStream_t st,
                               int64_t* launches, cudaEvent_t mark);
cudaError_t launch_weno_f64(int iorder, const Problem& p, const double* U, bool ns, int QS, cudaStream_t st,
                            int64_t* launches, cudaEvent_t mark);
cudaError_t launch_weno_f64_p4(const Problem& p, const double* U, bool ns, int QS, cudaStream_t st,
                               int64_t* launches, cudaEvent_t mark);
// the stencil least squares alone (FP64 tables) into p.gbuf: G is linear in
// U, so applied to a tangent dU it gives the tangent dG (adjoint.cu)
cudaError_t launch_lsq_f64(int iorder, const Problem& p, const double* U, cudaStream_t st);
cudaError_t launch_lsq_f64_p4(const Problem& p, const double* U, cudaStream_t st);

}  // namespace ucg
