// The per-cell table expansion into the engine's interleaved layout
// (k_expand_il), shared by the table upload (engine.cu) and the device
// set-up (setup.cu).
#pragma once

#include <cstdint>

namespace ucg {

// ======================================================================
// Interleaved layout: row j of cell c goes to ((c/32)*len + j)*32 + c%32
// (VEC = 1), or vector-interleaved to (((c/32)*len/VEC + j/VEC)*32 + c%32)*VEC
// + j%VEC (len a multiple of VEC).  One block moves a 32-cell x 64-row tile
// through shared memory, so both the per-cell source rows and the
// interleaved destination are accessed in contiguous runs.  Cells outside
// [first, first+count) or whose table set is outside [tlo, thi) are left
// untouched.  With `rowmap` (renumbered cells), device cell c takes source
// row rowmap[c] (-1: not in this upload) and every group of `n` cells is
// visited; otherwise cells [first, first + count) take rows 0.. in order.
template <typename D, typename S, int VEC>
__global__ void __launch_bounds__(256) k_expand_il(D* __restrict__ dst, const S* __restrict__ src,
                                                   const int32_t* __restrict__ tid, int64_t first, int64_t count,
                                                   int64_t len, int64_t tlo, int64_t thi,
                                                   const int32_t* __restrict__ rowmap = nullptr, int64_t n = 0) {
  __shared__ S tile[32][65];
  __shared__ int64_t trow[32];
  const int64_t g0 = rowmap ? 0 : first >> 5, g1 = rowmap ? (n - 1) >> 5 : (first + count - 1) >> 5;
  const int64_t ntile = (len + 63) / 64, nblk = (g1 - g0 + 1) * ntile;
  for (int64_t b = blockIdx.x; b < nblk; b += gridDim.x) {
    const int64_t g = g0 + b / ntile, j0 = (b % ntile) * 64;
    if (threadIdx.x < 32) {
      const int64_t c = g * 32 + threadIdx.x;
      int64_t t = -1;
      const int64_t cl = rowmap ? (c < n ? rowmap[c] : -1) : (c >= first && c < first + count ? c - first : -1);
      if (cl >= 0) {
        t = tid ? tid[cl] : cl;
        if (t < tlo || t >= thi) t = -1;
      }
      trow[threadIdx.x] = t;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 32 * 64; i += blockDim.x) {
      const int cell = i >> 6, jj = i & 63;
      const int64_t t = trow[cell];
      if (t >= 0 && j0 + jj < len) tile[cell][jj] = src[(t - tlo) * len + j0 + jj];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 64 * 32; i += blockDim.x) {
      const int r = i % VEC, lane = (i / VEC) & 31, jj = (i / (VEC * 32)) * VEC + r;
      const int64_t j = j0 + jj;
      if (trow[lane] >= 0 && j < len) dst[((g * len + j - r) * 32 + lane * VEC) + r] = D(tile[lane][jj]);
    }
    __syncthreads();
  }
}

}  // namespace ucg
