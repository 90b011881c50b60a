// FP64 reconstruction kernels, IORDER 4 (WENO5): the largest FP64
// instantiation, compiled on its own.
#include "recon2.cuh"

namespace ucg {

cudaError_t launch_weno_f64_p4(const Problem& p, const double* U, bool ns, int QS, cudaStream_t st,
                               int64_t* launches, cudaEvent_t mark) {
  return launch_weno_t<4, double>(p, U, ns, QS, st, launches, mark);
}

cudaError_t launch_lsq_f64_p4(const Problem& p, const double* U, cudaStream_t st) {
  k_lsq<4, double><<<(unsigned)((p.n + 127) / 128), 128, 0, st>>>(p, U);
  return cudaGetLastError();
}

}  // namespace ucg
