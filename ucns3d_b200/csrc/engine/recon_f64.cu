// FP64 reconstruction kernels, IORDER 1-3, and the dispatch over IORDER;
// IORDER 4 lives in recon_f64_p4.cu.
#include "recon2.cuh"

namespace ucg {

cudaError_t launch_weno_f64(int iorder, const Problem& p, const double* U, bool ns, int QS, cudaStream_t st,
                            int64_t* launches, cudaEvent_t mark) {
  switch (iorder) {
    case 1: return launch_weno_t<1, double>(p, U, ns, QS, st, launches, mark);
    case 2: return launch_weno_t<2, double>(p, U, ns, QS, st, launches, mark);
    case 3: return launch_weno_t<3, double>(p, U, ns, QS, st, launches, mark);
    case 4: return launch_weno_f64_p4(p, U, ns, QS, st, launches, mark);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_lsq_f64(int iorder, const Problem& p, const double* U, cudaStream_t st) {
  const unsigned b = (unsigned)((p.n + 127) / 128);
  switch (iorder) {
    case 1: k_lsq<1, double><<<b, 128, 0, st>>>(p, U); break;
    case 2: k_lsq<2, double><<<b, 128, 0, st>>>(p, U); break;
    case 3: k_lsq<3, double><<<b, 128, 0, st>>>(p, U); break;
    case 4: return launch_lsq_f64_p4(p, U, st);
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace ucg
