// Characteristic-variable WENO post-processing, IORDER 1-3, both precisions.
#define UCG_RECON_CHAR_TU
#include "recon2.cuh"

namespace ucg {

template cudaError_t launch_wpost_char<1, float>(const Problem&, const double*, cudaStream_t);
template cudaError_t launch_wpost_char<2, float>(const Problem&, const double*, cudaStream_t);
template cudaError_t launch_wpost_char<3, float>(const Problem&, const double*, cudaStream_t);
template cudaError_t launch_wpost_char<1, double>(const Problem&, const double*, cudaStream_t);
template cudaError_t launch_wpost_char<2, double>(const Problem&, const double*, cudaStream_t);
template cudaError_t launch_wpost_char<3, double>(const Problem&, const double*, cudaStream_t);

}  // namespace ucg
