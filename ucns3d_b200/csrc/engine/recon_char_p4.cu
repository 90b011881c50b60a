// Characteristic-variable WENO post-processing, IORDER 4 (WENO5), both
// precisions: the largest characteristic instantiations, compiled on their own.
#define UCG_RECON_CHAR_TU
#include "recon2.cuh"

namespace ucg {

template cudaError_t launch_wpost_char<4, float>(const Problem&, const double*, cudaStream_t);
template cudaError_t launch_wpost_char<4, double>(const Problem&, const double*, cudaStream_t);

}  // namespace ucg
