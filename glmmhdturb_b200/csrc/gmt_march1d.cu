// gmt_march1d.cu -- FP64 species pass of the march scheme (gmt_species.cuh), built with
// --fmad=false so that it evaluates the oracle's IEEE expressions.
#include "gmt_species.cuh"

namespace gmt {
cudaError_t launch_species(const MarchArgs<double>& A, const double* fmass, cudaStream_t s) {
    return species_go(A, fmass, s);
}
}  // namespace gmt
