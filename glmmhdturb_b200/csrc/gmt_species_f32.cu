// gmt_species_f32.cu -- FP32 species pass of the march scheme (gmt_species.cuh), built with fast
// math like the FP32 march step it follows.
#include "gmt_species.cuh"

namespace gmt {
cudaError_t launch_species(const MarchArgs<float>& A, const float* fmass, cudaStream_t s) {
    return species_go(A, fmass, s);
}
}  // namespace gmt
