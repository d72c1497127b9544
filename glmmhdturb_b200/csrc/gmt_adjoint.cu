// gmt_adjoint.cu -- FP64 instantiation of the adjoint kernels (gmt_adjoint_kern.cuh), built with
// --fmad=false like the FP64 forward step.
#include "gmt_adjoint_kern.cuh"

namespace gmt {
size_t adjoint_scratch_reals(size_t n) { return (size_t)(54 + 27 + 9 + 54 + 63) * n; }
template cudaError_t launch_adjoint<double>(const AdjArgs<double>&, const UnsplitArgs<double>*, cudaStream_t);
}  // namespace gmt
