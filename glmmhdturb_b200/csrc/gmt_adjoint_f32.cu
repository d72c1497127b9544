// gmt_adjoint_f32.cu -- FP32 instantiation of the adjoint kernels (gmt_adjoint_kern.cuh), built with
// --use_fast_math like the FP32 forward step (the gradient is an FP32 quantity either way).
#include "gmt_adjoint_kern.cuh"

namespace gmt {
template cudaError_t launch_adjoint<float>(const AdjArgs<float>&, const UnsplitArgs<float>*, cudaStream_t);
}  // namespace gmt
