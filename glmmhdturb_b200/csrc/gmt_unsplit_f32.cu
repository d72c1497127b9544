// FP32 unsplit step kernels, built with --use_fast_math (approximate reciprocal and square root,
// as the reference's own kernels are built, march_bridge/build_mhd.sh:25).  Two block shapes:
// up to 256 threads with 2 resident blocks per SM (<= 128 registers), and up to 512 threads with
// one block per SM for the larger tiles.
#include "gmt_unsplit_inst.cuh"

namespace gmt {
cudaError_t launch_unsplit(const UnsplitArgs<float>& A, int recon, int riem, cudaStream_t s) {
    if (A.ox * A.oy > 256) return unsplit_dispatch_t<float, 512, 1>(A, recon, riem, s);
    return unsplit_dispatch_t<float, 256, 2>(A, recon, riem, s);
}
int unsplit_regs_f32(int recon, int riem, int nthreads) {
    return nthreads > 256 ? unsplit_regs_of_t<float, 512, 1>(recon, riem) : unsplit_regs_of_t<float, 256, 2>(recon, riem);
}
}  // namespace gmt
