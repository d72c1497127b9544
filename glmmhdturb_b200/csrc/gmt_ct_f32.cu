// FP32 constrained-transport step kernels (gmt_ct_tile.cuh), built with --use_fast_math like the
// reference's own kernels (march_bridge/build_mhd.sh:25).  Tiles up to 512 threads, one block
// per SM.
#include "gmt_ct_tile.cuh"

namespace gmt {
cudaError_t launch_ct(const CTArgs<float>& A, cudaStream_t s) {
    if (A.ox * A.oy > 256) return ct_dispatch_t<float, 512, 1>(A, A.recon, A.riem, s, false);
    return ct_dispatch_t<float, 256, 2>(A, A.recon, A.riem, s, false);
}
cudaError_t ct_prepare_f32() {
    cudaError_t e = ct_configure_all_t<float, 512, 1>();
    if (e == cudaSuccess) e = ct_configure_all_t<float, 256, 2>();
    return e;
}
int ct_regs_f32(int recon, int riem, int nthreads) {
    return nthreads > 256 ? ct_regs_of_t<float, 512, 1>(recon, riem) : ct_regs_of_t<float, 256, 2>(recon, riem);
}
}  // namespace gmt
