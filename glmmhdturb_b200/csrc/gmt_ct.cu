// FP64 constrained-transport step kernels (gmt_ct_tile.cuh), built with --fmad=false so that each
// expression rounds as the oracle's IEEE evaluation; tiles up to 256 threads.  Also the size and
// register queries of both precisions.
#include "gmt_ct_tile.cuh"

namespace gmt {
int ct_regs_f32(int recon, int riem, int nthreads);

cudaError_t launch_ct(const CTArgs<double>& A, cudaStream_t s) {
    if (A.ox * A.oy > 256) return cudaErrorInvalidConfiguration;
    return ct_dispatch_t<double, 256, 1>(A, A.recon, A.riem, s, false);
}
cudaError_t ct_prepare_f64() { return ct_configure_all_t<double, 256, 1>(); }
int ct_regs_of(int dtype_bytes, int recon, int riem, int nthreads) {
    return dtype_bytes == 8 ? ct_regs_of_t<double, 256, 1>(recon, riem) : ct_regs_f32(recon, riem, nthreads);
}
size_t ct_smem_of(int dtype_bytes, int ox, int oy) {
    return dtype_bytes == 8 ? ct_tile_smem_bytes<double>(ox, oy) : ct_tile_smem_bytes<float>(ox, oy);
}
int ct_max_threads(int dtype_bytes) { return dtype_bytes == 8 ? 256 : 512; }
}  // namespace gmt
