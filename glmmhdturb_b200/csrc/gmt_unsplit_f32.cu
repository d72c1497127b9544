// FP32 unsplit step kernels: 256 threads, 2 resident blocks per SM (<= 128 registers).
#include "gmt_unsplit_inst.cuh"

namespace gmt {
cudaError_t launch_unsplit(const UnsplitArgs<float>& A, int recon, int riem, cudaStream_t s) {
    return unsplit_dispatch<float, 256, 2>(A, recon, riem, s);
}
int unsplit_regs_f32(int recon, int riem) { return unsplit_regs_of<float, 256, 2>(recon, riem); }
}  // namespace gmt
