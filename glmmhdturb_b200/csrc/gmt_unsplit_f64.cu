// FP64 unsplit step kernels: up to 256 threads, 1 resident block per SM.  Built with --fmad=false
// so each expression rounds exactly as the IEEE evaluation of the oracle.
#include "gmt_unsplit_inst.cuh"

namespace gmt {
cudaError_t launch_unsplit(const UnsplitArgs<double>& A, int recon, int riem, cudaStream_t s) {
    if (A.ox * A.oy > 256) return cudaErrorInvalidConfiguration;
    return unsplit_dispatch_t<double, 256, 1>(A, recon, riem, s);
}
int unsplit_regs_f64(int recon, int riem, int) { return unsplit_regs_of_t<double, 256, 1>(recon, riem); }
}  // namespace gmt
