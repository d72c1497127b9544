// FP64 unsplit step kernels: up to 256 threads, 1 resident block per SM.  Built with --fmad=false
// so each expression rounds exactly as the IEEE evaluation of the oracle.
#include "gmt_unsplit_inst.cuh"

namespace gmt {
// compile-time tiles for the production schemes (constant strides and loop bounds)
template <int TOX, int TOY>
static bool fixed_tile64(const UnsplitArgs<double>& A, int recon, int riem, cudaStream_t s, cudaError_t& e) {
    if (A.ox != TOX || A.oy != TOY) return false;
#define GMT_FIX(RC, RM) \
    if (recon == RC && riem == RM) { e = unsplit_go<double, RC, RM, 256, 1, TOX, TOY>(A, s); return true; }
    GMT_FIX(RECON_MC, RIEM_HLLD) GMT_FIX(RECON_MC, RIEM_HLL) GMT_FIX(RECON_PPM, RIEM_HLL)
#undef GMT_FIX
    return false;
}
cudaError_t launch_unsplit(const UnsplitArgs<double>& A, int recon, int riem, cudaStream_t s) {
    if (A.ox * A.oy > 256) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaSuccess;
    if (fixed_tile64<32, 8>(A, recon, riem, s, e) || fixed_tile64<16, 16>(A, recon, riem, s, e)) return e;
    return unsplit_dispatch_t<double, 256, 1>(A, recon, riem, s);
}
cudaError_t unsplit_prepare_f64() {
    cudaError_t e = unsplit_configure_all_t<double, 256, 1>();
#define GMT_FIX(RC, RM)                                                                          \
    if (e == cudaSuccess) e = unsplit_configure<double, RC, RM, 256, 1, 32, 8>();                \
    if (e == cudaSuccess) e = unsplit_configure<double, RC, RM, 256, 1, 16, 16>();
    GMT_FIX(RECON_MC, RIEM_HLLD) GMT_FIX(RECON_MC, RIEM_HLL) GMT_FIX(RECON_PPM, RIEM_HLL)
#undef GMT_FIX
    for (int rc = 0; e == cudaSuccess && rc < 3; ++rc)
        e = launch_ensemble((const UnsplitArgs<double>*)nullptr, nullptr, 0, nullptr, rc == 2 ? RECON_PPM : RECON_MC,
                            rc == 0 ? RIEM_HLLD : RIEM_HLL, 1, 0);
    UnsplitArgs<double> none{};
    for (int rc = 0; e == cudaSuccess && rc < 2; ++rc) e = march_dispatch_t<double, 256, 1>(none, rc ? RECON_PPM : RECON_MC, 0, true);
    return e;
}
int unsplit_regs_f64(int recon, int riem, int) { return unsplit_regs_of_t<double, 256, 1>(recon, riem); }
cudaError_t launch_march_tiled(const UnsplitArgs<double>& A, int recon, cudaStream_t s) {
    if (A.ox * A.oy > 256) return cudaErrorInvalidConfiguration;
    return march_dispatch_t<double, 256, 1>(A, recon, s, false);
}
int march_tiled_regs(const UnsplitArgs<double>*, int recon, int) { return march_regs_of_t<double, 256, 1>(recon); }
cudaError_t launch_ensemble(const UnsplitArgs<double>* boxes, const EnsItem* items, int nitems, unsigned* queue,
                            int recon, int riem, int nsm, cudaStream_t s) {
    if (recon == RECON_MC && riem == RIEM_HLLD) return ensemble_go<double, RECON_MC, RIEM_HLLD>(boxes, items, nitems, queue, nsm, s);
    if (recon == RECON_MC && riem == RIEM_HLL) return ensemble_go<double, RECON_MC, RIEM_HLL>(boxes, items, nitems, queue, nsm, s);
    if (recon == RECON_PPM && riem == RIEM_HLL) return ensemble_go<double, RECON_PPM, RIEM_HLL>(boxes, items, nitems, queue, nsm, s);
    return cudaErrorNotSupported;
}
}  // namespace gmt
