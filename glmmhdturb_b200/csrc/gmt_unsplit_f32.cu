// FP32 unsplit and tiled-march step kernels, built with --use_fast_math (approximate reciprocal and square root,
// as the reference's own kernels are built, march_bridge/build_mhd.sh:25).  Two block shapes:
// up to 256 threads with 2 resident blocks per SM (<= 128 registers), and up to 512 threads with
// one block per SM for the larger tiles.
#include "gmt_unsplit_inst.cuh"

namespace gmt {
// compile-time tiles for the production schemes (PLM-MC / PPM with HLLD / HLL)
template <int TOX, int TOY>
static bool fixed_tile(const UnsplitArgs<float>& A, int recon, int riem, cudaStream_t s, cudaError_t& e) {
    if (A.ox != TOX || A.oy != TOY) return false;
#define GMT_FIX(RC, RM) \
    if (recon == RC && riem == RM) { e = unsplit_go<float, RC, RM, 512, 1, TOX, TOY>(A, s); return true; }
    GMT_FIX(RECON_MC, RIEM_HLLD) GMT_FIX(RECON_MC, RIEM_HLL) GMT_FIX(RECON_PPM, RIEM_HLLD) GMT_FIX(RECON_PPM, RIEM_HLL)
#undef GMT_FIX
    return false;
}

cudaError_t launch_unsplit(const UnsplitArgs<float>& A, int recon, int riem, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    if (fixed_tile<32, 16>(A, recon, riem, s, e) || fixed_tile<64, 8>(A, recon, riem, s, e)) return e;
    if (A.ox * A.oy > 256) return unsplit_dispatch_t<float, 512, 1>(A, recon, riem, s);
    return unsplit_dispatch_t<float, 256, 2>(A, recon, riem, s);
}
cudaError_t unsplit_prepare_f32() {
    cudaError_t e = unsplit_configure_all_t<float, 256, 2>();
    if (e == cudaSuccess) e = unsplit_configure_all_t<float, 512, 1>();
    const int combos[4][2] = {{RECON_MC, RIEM_HLLD}, {RECON_MC, RIEM_HLL}, {RECON_PPM, RIEM_HLLD}, {RECON_PPM, RIEM_HLL}};
    (void)combos;
    if (e == cudaSuccess) e = unsplit_configure<float, RECON_MC, RIEM_HLLD, 512, 1, 32, 16>();
    if (e == cudaSuccess) e = unsplit_configure<float, RECON_MC, RIEM_HLL, 512, 1, 32, 16>();
    if (e == cudaSuccess) e = unsplit_configure<float, RECON_PPM, RIEM_HLLD, 512, 1, 32, 16>();
    if (e == cudaSuccess) e = unsplit_configure<float, RECON_PPM, RIEM_HLL, 512, 1, 32, 16>();
    if (e == cudaSuccess) e = unsplit_configure<float, RECON_MC, RIEM_HLLD, 512, 1, 64, 8>();
    if (e == cudaSuccess) e = unsplit_configure<float, RECON_MC, RIEM_HLL, 512, 1, 64, 8>();
    if (e == cudaSuccess) e = unsplit_configure<float, RECON_PPM, RIEM_HLLD, 512, 1, 64, 8>();
    if (e == cudaSuccess) e = unsplit_configure<float, RECON_PPM, RIEM_HLL, 512, 1, 64, 8>();
    for (int rc = 0; e == cudaSuccess && rc < 3; ++rc)
        e = launch_ensemble((const UnsplitArgs<float>*)nullptr, nullptr, 0, nullptr, rc == 2 ? RECON_PPM : RECON_MC,
                            rc == 0 ? RIEM_HLLD : RIEM_HLL, 1, 0);
    UnsplitArgs<float> none{};
    for (int rc = 0; e == cudaSuccess && rc < 2; ++rc) {
        e = march_dispatch_t<float, 512, 1>(none, rc ? RECON_PPM : RECON_MC, 0, true);
        if (e == cudaSuccess) e = march_dispatch_t<float, 256, 2>(none, rc ? RECON_PPM : RECON_MC, 0, true);
    }
    if (e == cudaSuccess) e = march_go<float, RECON_MC, 512, 1, 32, 16>(none, 0, true);
    if (e == cudaSuccess) e = march_go<float, RECON_PPM, 512, 1, 32, 16>(none, 0, true);
    return e;
}
cudaError_t launch_march_tiled(const UnsplitArgs<float>& A, int recon, cudaStream_t s) {
    if (A.ox == 32 && A.oy == 16)   // compile-time tile of the production shape
        return recon == RECON_PPM ? march_go<float, RECON_PPM, 512, 1, 32, 16>(A, s, false)
                                  : march_go<float, RECON_MC, 512, 1, 32, 16>(A, s, false);
    if (A.ox * A.oy > 256) return march_dispatch_t<float, 512, 1>(A, recon, s, false);
    return march_dispatch_t<float, 256, 2>(A, recon, s, false);
}
int march_tiled_regs(const UnsplitArgs<float>*, int recon, int nthreads) {
    return nthreads > 256 ? march_regs_of_t<float, 512, 1>(recon) : march_regs_of_t<float, 256, 2>(recon);
}
int unsplit_regs_f32(int recon, int riem, int nthreads) {
    return nthreads > 256 ? unsplit_regs_of_t<float, 512, 1>(recon, riem) : unsplit_regs_of_t<float, 256, 2>(recon, riem);
}
cudaError_t launch_ensemble(const UnsplitArgs<float>* boxes, const EnsItem* items, int nitems, unsigned* queue,
                            int recon, int riem, int nsm, cudaStream_t s) {
    if (recon == RECON_MC && riem == RIEM_HLLD) return ensemble_go<float, RECON_MC, RIEM_HLLD>(boxes, items, nitems, queue, nsm, s);
    if (recon == RECON_MC && riem == RIEM_HLL) return ensemble_go<float, RECON_MC, RIEM_HLL>(boxes, items, nitems, queue, nsm, s);
    if (recon == RECON_PPM && riem == RIEM_HLL) return ensemble_go<float, RECON_PPM, RIEM_HLL>(boxes, items, nitems, queue, nsm, s);
    return cudaErrorNotSupported;
}
}  // namespace gmt
