// FP32 constrained-transport step kernels (gmt_ct_tile.cuh), built with --use_fast_math like the
// reference's own kernels (march_bridge/build_mhd.sh:25).  Tiles up to 512 threads, one block
// per SM.
#include "gmt_ct_tile.cuh"

namespace gmt {
// compile-time tile of the production shape
template <int RC, int RM> static cudaError_t ct_fixed(const CTArgs<float>& A, cudaStream_t s, bool conf) {
    return ct_go<float, RC, RM, 512, 1, 32, 16>(A, s, conf);
}
static cudaError_t ct_fixed_dispatch(const CTArgs<float>& A, int recon, int riem, cudaStream_t s, bool conf) {
    const bool ppm = recon == RECON_PPM, hlld = riem == RIEM_HLLD;
    if (ppm && hlld) return ct_fixed<RECON_PPM, RIEM_HLLD>(A, s, conf);
    if (ppm) return ct_fixed<RECON_PPM, RIEM_HLL>(A, s, conf);
    if (hlld) return ct_fixed<RECON_MC, RIEM_HLLD>(A, s, conf);
    return ct_fixed<RECON_MC, RIEM_HLL>(A, s, conf);
}

cudaError_t launch_ct(const CTArgs<float>& A, cudaStream_t s) {
    if (A.ox == 32 && A.oy == 16) return ct_fixed_dispatch(A, A.recon, A.riem, s, false);
    if (A.ox * A.oy > 256) return ct_dispatch_t<float, 512, 1>(A, A.recon, A.riem, s, false);
    return ct_dispatch_t<float, 256, 2>(A, A.recon, A.riem, s, false);
}
cudaError_t ct_prepare_f32() {
    cudaError_t e = ct_configure_all_t<float, 512, 1>();
    if (e == cudaSuccess) e = ct_configure_all_t<float, 256, 2>();
    CTArgs<float> none{};
    for (int rc = 0; e == cudaSuccess && rc < 2; ++rc)
        for (int rm = 0; e == cudaSuccess && rm < 2; ++rm)
            e = ct_fixed_dispatch(none, rc ? RECON_PPM : RECON_MC, rm ? RIEM_HLL : RIEM_HLLD, 0, true);
    return e;
}
int ct_regs_f32(int recon, int riem, int nthreads) {
    return nthreads > 256 ? ct_regs_of_t<float, 512, 1>(recon, riem) : ct_regs_of_t<float, 256, 2>(recon, riem);
}
}  // namespace gmt
