// gmt_unsplit_inst.cuh -- instantiation and launch of the unsplit kernel for one real type.
// Included once by gmt_unsplit_f32.cu and once by gmt_unsplit_f64.cu (the FP64 unit is compiled
// without FMA contraction so that it evaluates the same IEEE expressions as the oracle).
#pragma once
#include "gmt_internal.h"
#include "gmt_unsplit.cuh"

namespace gmt {

template <class R, int RECON, int RIEM, int MAXT, int MINB>
static cudaError_t unsplit_go(const UnsplitArgs<R>& A, cudaStream_t s) {
    auto k = unsplit_kernel<R, RECON, RIEM, MAXT, MINB>;
    static int configured[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (e != cudaSuccess) return e;
        configured[dev] = 1;
    }
    const int nt = A.ox * A.oy;
    if (nt > MAXT || nt < 1) return cudaErrorInvalidConfiguration;
    dim3 grid(A.nx / A.ox, A.ny / A.oy, (A.nz + A.lz - 1) / A.lz);
    k<<<grid, nt, unsplit_smem_bytes<R>(A.ox, A.oy), s>>>(A);
    return cudaGetLastError();
}

template <class R, int MAXT, int MINB>
static cudaError_t unsplit_dispatch_t(const UnsplitArgs<R>& A, int recon, int riem, cudaStream_t s) {
#define GMT_CASE(RC, RM) \
    if (recon == RC && riem == RM) return unsplit_go<R, RC, RM, MAXT, MINB>(A, s);
    GMT_CASE(RECON_MC, RIEM_HLLD) GMT_CASE(RECON_MC, RIEM_HLL) GMT_CASE(RECON_MC, RIEM_LLF_BOUND)
    GMT_CASE(RECON_MINMOD, RIEM_HLLD) GMT_CASE(RECON_MINMOD, RIEM_HLL) GMT_CASE(RECON_MINMOD, RIEM_LLF_BOUND)
    GMT_CASE(RECON_PPM, RIEM_HLLD) GMT_CASE(RECON_PPM, RIEM_HLL) GMT_CASE(RECON_PPM, RIEM_LLF_BOUND)
#undef GMT_CASE
    return cudaErrorInvalidValue;
}

template <class R, int MAXT, int MINB> static int unsplit_regs_of_t(int recon, int riem) {
    cudaFuncAttributes fa{};
    cudaError_t e = cudaErrorInvalidValue;
#define GMT_CASE(RC, RM) \
    if (recon == RC && riem == RM) e = cudaFuncGetAttributes(&fa, unsplit_kernel<R, RC, RM, MAXT, MINB>);
    GMT_CASE(RECON_MC, RIEM_HLLD) GMT_CASE(RECON_MC, RIEM_HLL) GMT_CASE(RECON_MC, RIEM_LLF_BOUND)
    GMT_CASE(RECON_MINMOD, RIEM_HLLD) GMT_CASE(RECON_MINMOD, RIEM_HLL) GMT_CASE(RECON_MINMOD, RIEM_LLF_BOUND)
    GMT_CASE(RECON_PPM, RIEM_HLLD) GMT_CASE(RECON_PPM, RIEM_HLL) GMT_CASE(RECON_PPM, RIEM_LLF_BOUND)
#undef GMT_CASE
    return e == cudaSuccess ? fa.numRegs : -1;
}

}  // namespace gmt
