// gmt_unsplit_inst.cuh -- instantiation and launch of the unsplit kernel for one real type.
// Included once by gmt_unsplit_f32.cu and once by gmt_unsplit_f64.cu (the FP64 unit is compiled
// without FMA contraction so that it evaluates the same IEEE expressions as the oracle).
#pragma once
#include "gmt_internal.h"
#include "gmt_unsplit.cuh"

namespace gmt {

// Per device, once: allow the kernel up to 227 KB of dynamic shared memory.  Called for every
// instantiation when a context is created, so that no attribute call happens during a stream
// capture of the steps.
template <class K> static cudaError_t configure_once(K k, int* configured) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64 || configured[dev]) return cudaSuccess;
    // the per-block limit covers static plus dynamic shared memory
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, k);
    int optin = 227 * 1024;
    if (e == cudaSuccess) cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e;
    }
    configured[dev] = 1;
    return cudaSuccess;
}

template <class R, int RECON, int RIEM, int MAXT, int MINB, int TOX = 0, int TOY = 0> struct UnsplitCfg {
    static int configured[64];
};
template <class R, int RECON, int RIEM, int MAXT, int MINB, int TOX, int TOY>
int UnsplitCfg<R, RECON, RIEM, MAXT, MINB, TOX, TOY>::configured[64] = {0};

template <class R, int RECON, int RIEM, int MAXT, int MINB, int TOX = 0, int TOY = 0>
static cudaError_t unsplit_configure() {
    return configure_once(unsplit_kernel<R, RECON, RIEM, MAXT, MINB, TOX, TOY>,
                          UnsplitCfg<R, RECON, RIEM, MAXT, MINB, TOX, TOY>::configured);
}

template <class R, int RECON, int RIEM, int MAXT, int MINB, int TOX = 0, int TOY = 0>
static cudaError_t unsplit_go(const UnsplitArgs<R>& A, cudaStream_t s) {
    auto k = unsplit_kernel<R, RECON, RIEM, MAXT, MINB, TOX, TOY>;
    {
        cudaError_t e = unsplit_configure<R, RECON, RIEM, MAXT, MINB, TOX, TOY>();
        if (e != cudaSuccess) return e;
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

template <class R, int MAXT, int MINB> static cudaError_t unsplit_configure_all_t() {
    cudaError_t e = cudaSuccess;
#define GMT_CASE(RC, RM) \
    if (e == cudaSuccess) e = unsplit_configure<R, RC, RM, MAXT, MINB>();
    GMT_CASE(RECON_MC, RIEM_HLLD) GMT_CASE(RECON_MC, RIEM_HLL) GMT_CASE(RECON_MC, RIEM_LLF_BOUND)
    GMT_CASE(RECON_MINMOD, RIEM_HLLD) GMT_CASE(RECON_MINMOD, RIEM_HLL) GMT_CASE(RECON_MINMOD, RIEM_LLF_BOUND)
    GMT_CASE(RECON_PPM, RIEM_HLLD) GMT_CASE(RECON_PPM, RIEM_HLL) GMT_CASE(RECON_PPM, RIEM_LLF_BOUND)
#undef GMT_CASE
    return e;
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

namespace gmt {
// ensemble launcher: persistent grid, one (FP32) or two (FP64) blocks per SM
template <class R, int RECON, int RIEM>
static cudaError_t ensemble_go(const UnsplitArgs<R>* boxes, const EnsItem* items, int nitems, unsigned* queue,
                               int nsm, cudaStream_t s) {
    // FP32: 32x16 tiles, 512 threads, one block per SM; FP64: 16x16 tiles, 256 threads
    constexpr bool F32 = sizeof(R) == 4;
    constexpr int OX = ens_tile_x<R>(), OY = 16, NT = OX * OY, MB = F32 ? 1 : 2;
    auto k = ensemble_kernel<R, RECON, RIEM, OX, OY, NT, MB>;
    static int configured[64] = {0};
    {
        cudaError_t e = configure_once(k, configured);
        if (e != cudaSuccess) return e;
    }
    if (nitems <= 0) return cudaSuccess;   // configure only
    int nb = std::max(1, std::min(nitems, MB * nsm));
    k<<<nb, NT, unsplit_smem_bytes<R>(OX, OY), s>>>(boxes, items, nitems, queue);
    return cudaGetLastError();
}
}  // namespace gmt

namespace gmt {
// tiled march launcher (recon MC or PPM; the march has no minmod variant, spike_mhd.cu:118-123);
// nt <= 0 configures the kernel only
template <class R, int RECON, int MAXT, int MINB, int TOX = 0, int TOY = 0>
static cudaError_t march_go(const UnsplitArgs<R>& A, cudaStream_t s, bool configure_only) {
    auto k = march_tile_kernel<R, RECON, MAXT, MINB, TOX, TOY>;
    static int configured[64] = {0};
    {
        cudaError_t e = configure_once(k, configured);
        if (e != cudaSuccess) return e;
    }
    if (configure_only) return cudaSuccess;
    const int nt = A.ox * A.oy;
    if (nt > MAXT || nt < 1) return cudaErrorInvalidConfiguration;
    dim3 grid(A.nx / A.ox, A.ny / A.oy, (A.nz + A.lz - 1) / A.lz);
    k<<<grid, nt, unsplit_smem_bytes<R>(A.ox, A.oy), s>>>(A);
    return cudaGetLastError();
}
template <class R, int MAXT, int MINB>
static cudaError_t march_dispatch_t(const UnsplitArgs<R>& A, int recon, cudaStream_t s, bool configure_only) {
    if (recon == RECON_PPM) return march_go<R, RECON_PPM, MAXT, MINB>(A, s, configure_only);
    return march_go<R, RECON_MC, MAXT, MINB>(A, s, configure_only);
}
template <class R, int MAXT, int MINB> static int march_regs_of_t(int recon) {
    cudaFuncAttributes fa{};
    cudaError_t e = recon == RECON_PPM ? cudaFuncGetAttributes(&fa, march_tile_kernel<R, RECON_PPM, MAXT, MINB>)
                                       : cudaFuncGetAttributes(&fa, march_tile_kernel<R, RECON_MC, MAXT, MINB>);
    return e == cudaSuccess ? fa.numRegs : -1;
}
}  // namespace gmt
