// gmt_common.cuh -- kernel argument blocks and small device helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "gmt_phys.cuh"

namespace gmt {

constexpr int NV = 9;

// Nine plane pointers (the bridge passes one device pointer per SoA plane,
// march_bridge/MarchBridge.jl:64; a single base pointer with plane stride n maps onto it).
template <class R> struct Planes { R* p[9]; };
template <class R> struct CPlanes { const R* p[9]; };
// CT state: [rho, mx, my, mz, E, bxf, byf, bzf]
template <class R> struct Planes8 { R* p[8]; };
template <class R> struct CPlanes8 { const R* p[8]; };

// Arguments of one unsplit GLM step (glmmhd_turb.jl:746-767 / 878-908 with ch, glm_fac and
// the forcing ramp supplied by the caller, as march_set_glm does for the bridge).
template <class R> struct UnsplitArgs {
    CPlanes<R> u;          // old state
    Planes<R> o;           // new state
    int nx, ny, nz;
    int ox, oy, lz;        // tile: ox*oy owned columns per block, lz planes per z chunk
    R dt, dtdx, ch, glm_fac, ramp;
    Consts<R> K;
    int iflo, use_llf, do_turb;
    const R* btab;         // forcing row table [nz][ny][4 kx][3 comp][2] (re, im) or null
    const R* trigx;        // [4 m][2 cos|sin][nx]
    unsigned long long* cfl_out;  // [2] bits of non-negative doubles (max ctot, max signal) or null
    int* err;              // set to 1 when a bounded wait gives up (never expected)
};

// cp.async 4-byte global -> shared copy (L1-allocating), plus group commit / wait.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// mbarrier completion of cp.async groups: every thread arrives once per phase after issuing its
// copies; the phase completes when all of them have landed in shared memory.
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    unsigned s = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(s), "r"(count));
}
__device__ __forceinline__ void mbar_arrive_cp_async(uint64_t* bar) {
    unsigned s = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(s) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned s = (unsigned)__cvta_generic_to_shared(bar);
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(s), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: gives up after ~2^20 polls, records the failure and returns false
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err) {
    for (int it = 0; it < (1 << 20); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicExch(err, 1);
    return false;
}

template <class R> __device__ __forceinline__ void cp_async_r(R* smem, const R* gmem);
template <> __device__ __forceinline__ void cp_async_r(float* s, const float* g) { cp_async4(s, g); }
template <> __device__ __forceinline__ void cp_async_r(double* s, const double* g) { cp_async8(s, g); }

__device__ __forceinline__ int wrapi(int i, int n) {
    i = i % n;
    return i < 0 ? i + n : i;
}

// max of a non-negative double across the block, then one atomicMax on its bit pattern
// (non-negative IEEE doubles order like their unsigned bit patterns)
__device__ __forceinline__ void block_max_atomic(double v, unsigned long long* dst, double* red) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        double x = lane < nw ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0 && x > 0.0) atomicMax(dst, (unsigned long long)__double_as_longlong(x));
    }
}

// CFL signal speeds of a conserved state (glmmhd_turb.jl:1963-1971)
template <class R>
__device__ __forceinline__ void cfl_speeds(const Q9<R>& c, const Consts<R>& K, R& ctot, R& smax) {
    Q9<R> q = cons2prim(c, K.gamma, K.smallr, K.pfl);
    R sx = rabs(q.v[1]) + fast_speed(q, K.gamma, q.v[5]);
    R sy = rabs(q.v[2]) + fast_speed(q, K.gamma, q.v[6]);
    R sz = rabs(q.v[3]) + fast_speed(q, K.gamma, q.v[7]);
    ctot = sx + sy + sz;
    smax = rmax(rmax(sx, sy), sz);
}

// forcing acceleration at one cell from the per-row table (same order as the oracle)
template <class R>
__device__ __forceinline__ void force_accel(const R* btab_row, const R* trigx, int nx, int i, R ramp, R& ax, R& ay,
                                            R& az) {
    R S0 = R(0), S1 = R(0), S2 = R(0);
#pragma unroll
    for (int kx = 0; kx < 4; ++kx) {
        R cx = trigx[(2 * kx) * nx + i], sx = trigx[(2 * kx + 1) * nx + i];
        const R* b = btab_row + kx * 6;
        S0 = S0 + R(2) * (b[0] * cx - b[1] * sx);
        S1 = S1 + R(2) * (b[2] * cx - b[3] * sx);
        S2 = S2 + R(2) * (b[4] * cx - b[5] * sx);
    }
    ax = ramp * S0; ay = ramp * S1; az = ramp * S2;
}

}  // namespace gmt
