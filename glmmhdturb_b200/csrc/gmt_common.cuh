// gmt_common.cuh -- kernel argument blocks and small device helpers shared by the kernels.
#pragma once
#include <type_traits>
#include <cuda.h>   // CUtensorMap (the type only; the library does not link libcuda)
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
    const R* trig8;        // FP32 or null: [nx][4 m][2 cos|sin] holding 2 cos and -2 sin (force_accel_f32)
    unsigned long long* cfl_out;  // [2] bits of non-negative doubles (max ctot, max signal) or null
    int* err;              // set to 1 when a bounded wait gives up (never expected)
    R dx;                  // cell size (dt/dx of device-supplied steps)
    const double* dparams; // if set: dt, ch, glm_fac, ramp of this step read from device memory
    R* fmass;              // if set: the mass fluxes of every cell's lower x, y, z faces (3 planes),
                           // for the passive-species pass of the march scheme
    int use_tma;           // tmap describes u: tiles clear of the box edges stage by TMA
    CUtensorMap tmap;      // 4-D map (x, y, z, variable) of u; box (ox+8) x (oy+4) x 1 x 9
    long long wait_cycles; // budget of each bounded wait (GMT_WAIT_CYCLES)
    int wait_test;         // failure-path tests only: the next plane is not staged and no thread
                           // arrives on the staging mbarrier, so every wait runs out (0 in production)
    // adjoint record mode (a scheme with kRecord): the step writes every cell's six interface
    // states and, in place of the new state, the adjoint of its update epilogue
    R* rec_fs;             // 54 planes: interface states +x, -x, +y, -y, +z, -z of every cell
    const R* rec_ubn;      // 9 planes: adjoint of the step's output
    R* rec_r1b;            // 9 planes: adjoint of the pre-epilogue state
    R* rec_ub;             // 9 planes: adjoint of the step's input, identity part
    double* rec_damp;      // dL/d(forcing amplitude) accumulator
    R rec_amp;             // forcing amplitude
};

// step values of one box, from the kernel arguments or from device memory
template <class R> struct StepVals {
    R dt, dtdx, ch, glm_fac, ramp;
};
template <class R> __device__ __forceinline__ StepVals<R> step_vals(const UnsplitArgs<R>& A) {
    StepVals<R> V;
    if (A.dparams) {
        V.dt = (R)A.dparams[0];
        V.dtdx = V.dt / A.dx;
        V.ch = (R)A.dparams[1];
        V.glm_fac = (R)A.dparams[2];
        V.ramp = (R)A.dparams[3];
    } else {
        V.dt = A.dt; V.dtdx = A.dtdx; V.ch = A.ch; V.glm_fac = A.glm_fac; V.ramp = A.ramp;
    }
    return V;
}

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
// wait until at most N of this thread's most recent cp.async groups are still in flight
template <int N> __device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// mbarrier completion of cp.async groups: every thread arrives once per phase after issuing its
// copies; the phase completes when all of them have landed in shared memory.
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    unsigned s = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(s), "r"(count));
}
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    unsigned s = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(s) : "memory");
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
// TMA (cp.async.bulk.tensor) staging: one elected thread arms the mbarrier with the byte count of
// the box and issues the copy; the mbarrier phase completes when the bytes have landed.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    unsigned s = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(s), "r"(bytes) : "memory");
}
// make an initialised mbarrier visible to the async (TMA) proxy
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// order this CTA's earlier generic-proxy accesses of shared memory before later async-proxy ones
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// 4-D tiled load of the box at (c0, c1, c2, c3) into shared memory; the map must live in
// kernel-parameter (grid-constant), constant or global memory
__device__ __forceinline__ void tma_load_4d(void* smem_dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(d),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(b)
        : "memory");
}

// Bounded wait for an mbarrier phase: polls until the phase completes or `budget` SM clock
// cycles (clock64) have passed since the first poll; then it records the failure in *err and
// returns false, and the caller carries on (its output is reported invalid by the host).
// GMT_WAIT_CYCLES, about 0.5 s at the B200's 1.965 GHz, is the default budget of the tile kernels;
// a staged plane lands in microseconds.
#define GMT_WAIT_CYCLES (1LL << 30)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err, long long budget) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > budget) {
            if (err) atomicExch(err, 1);
            return false;
        }
    }
    return true;
}

template <class R> __device__ __forceinline__ void cp_async_r(R* smem, const R* gmem);
template <> __device__ __forceinline__ void cp_async_r(float* s, const float* g) { cp_async4(s, g); }
template <> __device__ __forceinline__ void cp_async_r(double* s, const double* g) { cp_async8(s, g); }

// coordinates of linear cell index c = x + nx (y + ny z); 32-bit divisions while n < 2^32
GMT_HD void cell_coords(size_t c, int nx, int ny, size_t n, int& x, int& y, int& z) {
    if (n <= 0xffffffffu) {
        const unsigned cc = (unsigned)c, q = cc / (unsigned)nx;
        x = (int)(cc - q * (unsigned)nx);
        y = (int)(q % (unsigned)ny);
        z = (int)(q / (unsigned)ny);
    } else {
        x = (int)(c % nx);
        y = (int)((c / nx) % ny);
        z = (int)(c / ((size_t)nx * ny));
    }
}
// periodic image of i for -n <= i < 2n
GMT_HD int wrap1(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

GMT_HD int wrapi(int i, int n) {
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
    R sx, sy, sz;
    if constexpr (std::is_same<R, float>::value) {
        // FP32: the three fast speeds share 1/rho, c^2 and d^2 (fast_speed's expressions with the
        // division by rho taken once, as the fast-math build evaluates it anyway)
        const R ir = R(1) / q.v[0];
        const R c2 = K.gamma * q.v[4] * ir;
        const R b2 = (q.v[5] * q.v[5] + q.v[6] * q.v[6] + q.v[7] * q.v[7]) * ir;
        const R d2 = R(0.5) * (b2 + c2), t = c2 * ir;
        sx = rabs(q.v[1]) + sqrt_r(d2 + sqrt_r(rmax(d2 * d2 - t * q.v[5] * q.v[5], R(0))));
        sy = rabs(q.v[2]) + sqrt_r(d2 + sqrt_r(rmax(d2 * d2 - t * q.v[6] * q.v[6], R(0))));
        sz = rabs(q.v[3]) + sqrt_r(d2 + sqrt_r(rmax(d2 * d2 - t * q.v[7] * q.v[7], R(0))));
    } else {
        sx = rabs(q.v[1]) + fast_speed(q, K.gamma, q.v[5]);
        sy = rabs(q.v[2]) + fast_speed(q, K.gamma, q.v[6]);
        sz = rabs(q.v[3]) + fast_speed(q, K.gamma, q.v[7]);
    }
    ctot = sx + sy + sz;
    smax = rmax(rmax(sx, sy), sz);
}

// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11)
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}

// One OU step of mode q with wavevector (kx,ky,kz): ahat <- alpha*ahat + beta*sigma_k*P_k(xi),
// xi = 6 normals from Philox(counter = {counter, q, 0|1, 0}, key = {seed, 0x9E3779B9}) + Box-Muller,
// P_k the solenoidal projector, sigma_k = sigma0/|k| (modes: [61][3][2] doubles)
__device__ __forceinline__ void ou_mode_update(double* modes, int q, int ikx, int iky, int ikz, uint32_t seed,
                                               uint32_t counter, double alpha, double beta, double sigma0) {
    uint32_t r[8] = {counter, (uint32_t)q, 0u, 0u, counter, (uint32_t)q, 1u, 0u};
    philox4x32_10(r, seed, 0x9E3779B9u);
    philox4x32_10(r + 4, seed, 0x9E3779B9u);
    const double twopi = 6.283185307179586476925286766559;
    double z[6];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        double u1 = ((double)r[2 * b] + 0.5) * 2.3283064365386962890625e-10;
        double u2 = ((double)r[2 * b + 1] + 0.5) * 2.3283064365386962890625e-10;
        double rr = sqrt(-2.0 * log(u1));
        double th = twopi * u2;
        z[2 * b] = rr * cos(th);
        z[2 * b + 1] = rr * sin(th);
    }
    double kx = ikx, ky = iky, kz = ikz;
    double kk = sqrt(kx * kx + ky * ky + kz * kz);
    double ux = kx / kk, uy = ky / kk, uz = kz / kk;
    double sig = sigma0 / kk;
    double kr = ux * z[0] + uy * z[2] + uz * z[4];
    double ki = ux * z[1] + uy * z[3] + uz * z[5];
    double uu[3] = {ux, uy, uz};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double pr = z[2 * c] - uu[c] * kr;
        double pi = z[2 * c + 1] - uu[c] * ki;
        double* m = modes + (q * 3 + c) * 2;
        m[0] = alpha * m[0] + beta * sig * pr;
        m[1] = alpha * m[1] + beta * sig * pi;
    }
}

// per-row mode table B[kx][c] of row (j, k) (same summation order as the oracle's Forcer::accel)
template <class R>
__device__ __forceinline__ void btab_row(const double* modes, const int* mode_k, const R* trigy, const R* trigz, int ny,
                                         int nz, int j, int k, R* out) {
    int q = 0;
    for (int kx = 0; kx <= 3; ++kx) {
        R Br[3] = {R(0), R(0), R(0)}, Bi[3] = {R(0), R(0), R(0)};
        while (q < 61 && mode_k[3 * q] == kx) {
            int ky = mode_k[3 * q + 1], kz = mode_k[3 * q + 2];
            int ay = ky < 0 ? -ky : ky, az = kz < 0 ? -kz : kz;
            R eyr = trigy[(2 * ay) * ny + j], eyi = trigy[(2 * ay + 1) * ny + j];
            R ezr = trigz[(2 * az) * nz + k], ezi = trigz[(2 * az + 1) * nz + k];
            if (ky < 0) eyi = -eyi;
            if (kz < 0) ezi = -ezi;
            R er = eyr * ezr - eyi * ezi;
            R ei = eyr * ezi + eyi * ezr;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                R ar = (R)modes[(q * 3 + c) * 2], ai = (R)modes[(q * 3 + c) * 2 + 1];
                Br[c] = Br[c] + (ar * er - ai * ei);
                Bi[c] = Bi[c] + (ar * ei + ai * er);
            }
            ++q;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) { out[kx * 6 + 2 * c] = Br[c]; out[kx * 6 + 2 * c + 1] = Bi[c]; }
    }
}

// FP32 forcing acceleration with vectorised table loads: the row table's 24 values as six float4,
// the x table (2 cos, -2 sin per m) as two float4, and 24 FMAs; the same sum as force_accel in
// another order (FP32 round-off)
__device__ __forceinline__ void force_accel_f32(const float* __restrict__ btab_row, const float* __restrict__ trig8,
                                                int i, float ramp, float& ax, float& ay, float& az) {
    const float4* t = reinterpret_cast<const float4*>(trig8 + 8 * i);
    const float4 t0 = t[0], t1 = t[1];   // (2c0, -2s0, 2c1, -2s1), (2c2, -2s2, 2c3, -2s3)
    const float4* b = reinterpret_cast<const float4*>(btab_row);
    const float4 b0 = b[0], b1 = b[1], b2 = b[2], b3 = b[3], b4 = b[4], b5 = b[5];
    // row layout [kx][component][re, im]
    float S0 = fmaf(b0.x, t0.x, b0.y * t0.y), S1 = fmaf(b0.z, t0.x, b0.w * t0.y), S2 = fmaf(b1.x, t0.x, b1.y * t0.y);
    S0 = fmaf(b1.z, t0.z, fmaf(b1.w, t0.w, S0));
    S1 = fmaf(b2.x, t0.z, fmaf(b2.y, t0.w, S1));
    S2 = fmaf(b2.z, t0.z, fmaf(b2.w, t0.w, S2));
    S0 = fmaf(b3.x, t1.x, fmaf(b3.y, t1.y, S0));
    S1 = fmaf(b3.z, t1.x, fmaf(b3.w, t1.y, S1));
    S2 = fmaf(b4.x, t1.x, fmaf(b4.y, t1.y, S2));
    S0 = fmaf(b4.z, t1.z, fmaf(b4.w, t1.w, S0));
    S1 = fmaf(b5.x, t1.z, fmaf(b5.y, t1.w, S1));
    S2 = fmaf(b5.z, t1.z, fmaf(b5.w, t1.w, S2));
    ax = ramp * S0; ay = ramp * S1; az = ramp * S2;
}

// forcing acceleration at one cell from the per-row table (same order as the oracle)
template <class R>
GMT_HD void force_accel(const R* btab_row, const R* trigx, int nx, int i, R ramp, R& ax, R& ay,
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
