// gmt_aux.cu -- CFL reduction, diagnostics, OU mode forcing, initial conditions.
//
// CFL: ctot = sum_d(|v_d| + c_f(B_d)) per cell, dt = courant*dx/max(ctot) (glmmhd_turb.jl:1963-1978),
// reduced in FP64 with a warp-shuffle max and one atomic per block.
// Diagnostics (glmmhd_turb.jl:1996-2018): FP64 sums over a fixed grid and a fixed tree, so the
// result does not depend on scheduling.
// Forcing: the 61 +/- mode pairs with 1 <= |k|^2 <= 9 advance by an OU step driven by
// Philox4x32-10 normals (solenoidal projection as glmmhd_turb.jl:2104-2108 with comp_frac = 0);
// the per-row table B[kx][c] = sum_{modes with kx} ahat_c e^{i(ky y + kz z)} turns the step
// kernel's mode sum into 4 complex multiply-adds per component.
#include <cstdio>

#include "gmt_internal.h"

namespace gmt {

__constant__ int c_mode_k[NMODES * 3];

// ------------------------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) cfl_kernel(const CPlanes<R> u, size_t n, const Consts<R> K,
                                                  unsigned long long* out) {
    __shared__ double red[32];
    double cm = 0.0, sm = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        Q9<R> c;
#pragma unroll
        for (int v = 0; v < 9; ++v) c.v[v] = u.p[v][i];
        R ct, sg;
        cfl_speeds(c, K, ct, sg);
        cm = fmax(cm, (double)ct);
        sm = fmax(sm, (double)sg);
    }
    block_max_atomic(cm, out, red);
    __syncthreads();
    block_max_atomic(sm, out + 1, red);
}

// FP32, four cells per thread: one 16-byte load per plane; the maxima are the scalar kernel's exactly
__global__ void __launch_bounds__(256) cfl_kernel4(const CPlanes<float> u, size_t n, const Consts<float> K,
                                                   unsigned long long* out) {
    __shared__ double red[32];
    double cm = 0.0, sm = 0.0;
    const size_t nq = n / 4;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += (size_t)gridDim.x * blockDim.x) {
        float4 v[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) v[k] = __ldg(reinterpret_cast<const float4*>(u.p[k]) + q);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            Q9<float> c;
#pragma unroll
            for (int k = 0; k < 9; ++k) c.v[k] = j == 0 ? v[k].x : (j == 1 ? v[k].y : (j == 2 ? v[k].z : v[k].w));
            float ct, sg;
            cfl_speeds(c, K, ct, sg);
            cm = fmax(cm, (double)ct);
            sm = fmax(sm, (double)sg);
        }
    }
    block_max_atomic(cm, out, red);
    __syncthreads();
    block_max_atomic(sm, out + 1, red);
}

template <class R>
cudaError_t launch_cfl(const CPlanes<R>& u, size_t n, const Consts<R>& K, unsigned long long* out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), s);
    if constexpr (std::is_same<R, float>::value) {
        bool quad = n % 4 == 0;
        for (int v = 0; v < 9; ++v) quad = quad && (reinterpret_cast<uintptr_t>(u.p[v]) & 15u) == 0;
        if (quad) {
            const int nb4 = (int)std::min<size_t>((n / 4 + 255) / 256, 148 * 8);
            cfl_kernel4<<<nb4, 256, 0, s>>>(u, n, K, out);
            return cudaGetLastError();
        }
    }
    int nb = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
    cfl_kernel<R><<<nb, 256, 0, s>>>(u, n, K, out);
    return cudaGetLastError();
}

// CT: cell prims from the face-averaged field
template <class R>
__global__ void __launch_bounds__(256) ct_cfl_kernel(const CPlanes8<R> qv, int nx, int ny, int nz, const Consts<R> K,
                                                     unsigned long long* out) {
    __shared__ double red[32];
    const R* const* q = qv.p;
    size_t n = (size_t)nx * ny * nz;
    double cm = 0.0, sm = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_coords(i, nx, ny, n, x, y, z);   // 32-bit divisions below 2^32 cells
        size_t ixp = (size_t)wrapi(x + 1, nx) + (size_t)nx * (y + (size_t)ny * z);
        size_t iyp = (size_t)x + (size_t)nx * (wrapi(y + 1, ny) + (size_t)ny * z);
        size_t izp = (size_t)x + (size_t)nx * (y + (size_t)ny * wrapi(z + 1, nz));
        Q9<R> c;
#pragma unroll
        for (int v = 0; v < 5; ++v) c.v[v] = q[v][i];
        c.v[5] = R(0.5) * (q[5][i] + q[5][ixp]);
        c.v[6] = R(0.5) * (q[6][i] + q[6][iyp]);
        c.v[7] = R(0.5) * (q[7][i] + q[7][izp]);
        c.v[8] = R(0);
        R ct, sg;
        cfl_speeds(c, K, ct, sg);
        cm = fmax(cm, (double)ct);
        sm = fmax(sm, (double)sg);
    }
    block_max_atomic(cm, out, red);
    __syncthreads();
    block_max_atomic(sm, out + 1, red);
}

// FP32 CT CFL four cells x0..x0+3 (x0 = 4k) per thread: 16-byte loads, the +x face field of the
// quad from the quad and the next cell of the row (periodic); maxima exactly the one-cell pass's
__global__ void __launch_bounds__(256) ct_cfl_kernel4(const CPlanes8<float> qv, int nx, int ny, int nz,
                                                      const Consts<float> K, unsigned long long* out) {
    __shared__ double red[32];
    const float* const* q = qv.p;
    const size_t n = (size_t)nx * ny * nz, nq = n / 4;
    auto ld = [](const float* p, size_t i) { return __ldg(reinterpret_cast<const float4*>(p + i)); };
    auto el = [](const float4& v, int j) { return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w)); };
    double cm = 0.0, sm = 0.0;
    for (size_t qd = (size_t)blockIdx.x * blockDim.x + threadIdx.x; qd < nq; qd += (size_t)gridDim.x * blockDim.x) {
        const size_t c = 4 * qd;
        int x, y, z;
        cell_coords(c, nx, ny, n, x, y, z);
        const size_t iyp = (size_t)x + (size_t)nx * (wrap1(y + 1, ny) + (size_t)ny * z);
        const size_t izp = (size_t)x + (size_t)nx * (y + (size_t)ny * wrap1(z + 1, nz));
        float4 v[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) v[k] = ld(q[k], c);
        const float4 bx = ld(q[5], c), by = ld(q[6], c), bz = ld(q[7], c), byp = ld(q[6], iyp), bzp = ld(q[7], izp);
        const float bxn = __ldg(q[5] + (x + 4 == nx ? c + 4 - nx : c + 4));
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            Q9<float> cc;
#pragma unroll
            for (int k = 0; k < 5; ++k) cc.v[k] = el(v[k], j);
            cc.v[5] = 0.5f * (el(bx, j) + (j < 3 ? el(bx, j + 1) : bxn));
            cc.v[6] = 0.5f * (el(by, j) + el(byp, j));
            cc.v[7] = 0.5f * (el(bz, j) + el(bzp, j));
            cc.v[8] = 0.0f;
            float ct, sg;
            cfl_speeds(cc, K, ct, sg);
            cm = fmax(cm, (double)ct);
            sm = fmax(sm, (double)sg);
        }
    }
    block_max_atomic(cm, out, red);
    __syncthreads();
    block_max_atomic(sm, out + 1, red);
}

template <class R>
cudaError_t launch_ct_cfl(const CPlanes8<R>& q, int nx, int ny, int nz, const Consts<R>& K, unsigned long long* out,
                          cudaStream_t s) {
    size_t n = (size_t)nx * ny * nz;
    cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), s);
    if constexpr (std::is_same<R, float>::value) {
        bool quad = nx % 4 == 0;
        for (int v = 0; v < 8; ++v) quad = quad && (reinterpret_cast<uintptr_t>(q.p[v]) & 15u) == 0;
        if (quad) {
            const int nb4 = (int)std::min<size_t>((n / 4 + 255) / 256, 148 * 8);
            ct_cfl_kernel4<<<nb4, 256, 0, s>>>(q, nx, ny, nz, K, out);
            return cudaGetLastError();
        }
    }
    int nb = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
    ct_cfl_kernel<R><<<nb, 256, 0, s>>>(q, nx, ny, nz, K, out);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// diagnostics: 8 quantities per block, then a single-block fixed-order reduction
// ------------------------------------------------------------------------------------------
constexpr int NDIAG = 8;  // mass, ke2, etot, psi2, divb2, divbmax, rhomin, nonfinite

__device__ __forceinline__ void diag_combine(double* a, const double* b) {
    for (int k = 0; k < 5; ++k) a[k] += b[k];
    a[5] = fmax(a[5], b[5]);
    a[6] = fmin(a[6], b[6]);
    a[7] += b[7];
}

template <class R>
__global__ void __launch_bounds__(256) diag_kernel(const CPlanes<R> u, int nx, int ny, int nz, double dx, double smallr,
                                                   double* partials) {
    __shared__ double sh[256 * NDIAG];
    double acc[NDIAG] = {0, 0, 0, 0, 0, 0, 1e300, 0};
    const size_t n = (size_t)nx * ny * nz;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_coords(i, nx, ny, n, x, y, z);   // 32-bit divisions below 2^32 cells
        double rho = (double)u.p[0][i], mx = (double)u.p[1][i], my = (double)u.p[2][i], mz = (double)u.p[3][i];
        double ps = (double)u.p[8][i];
        acc[0] += rho;
        acc[1] += (mx * mx + my * my + mz * mz) / fmax(rho, smallr);
        acc[2] += (double)u.p[4][i];
        acc[3] += ps * ps;
        auto at = [&](int a, int b, int c) {
            return (size_t)wrapi(a, nx) + (size_t)nx * ((size_t)wrapi(b, ny) + (size_t)ny * wrapi(c, nz));
        };
        double bxp = u.p[5][at(x + 1, y, z)], bxm = u.p[5][at(x - 1, y, z)];
        double byp = u.p[6][at(x, y + 1, z)], bym = u.p[6][at(x, y - 1, z)];
        double bzp = u.p[7][at(x, y, z + 1)], bzm = u.p[7][at(x, y, z - 1)];
        double db = fabs((bxp - bxm) + (byp - bym) + (bzp - bzm)) / (2.0 * dx);
        acc[4] += db * db;
        acc[5] = fmax(acc[5], db);
        acc[6] = fmin(acc[6], rho);
        bool fin = true;
#pragma unroll
        for (int v = 0; v < 9; ++v) fin = fin && isfinite((double)u.p[v][i]);
        acc[7] += fin ? 0.0 : 1.0;
    }
    for (int k = 0; k < NDIAG; ++k) sh[threadIdx.x * NDIAG + k] = acc[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) diag_combine(&sh[threadIdx.x * NDIAG], &sh[(threadIdx.x + s) * NDIAG]);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < NDIAG; ++k) partials[blockIdx.x * NDIAG + k] = sh[k];
}

__global__ void __launch_bounds__(256) diag_final(const double* partials, int nb, double* out) {
    __shared__ double sh[256 * NDIAG];
    double acc[NDIAG] = {0, 0, 0, 0, 0, 0, 1e300, 0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) diag_combine(acc, partials + b * NDIAG);
    for (int k = 0; k < NDIAG; ++k) sh[threadIdx.x * NDIAG + k] = acc[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) diag_combine(&sh[threadIdx.x * NDIAG], &sh[(threadIdx.x + s) * NDIAG]);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < NDIAG; ++k) out[k] = sh[k];
}

// FP32 diagnostics four cells x0..x0+3 (x0 = 4k) per thread: 16-byte loads of every plane, the
// x neighbours of Bx from the quad plus the cells either side of it (periodic); each cell's
// contributions are the scalar kernel's, accumulated in FP64 in cell order within the quad.
__global__ void __launch_bounds__(256) diag_kernel4(const CPlanes<float> u, int nx, int ny, int nz, double dx,
                                                    double smallr, double* partials) {
    __shared__ double sh[256 * NDIAG];
    double acc[NDIAG] = {0, 0, 0, 0, 0, 0, 1e300, 0};
    const size_t n = (size_t)nx * ny * nz, nq = n / 4;
    auto ld = [](const float* p, size_t i) { return __ldg(reinterpret_cast<const float4*>(p + i)); };
    auto el = [](const float4& v, int j) { return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w)); };
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += (size_t)gridDim.x * blockDim.x) {
        const size_t c = 4 * q;
        int x, y, z;
        cell_coords(c, nx, ny, n, x, y, z);
        const size_t cyp = (size_t)x + (size_t)nx * (wrap1(y + 1, ny) + (size_t)ny * z);
        const size_t cym = (size_t)x + (size_t)nx * (wrap1(y - 1, ny) + (size_t)ny * z);
        const size_t czp = (size_t)x + (size_t)nx * (y + (size_t)ny * wrap1(z + 1, nz));
        const size_t czm = (size_t)x + (size_t)nx * (y + (size_t)ny * wrap1(z - 1, nz));
        float4 v[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) v[k] = ld(u.p[k], c);
        const float4 byp = ld(u.p[6], cyp), bym = ld(u.p[6], cym), bzp = ld(u.p[7], czp), bzm = ld(u.p[7], czm);
        const float bxl = __ldg(u.p[5] + (x == 0 ? c + nx - 1 : c - 1));       // cell x0-1
        const float bxr = __ldg(u.p[5] + (x + 4 == nx ? c + 4 - nx : c + 4));  // cell x0+4
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double rho = (double)el(v[0], j), mx = (double)el(v[1], j), my = (double)el(v[2], j),
                         mz = (double)el(v[3], j), ps = (double)el(v[8], j);
            acc[0] += rho;
            acc[1] += (mx * mx + my * my + mz * mz) / fmax(rho, smallr);
            acc[2] += (double)el(v[4], j);
            acc[3] += ps * ps;
            const double bxp = j < 3 ? el(v[5], j + 1) : bxr, bxm = j > 0 ? el(v[5], j - 1) : bxl;
            const double byp_ = el(byp, j), bym_ = el(bym, j), bzp_ = el(bzp, j), bzm_ = el(bzm, j);
            const double db = fabs((bxp - bxm) + (byp_ - bym_) + (bzp_ - bzm_)) / (2.0 * dx);
            acc[4] += db * db;
            acc[5] = fmax(acc[5], db);
            acc[6] = fmin(acc[6], rho);
            bool fin = true;
#pragma unroll
            for (int k = 0; k < 9; ++k) fin = fin && isfinite((double)el(v[k], j));
            acc[7] += fin ? 0.0 : 1.0;
        }
    }
    for (int k = 0; k < NDIAG; ++k) sh[threadIdx.x * NDIAG + k] = acc[k];
    __syncthreads();
    for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
        if ((int)threadIdx.x < s2) diag_combine(&sh[threadIdx.x * NDIAG], &sh[(threadIdx.x + s2) * NDIAG]);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < NDIAG; ++k) partials[blockIdx.x * NDIAG + k] = sh[k];
}

template <class R>
cudaError_t launch_diag(const CPlanes<R>& u, int nx, int ny, int nz, double dx, double smallr, double* partials,
                        int nblocks, double* out, cudaStream_t s) {
    bool quad = false;
    if constexpr (std::is_same<R, float>::value) {
        quad = nx % 4 == 0 && nx >= 8;
        for (int v = 0; v < 9; ++v) quad = quad && (reinterpret_cast<uintptr_t>(u.p[v]) & 15u) == 0;
    }
    if constexpr (std::is_same<R, float>::value) {
        if (quad) {
            diag_kernel4<<<nblocks, 256, 0, s>>>(u, nx, ny, nz, dx, smallr, partials);
            diag_final<<<1, 256, 0, s>>>(partials, nblocks, out);
            return cudaGetLastError();
        }
    }
    diag_kernel<R><<<nblocks, 256, 0, s>>>(u, nx, ny, nz, dx, smallr, partials);
    diag_final<<<1, 256, 0, s>>>(partials, nblocks, out);
    return cudaGetLastError();
}

// CT face div B max: (upper - lower)/dx per dim (ct_mhd.jl:190-194)
template <class R>
__global__ void __launch_bounds__(256) ct_divb_kernel(const CPlanes8<R> qv, int nx, int ny, int nz, double dx,
                                                      unsigned long long* out) {
    __shared__ double red[32];
    const R* bx = qv.p[5];
    const R* by = qv.p[6];
    const R* bz = qv.p[7];
    size_t n = (size_t)nx * ny * nz;
    double m = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_coords(i, nx, ny, n, x, y, z);   // 32-bit divisions below 2^32 cells
        size_t ixp = (size_t)wrapi(x + 1, nx) + (size_t)nx * (y + (size_t)ny * z);
        size_t iyp = (size_t)x + (size_t)nx * (wrapi(y + 1, ny) + (size_t)ny * z);
        size_t izp = (size_t)x + (size_t)nx * (y + (size_t)ny * wrapi(z + 1, nz));
        double d = ((double)bx[ixp] - (double)bx[i] + (double)by[iyp] - (double)by[i] + (double)bz[izp] -
                    (double)bz[i]) / dx;
        m = fmax(m, fabs(d));
    }
    block_max_atomic(m, out, red);
}

template <class R>
cudaError_t launch_ct_divb(const CPlanes8<R>& q, int nx, int ny, int nz, double dx, unsigned long long* out,
                           cudaStream_t s) {
    size_t n = (size_t)nx * ny * nz;
    int nb = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
    cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
    ct_divb_kernel<R><<<nb, 256, 0, s>>>(q, nx, ny, nz, dx, out);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// forcing
// ------------------------------------------------------------------------------------------
cudaError_t mode_table_device(const int** ptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, c_mode_k);
    *ptr = static_cast<const int*>(p);
    return e;
}

cudaError_t upload_mode_table() {
    int k[NMODES * 3];
    int n = 0;
    for (int kx = 0; kx <= 3; ++kx)
        for (int ky = -3; ky <= 3; ++ky)
            for (int kz = -3; kz <= 3; ++kz) {
                int k2 = kx * kx + ky * ky + kz * kz;
                if (k2 < 1 || k2 > 9) continue;
                bool half = kx > 0 || (kx == 0 && ky > 0) || (kx == 0 && ky == 0 && kz > 0);
                if (!half) continue;
                if (n < NMODES) { k[3 * n] = kx; k[3 * n + 1] = ky; k[3 * n + 2] = kz; }
                ++n;
            }
    if (n != NMODES) return cudaErrorInvalidValue;
    return cudaMemcpyToSymbol(c_mode_k, k, sizeof(k));
}

__global__ void ou_update_kernel(double* modes, uint32_t seed, uint32_t counter, double alpha, double beta,
                                 double sigma0) {
    int q = threadIdx.x;
    if (q >= NMODES) return;
    ou_mode_update(modes, q, c_mode_k[3 * q], c_mode_k[3 * q + 1], c_mode_k[3 * q + 2], seed, counter, alpha, beta,
                   sigma0);
}

cudaError_t launch_ou_update(double* modes, uint32_t seed, uint32_t counter, double alpha, double beta, double sigma0,
                             cudaStream_t s) {
    ou_update_kernel<<<1, 64, 0, s>>>(modes, seed, counter, alpha, beta, sigma0);
    return cudaGetLastError();
}

// B[kx][c] per (y,z) row, same summation order as the oracle's Forcer::accel
template <class R>
__global__ void __launch_bounds__(256) btab_kernel(const double* modes, const R* trigy, const R* trigz, int ny, int nz,
                                                   R* btab) {
    int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= ny * nz) return;
    btab_row(modes, c_mode_k, trigy, trigz, ny, nz, row % ny, row / ny, btab + (size_t)row * 24);
}

template <class R>
cudaError_t launch_btab(const double* modes, const R* trigy, const R* trigz, int ny, int nz, R* btab, cudaStream_t s) {
    int rows = ny * nz;
    btab_kernel<R><<<(rows + 255) / 256, 256, 0, s>>>(modes, trigy, trigz, ny, nz, btab);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// initial conditions
// ------------------------------------------------------------------------------------------
template <class R>
__global__ void ic_ot_kernel(const Planes<R> u, int nx, int ny, int nz, double gamma) {
    size_t n = (size_t)nx * ny * nz;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(c % nx), j = (int)((c / nx) % ny);
        const double pi = 3.14159265358979323846, twopi = 2.0 * pi;
        double x = (i + 0.5) / nx, y = (j + 0.5) / ny;
        double rho = 25.0 / (36.0 * pi), pr = 5.0 / (12.0 * pi);
        double vx = -sin(twopi * y), vy = sin(twopi * x);
        double sb = 1.0 / sqrt(4.0 * pi);
        double bx = -sb * sin(twopi * y), by = sb * sin(2.0 * twopi * x);
        double ekin = 0.5 * rho * (vx * vx + vy * vy), emag = 0.5 * (bx * bx + by * by);
        double v9[9] = {rho, rho * vx, rho * vy, 0.0, pr / (gamma - 1.0) + ekin + emag, bx, by, 0.0, 0.0};
#pragma unroll
        for (int v = 0; v < 9; ++v) u.p[v][c] = (R)v9[v];
    }
}

template <class R>
cudaError_t launch_ic_ot(const Planes<R>& u, int nx, int ny, int nz, double gamma, cudaStream_t s) {
    size_t n = (size_t)nx * ny * nz;
    int nb = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    ic_ot_kernel<R><<<nb, 256, 0, s>>>(u, nx, ny, nz, gamma);
    return cudaGetLastError();
}

template <class R> struct V9 { double v[9]; };

template <class R>
__global__ void ic_uniform_kernel(const Planes<R> u, size_t n, const V9<R> val) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int v = 0; v < 9; ++v) u.p[v][c] = (R)val.v[v];
    }
}

template <class R>
cudaError_t launch_ic_uniform(const Planes<R>& u, size_t n, const double v9[9], cudaStream_t s) {
    V9<R> val;
    for (int v = 0; v < 9; ++v) val.v[v] = v9[v];
    int nb = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    ic_uniform_kernel<R><<<nb, 256, 0, s>>>(u, n, val);
    return cudaGetLastError();
}

template <class R>
__global__ void ct_ic_ot_kernel(const Planes8<R> qv, int nx, int ny, int nz, double gamma, int phase) {
    R* const* q = qv.p;
    size_t n = (size_t)nx * ny * nz;
    const double pi = 3.14159265358979323846, twopi = 2.0 * pi;
    const double sb = 1.0 / sqrt(4.0 * pi);
    const double dx = 1.0 / nx, dy = 1.0 / ny;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((size_t)nx * ny));
        auto Az = [&](double x, double y) {
            return sb * (cos(twopi * y) / twopi + cos(2.0 * twopi * x) / (2.0 * twopi));
        };
        if (phase == 0) {
            double xl = i * dx, yl = j * dy;
            q[5][c] = (R)((Az(xl, yl + dy) - Az(xl, yl)) / dy);
            q[6][c] = (R)(-(Az(xl + dx, yl) - Az(xl, yl)) / dx);
            q[7][c] = (R)0;
        } else {
            double x = (i + 0.5) * dx, y = (j + 0.5) * dy;
            double rho = 25.0 / (36.0 * pi), pr = 5.0 / (12.0 * pi);
            double vx = -sin(twopi * y), vy = sin(twopi * x);
            size_t cxp = (size_t)wrapi(i + 1, nx) + (size_t)nx * (j + (size_t)ny * k);
            size_t cyp = (size_t)i + (size_t)nx * (wrapi(j + 1, ny) + (size_t)ny * k);
            double bx = 0.5 * ((double)q[5][c] + (double)q[5][cxp]);
            double by = 0.5 * ((double)q[6][c] + (double)q[6][cyp]);
            double ekin = 0.5 * rho * (vx * vx + vy * vy), emag = 0.5 * (bx * bx + by * by);
            q[0][c] = (R)rho; q[1][c] = (R)(rho * vx); q[2][c] = (R)(rho * vy); q[3][c] = (R)0;
            q[4][c] = (R)(pr / (gamma - 1.0) + ekin + emag);
        }
    }
}

template <class R>
cudaError_t launch_ct_ic_ot(const Planes8<R>& q, int nx, int ny, int nz, double gamma, cudaStream_t s) {
    size_t n = (size_t)nx * ny * nz;
    int nb = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    ct_ic_ot_kernel<R><<<nb, 256, 0, s>>>(q, nx, ny, nz, gamma, 0);
    ct_ic_ot_kernel<R><<<nb, 256, 0, s>>>(q, nx, ny, nz, gamma, 1);
    return cudaGetLastError();
}

// Seeded synthetic turbulent state: uniform (rho0, p0, B0) with v = vscale*a(x), dB = bscale*a(x),
// rho = rho0*exp(0.2*a_y(x)), where a(x) is one stationary draw of the solenoidal 61-mode field
// with unit rms (the forcing's own mode sum).  Stand-in for a pre-evolved turbulent checkpoint.
template <class R>
__global__ void ic_turb_kernel(const Planes<R> u, int nx, int ny, int nz, const R* btab, const R* trigx, double rho0,
                               double p0, double b0x, double b0y, double b0z, double vscale, double bscale,
                               double gamma) {
    size_t n = (size_t)nx * ny * nz;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((size_t)nx * ny));
        R ax, ay, az;
        force_accel(btab + ((size_t)k * ny + j) * 24, trigx, nx, i, R(1), ax, ay, az);
        double rho = rho0 * exp(0.2 * (double)ay);
        double vx = vscale * (double)ax, vy = vscale * (double)ay, vz = vscale * (double)az;
        double bx = b0x + bscale * (double)ax, by = b0y + bscale * (double)ay, bz = b0z + bscale * (double)az;
        double e = p0 / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz) + 0.5 * (bx * bx + by * by + bz * bz);
        double v9[9] = {rho, rho * vx, rho * vy, rho * vz, e, bx, by, bz, 0.0};
#pragma unroll
        for (int v = 0; v < 9; ++v) u.p[v][c] = (R)v9[v];
    }
}

template <class R>
cudaError_t launch_ic_turb(const Planes<R>& u, int nx, int ny, int nz, const R* btab, const R* trigx, double rho0,
                           double p0, const double b0[3], double vscale, double bscale, double gamma, cudaStream_t s) {
    size_t n = (size_t)nx * ny * nz;
    int nb = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    ic_turb_kernel<R><<<nb, 256, 0, s>>>(u, nx, ny, nz, btab, trigx, rho0, p0, b0[0], b0[1], b0[2], vscale, bscale,
                                        gamma);
    return cudaGetLastError();
}

// Turbulent CT state: the GLM state's density and velocity (one unit-rms draw a(x) of the 61-mode
// solenoidal field, evaluated at cell centres by direct mode sum), and face fields
// B = B0 + curl(A) with A = db / (4 pi) a evaluated on the cell edges.  The discrete curl of an
// edge potential has zero face divergence to round-off.
__device__ __forceinline__ void mode_field(const double* modes, double x, double y, double z, double a[3]) {
    a[0] = a[1] = a[2] = 0.0;
    const double twopi = 6.283185307179586476925286766559;
    for (int q = 0; q < NMODES; ++q) {
        const double ph = twopi * (c_mode_k[3 * q] * x + c_mode_k[3 * q + 1] * y + c_mode_k[3 * q + 2] * z);
        double sn, cs;
        sincos(ph, &sn, &cs);
#pragma unroll
        for (int c = 0; c < 3; ++c) a[c] += 2.0 * (modes[(q * 3 + c) * 2] * cs - modes[(q * 3 + c) * 2 + 1] * sn);
    }
}

// pass 1: edge potentials Ax (i, j-1/2, k-1/2), Ay (i-1/2, j, k-1/2), Az (i-1/2, j-1/2, k) of every cell
template <class R>
__global__ void ct_turb_edges_kernel(R* ax, R* ay, R* az, int nx, int ny, int nz, const double* modes, double scale) {
    const size_t n = (size_t)nx * ny * nz;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((size_t)nx * ny));
        const double x = (i + 0.5) / nx, y = (j + 0.5) / ny, z = (k + 0.5) / nz;
        const double xl = (double)i / nx, yl = (double)j / ny, zl = (double)k / nz;
        double a[3];
        mode_field(modes, x, yl, zl, a);
        ax[c] = (R)(scale * a[0]);
        mode_field(modes, xl, y, zl, a);
        ay[c] = (R)(scale * a[1]);
        mode_field(modes, xl, yl, z, a);
        az[c] = (R)(scale * a[2]);
    }
}

// pass 2: rho, momentum at cell centres and face B = B0 + curl A (lower faces)
template <class R>
__global__ void ct_turb_faces_kernel(const Planes8<R> q, const R* ax, const R* ay, const R* az, int nx, int ny, int nz,
                                     const double* modes, double rho0, double vscale, double b0x, double b0y, double b0z) {
    const size_t n = (size_t)nx * ny * nz;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((size_t)nx * ny));
        const size_t cyp = (size_t)i + (size_t)nx * (wrapi(j + 1, ny) + (size_t)ny * k);
        const size_t czp = (size_t)i + (size_t)nx * (j + (size_t)ny * wrapi(k + 1, nz));
        const size_t cxp = (size_t)wrapi(i + 1, nx) + (size_t)nx * (j + (size_t)ny * k);
        // Bx(i-1/2, j, k) = dAz/dy - dAy/dz;  By(i, j-1/2, k) = dAx/dz - dAz/dx;  Bz(i, j, k-1/2) = dAy/dx - dAx/dy
        q.p[5][c] = (R)(b0x + ((double)az[cyp] - (double)az[c]) * ny - ((double)ay[czp] - (double)ay[c]) * nz);
        q.p[6][c] = (R)(b0y + ((double)ax[czp] - (double)ax[c]) * nz - ((double)az[cxp] - (double)az[c]) * nx);
        q.p[7][c] = (R)(b0z + ((double)ay[cxp] - (double)ay[c]) * nx - ((double)ax[cyp] - (double)ax[c]) * ny);
        double a[3];
        mode_field(modes, (i + 0.5) / nx, (j + 0.5) / ny, (k + 0.5) / nz, a);
        const double rho = rho0 * exp(0.2 * a[1]);
        q.p[0][c] = (R)rho;
        q.p[1][c] = (R)(rho * vscale * a[0]);
        q.p[2][c] = (R)(rho * vscale * a[1]);
        q.p[3][c] = (R)(rho * vscale * a[2]);
    }
}

// pass 3: total energy with the face-averaged field
template <class R>
__global__ void ct_turb_energy_kernel(const Planes8<R> q, int nx, int ny, int nz, double p0, double gamma) {
    const size_t n = (size_t)nx * ny * nz;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((size_t)nx * ny));
        const size_t cxp = (size_t)wrapi(i + 1, nx) + (size_t)nx * (j + (size_t)ny * k);
        const size_t cyp = (size_t)i + (size_t)nx * (wrapi(j + 1, ny) + (size_t)ny * k);
        const size_t czp = (size_t)i + (size_t)nx * (j + (size_t)ny * wrapi(k + 1, nz));
        const double bx = 0.5 * ((double)q.p[5][c] + (double)q.p[5][cxp]);
        const double by = 0.5 * ((double)q.p[6][c] + (double)q.p[6][cyp]);
        const double bz = 0.5 * ((double)q.p[7][c] + (double)q.p[7][czp]);
        const double rho = q.p[0][c], mx = q.p[1][c], my = q.p[2][c], mz = q.p[3][c];
        q.p[4][c] = (R)(p0 / (gamma - 1.0) + 0.5 * (mx * mx + my * my + mz * mz) / rho + 0.5 * (bx * bx + by * by + bz * bz));
    }
}

template <class R>
cudaError_t launch_ct_ic_turb(const Planes8<R>& q, int nx, int ny, int nz, const double* modes, R* scratch, double rho0,
                              double p0, const double b0[3], double vscale, double db, double gamma, cudaStream_t s) {
    const size_t n = (size_t)nx * ny * nz;
    const int nb = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    const double scale = db / (4.0 * 3.141592653589793238462643383279);
    ct_turb_edges_kernel<R><<<nb, 256, 0, s>>>(scratch, scratch + n, scratch + 2 * n, nx, ny, nz, modes, scale);
    ct_turb_faces_kernel<R><<<nb, 256, 0, s>>>(q, scratch, scratch + n, scratch + 2 * n, nx, ny, nz, modes, rho0, vscale,
                                               b0[0], b0[1], b0[2]);
    ct_turb_energy_kernel<R><<<nb, 256, 0, s>>>(q, nx, ny, nz, p0, gamma);
    return cudaGetLastError();
}

#define GMT_INST(R)                                                                                              \
    template cudaError_t launch_cfl<R>(const CPlanes<R>&, size_t, const Consts<R>&, unsigned long long*,         \
                                       cudaStream_t);                                                            \
    template cudaError_t launch_ct_cfl<R>(const CPlanes8<R>&, int, int, int, const Consts<R>&, unsigned long long*, \
                                          cudaStream_t);                                                         \
    template cudaError_t launch_diag<R>(const CPlanes<R>&, int, int, int, double, double, double*, int, double*, \
                                        cudaStream_t);                                                           \
    template cudaError_t launch_ct_divb<R>(const CPlanes8<R>&, int, int, int, double, unsigned long long*,          \
                                           cudaStream_t);                                                        \
    template cudaError_t launch_btab<R>(const double*, const R*, const R*, int, int, R*, cudaStream_t);          \
    template cudaError_t launch_ic_ot<R>(const Planes<R>&, int, int, int, double, cudaStream_t);                 \
    template cudaError_t launch_ic_uniform<R>(const Planes<R>&, size_t, const double*, cudaStream_t);            \
    template cudaError_t launch_ic_turb<R>(const Planes<R>&, int, int, int, const R*, const R*, double, double,       \
                                           const double*, double, double, double, cudaStream_t);                 \
    template cudaError_t launch_ct_ic_ot<R>(const Planes8<R>&, int, int, int, double, cudaStream_t);                \
    template cudaError_t launch_ct_ic_turb<R>(const Planes8<R>&, int, int, int, const double*, R*, double, double,   \
                                              const double*, double, double, double, cudaStream_t);
GMT_INST(float)
GMT_INST(double)

}  // namespace gmt
