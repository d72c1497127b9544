// gmt_noalloc.cu -- diagnostics of a GLM state without any allocation: gmt_diagnostics_noalloc.
//
// Who needs it: callers that must not allocate device memory.
//  - A driver loop that logs diagnostics every few steps.  cudaMalloc and cudaFree synchronise
//    the whole device, which would stall the step pipeline the driver is keeping busy.
//  - A host framework that owns the GPU memory budget through its own pool (a Julia CUDA.jl or
//    PyTorch caching allocator holding the device at its limit).  An allocation behind that
//    pool's back can fail or evict the pool's memory.
//  - A monitoring hook that is handed only a device pointer to the state and has no
//    gmt_create context (whose creation allocates).
//
// The scratch is one file-scope static __device__ array, part of the library image, so every GPU
// that loads the library holds it until the process exits.  It has one row of 8 partial sums per
// z-plane (at most GMT_NOALLOC_MAX_PLANES planes) plus the 8 final values.  Host code cannot pass
// the array's name to a kernel: in host code that name is only a host-side stand-in, not a
// device address.  So the first call on each device, with that device current, looks the address
// up once with cudaGetSymbolAddress and keeps it.  Make that first call on a device before any
// stream capture begins.
//
// Nothing in the array has to start at zero: each call writes every partial row it reads, and
// the final row, before reading them.  All calls share the one array, so calls that can overlap
// on the GPU (on different streams, or from different host threads) race on it and must be
// serialised by the caller.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/glmmhd_b200.h"
#include "gmt_internal.h"

namespace {

constexpr int kMaxPlanes = GMT_NOALLOC_MAX_PLANES;
constexpr int kQ = 8;  // mass, ke2, etot, psi2, divb2, divbmax, rhomin, nonfinite

static __device__ __align__(256) double g_diag_scratch[(kMaxPlanes + 1) * kQ];

std::mutex g_mu;
double* g_scratch_dev[64] = {nullptr};

// the message is reported through gmt_last_error() of the calling thread
int fail(int code, const std::string& m) {
    gmt::set_last_error(m);
    return code;
}

__device__ __forceinline__ void combine(double* a, const double* b) {
    for (int k = 0; k < 5; ++k) a[k] += b[k];
    a[5] = fmax(a[5], b[5]);
    a[6] = fmin(a[6], b[6]);
    a[7] += b[7];
}

__device__ __forceinline__ void block_reduce_store(double* acc, double* sh, double* dst) {
    for (int k = 0; k < kQ; ++k) sh[threadIdx.x * kQ + k] = acc[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) combine(&sh[threadIdx.x * kQ], &sh[(threadIdx.x + s) * kQ]);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < kQ; ++k) dst[k] = sh[k];
}

// one block per z-plane: the same quantities as diag_kernel, written to row k of the scratch
template <class R>
__global__ void __launch_bounds__(256) diag_plane_kernel(const gmt::CPlanes<R> u, int nx, int ny, int nz, double dx,
                                                         double smallr, double* scratch) {
    __shared__ double sh[256 * kQ];
    double acc[kQ] = {0, 0, 0, 0, 0, 0, 1e300, 0};
    const int k = blockIdx.x;
    const size_t plane = (size_t)nx * ny;
    auto at = [&](int a, int b, int c) {
        return (size_t)gmt::wrapi(a, nx) + (size_t)nx * ((size_t)gmt::wrapi(b, ny) + (size_t)ny * gmt::wrapi(c, nz));
    };
    for (size_t c = threadIdx.x; c < plane; c += blockDim.x) {
        int x = (int)(c % nx), y = (int)(c / nx);
        size_t i = c + plane * k;
        double rho = (double)u.p[0][i], mx = (double)u.p[1][i], my = (double)u.p[2][i], mz = (double)u.p[3][i];
        double ps = (double)u.p[8][i];
        acc[0] += rho;
        acc[1] += (mx * mx + my * my + mz * mz) / fmax(rho, smallr);
        acc[2] += (double)u.p[4][i];
        acc[3] += ps * ps;
        double db = fabs(((double)u.p[5][at(x + 1, y, k)] - (double)u.p[5][at(x - 1, y, k)]) +
                         ((double)u.p[6][at(x, y + 1, k)] - (double)u.p[6][at(x, y - 1, k)]) +
                         ((double)u.p[7][at(x, y, k + 1)] - (double)u.p[7][at(x, y, k - 1)])) / (2.0 * dx);
        acc[4] += db * db;
        acc[5] = fmax(acc[5], db);
        acc[6] = fmin(acc[6], rho);
        bool fin = true;
        for (int v = 0; v < 9; ++v) fin = fin && isfinite((double)u.p[v][i]);
        acc[7] += fin ? 0.0 : 1.0;
    }
    block_reduce_store(acc, sh, scratch + (size_t)k * kQ);
}

// rows 0..nz-1 -> final row kMaxPlanes
__global__ void __launch_bounds__(256) diag_plane_final(int nz, double* scratch) {
    __shared__ double sh[256 * kQ];
    double acc[kQ] = {0, 0, 0, 0, 0, 0, 1e300, 0};
    for (int r = threadIdx.x; r < nz; r += blockDim.x) combine(acc, scratch + (size_t)r * kQ);
    block_reduce_store(acc, sh, scratch + (size_t)kMaxPlanes * kQ);
}

// device address of the static scratch on the current device, looked up once per device
int scratch_for_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(GMT_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return fail(GMT_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_dev[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_diag_scratch);
        if (e != cudaSuccess || !p)
            return fail(GMT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_dev[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_dev[dev];
    return GMT_OK;
}

template <class R>
int run(const void* u, int nx, int ny, int nz, double boxlen, double smallr, gmt_diag* out, cudaStream_t s) {
    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != GMT_OK) return rc;
    gmt::CPlanes<R> P;
    const size_t n = (size_t)nx * ny * nz;
    for (int v = 0; v < 9; ++v) P.p[v] = static_cast<const R*>(u) + (size_t)v * n;
    diag_plane_kernel<R><<<nz, 256, 0, s>>>(P, nx, ny, nz, boxlen / nx, smallr, scratch);
    diag_plane_final<<<1, 256, 0, s>>>(nz, scratch);
    cudaError_t e = cudaGetLastError();
    double h[kQ];
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h, scratch + (size_t)kMaxPlanes * kQ, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(GMT_ERR_CUDA, std::string("gmt_diagnostics_noalloc: ") + cudaGetErrorString(e));
    out->mass = h[0];
    out->ke2 = h[1];
    out->etot = h[2];
    out->psi_l2 = std::sqrt(h[3] / (double)n);
    out->divb_l2 = std::sqrt(h[4] / (double)n);
    out->divbmax = h[5];
    out->rhomin = h[6];
    out->vrms = std::sqrt(h[1] / h[0]);
    out->nonfinite_cells = (int32_t)h[7];
    out->finite = h[7] == 0.0;
    return GMT_OK;
}

}  // namespace

extern "C" {

int gmt_diagnostics_noalloc(const void* u, int32_t nx, int32_t ny, int32_t nz, int32_t dtype, double boxlen,
                            double smallr, gmt_diag* out, void* stream) {
    if (!u || !out) return fail(GMT_ERR_ARG, "gmt_diagnostics_noalloc: null argument");
    if (nx < 1 || ny < 1 || nz < 1) return fail(GMT_ERR_ARG, "gmt_diagnostics_noalloc: grid dimensions must be >= 1");
    if (nz > kMaxPlanes)
        return fail(GMT_ERR_ARG, "gmt_diagnostics_noalloc: nz = " + std::to_string(nz) +
                                     " exceeds the static scratch of " + std::to_string(kMaxPlanes) + " z-planes");
    if (dtype != GMT_F32 && dtype != GMT_F64) return fail(GMT_ERR_ARG, "gmt_diagnostics_noalloc: dtype must be GMT_F32 or GMT_F64");
    if (!(boxlen > 0.0) || !(smallr > 0.0)) return fail(GMT_ERR_ARG, "gmt_diagnostics_noalloc: boxlen and smallr must be positive");
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == GMT_F64 ? run<double>(u, nx, ny, nz, boxlen, smallr, out, s)
                            : run<float>(u, nx, ny, nz, boxlen, smallr, out, s);
}

}  // extern "C"
