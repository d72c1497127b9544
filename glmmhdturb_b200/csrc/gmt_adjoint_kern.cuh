// gmt_adjoint_kern.cuh -- the six grid-stride kernels of the discrete adjoint of the unsplit step
// (one thread per cell; the per-cell passes are in gmt_adjoint.cuh) and their launcher.  Included
// by gmt_adjoint.cu (FP64, IEEE, bit-stable) and gmt_adjoint_f32.cu (FP32, fast math like the FP32
// forward step).
#pragma once
#include <algorithm>

#include "gmt_adjoint.cuh"

namespace gmt {

#define GMT_ADJ_LOOP for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)

template <class R> __global__ void __launch_bounds__(128) adj_faces_kernel(const AdjArgs<R> A) {
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    GMT_ADJ_LOOP adj_faces_cell(A, c);
}
template <int RIEM, class R> __global__ void __launch_bounds__(128) adj_flux_kernel(const AdjArgs<R> A) {
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    GMT_ADJ_LOOP adj_flux_cell<RIEM>(A, c);
}
template <class R> __global__ void __launch_bounds__(128) adj_update_kernel(const AdjArgs<R> A) {
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    __shared__ double red[128];
    double damp = 0.0;
    GMT_ADJ_LOOP damp += adj_update_cell(A, c);
    red[threadIdx.x] = damp;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0 && A.damp) atomicAdd(A.damp, red[0]);
}
template <int RIEM, bool DUALS, class R> __global__ void __launch_bounds__(128, 3) adj_riemann_kernel(const AdjArgs<R> A) {
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    GMT_ADJ_LOOP adj_riemann_cell<RIEM, DUALS>(A, c);
}
template <class R> __global__ void __launch_bounds__(128, 3) adj_recon_kernel(const AdjArgs<R> A) {
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    GMT_ADJ_LOOP adj_recon_cell(A, c);
}
template <class R> __global__ void __launch_bounds__(128) adj_gather_kernel(const AdjArgs<R> A) {
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    GMT_ADJ_LOOP adj_gather_cell(A, c);
}

template <class R> cudaError_t launch_adjoint_t(const AdjArgs<R>& A, cudaStream_t s) {
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    const int nb = (int)std::min<size_t>((n + 127) / 128, 148 * 16);
    adj_faces_kernel<R><<<nb, 128, 0, s>>>(A);
    if (A.riem == RIEM_HLL) adj_flux_kernel<RIEM_HLL, R><<<nb, 128, 0, s>>>(A);
    else if (A.riem == RIEM_LLF_BOUND) adj_flux_kernel<RIEM_LLF_BOUND, R><<<nb, 128, 0, s>>>(A);
    else adj_flux_kernel<RIEM_HLLD, R><<<nb, 128, 0, s>>>(A);
    adj_update_kernel<R><<<nb, 128, 0, s>>>(A);
    const bool llf_switch = A.use_llf || A.K.llf_dmin > R(0) || A.K.llf_pmin > R(0);
    if (A.riem == RIEM_HLL) adj_riemann_kernel<RIEM_HLL, false, R><<<nb, 128, 0, s>>>(A);
    else if (A.riem == RIEM_LLF_BOUND) adj_riemann_kernel<RIEM_LLF_BOUND, true, R><<<nb, 128, 0, s>>>(A);
    else if (llf_switch) adj_riemann_kernel<RIEM_HLLD, true, R><<<nb, 128, 0, s>>>(A);
    else adj_riemann_kernel<RIEM_HLLD, false, R><<<nb, 128, 0, s>>>(A);
    adj_recon_kernel<R><<<nb, 128, 0, s>>>(A);
    adj_gather_kernel<R><<<nb, 128, 0, s>>>(A);
    return cudaGetLastError();
}

// one unit instantiates it per real type (gmt_adjoint.cu: double, gmt_adjoint_f32.cu: float)
template <class R> cudaError_t launch_adjoint(const AdjArgs<R>& A, cudaStream_t s) { return launch_adjoint_t(A, s); }

}  // namespace gmt
