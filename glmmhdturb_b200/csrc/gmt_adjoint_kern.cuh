// gmt_adjoint_kern.cuh -- the six grid-stride kernels of the discrete adjoint of the unsplit step
// (one thread per cell; the per-cell passes are in gmt_adjoint.cuh) and their launcher.  Included
// by gmt_adjoint.cu (FP64, IEEE, bit-stable) and gmt_adjoint_f32.cu (FP32, fast math like the FP32
// forward step).
#pragma once
#include <algorithm>
#include <type_traits>

#include "gmt_adjoint.cuh"
#include "gmt_unsplit_inst.cuh"

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

// ---- passes 4 and 5 with their inputs staged through shared memory -----------------------------
// Both passes do much arithmetic per cell at a register budget that leaves 12 warps per SM, too few
// to hide the latency of their scratch loads.  Here every thread copies the inputs of its next cell
// (one grid stride ahead) into its own shared-memory slots by cp.async, so those loads are in
// flight while the current cell computes.  A thread reads only the slots it filled itself, so the
// per-thread cp.async group waits order everything and no block barrier is needed.  Slot s of a
// thread lives at S[s * ADJ_NT + threadIdx.x] (consecutive threads, consecutive banks).
constexpr int ADJ_NT = 128;
constexpr int RS_SLOTS = 3 * 27 + 2 * 9;   // per direction FS(c,+d), FS(c+d,-d), R1b(c+d); R1b(c) twice
constexpr int RC_SLOTS = 63 + 54;          // conserved stencil (7 cells), FSbar of the cell

template <class R> __device__ __forceinline__ size_t face_nbr(const Idx<R>& I, int x, int y, int z, int d) {
    return d == 0 ? I.at(x + 1, y, z) : (d == 1 ? I.at(x, y + 1, z) : I.at(x, y, z + 1));
}
__device__ __forceinline__ void compiler_fence() { asm volatile("" ::: "memory"); }

// inputs of direction d of cell c (and R1b(c) with direction 0, into buffer buf); an empty group
// past the end keeps the per-thread group count uniform
template <class R>
__device__ __forceinline__ void riemann_issue(const AdjArgs<R>& A, const Idx<R>& I, R* S, size_t c, int x, int y,
                                              int z, int d, int buf) {
    if (c < I.n) {
        const size_t cp = face_nbr(I, x, y, z, d);
        R* s = S + (size_t)(27 * d) * ADJ_NT;
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            cp_async_r(s + v * ADJ_NT, A.FS + (size_t)(2 * d * 9 + v) * I.n + c);
            cp_async_r(s + (9 + v) * ADJ_NT, A.FS + (size_t)((2 * d + 1) * 9 + v) * I.n + cp);
            cp_async_r(s + (18 + v) * ADJ_NT, A.R1b + (size_t)v * I.n + cp);
        }
        if (d == 0) {
#pragma unroll
            for (int v = 0; v < 9; ++v) cp_async_r(S + (size_t)(81 + 9 * buf + v) * ADJ_NT, A.R1b + (size_t)v * I.n + c);
        }
    }
    cp_async_commit();
}

template <int RIEM, bool DUALS, class R>
__global__ void __launch_bounds__(ADJ_NT, 3) adj_riemann_staged_kernel(const AdjArgs<R> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* S = reinterpret_cast<R*>(smem_raw) + threadIdx.x;
    const Idx<R> I = idx_of(A);
    const size_t stride = (size_t)gridDim.x * ADJ_NT;
    const bool ul = A.use_llf != 0;
    size_t c = (size_t)blockIdx.x * ADJ_NT + threadIdx.x;
    int x, y, z;   // coordinates of cell c
    cell_xyz(A, c, x, y, z);
#pragma unroll 1
    for (int d = 0; d < 3; ++d) riemann_issue(A, I, S, c, x, y, z, d, 0);
    int buf = 0;
    for (; c < I.n; c += stride, buf ^= 1) {
        int xn, yn, zn;   // coordinates of the next cell
        cell_xyz(A, c + stride, xn, yn, zn);
#pragma unroll 1
        for (int d = 0; d < 3; ++d) {
            cp_async_wait_group<2>();   // direction d of cell c has landed
            const R* s = S + (size_t)(27 * d) * ADJ_NT;
            Q9<R> L, Rr, Fb;
#pragma unroll
            for (int v = 0; v < 9; ++v) {
                L.v[v] = s[v * ADJ_NT];
                Rr.v[v] = s[(9 + v) * ADJ_NT];
                Fb.v[v] = A.dtdx * (s[(18 + v) * ADJ_NT] - S[(size_t)(81 + 9 * buf + v) * ADJ_NT]);
            }
            compiler_fence();
            riemann_issue(A, I, S, c + stride, xn, yn, zn, d, buf ^ 1);   // refill the slots just read
            adj_riemann_face<RIEM, DUALS>(A, I.n, c, face_nbr(I, x, y, z, d), d, L, Rr, Fb, ul);
        }
        x = xn;
        y = yn;
        z = zn;
    }
    cp_async_wait_all();
}

template <class R> struct StencilStaged {
    const R* S;
    __device__ Q9<R> operator()(int j) const {
        Q9<R> q;
#pragma unroll
        for (int v = 0; v < 9; ++v) q.v[v] = S[(size_t)(9 * j + v) * ADJ_NT];
        return q;
    }
};
template <class R>
__device__ __forceinline__ void recon_issue_u(const AdjArgs<R>& A, const Idx<R>& I, R* S, size_t c) {
    if (c < I.n) {
        int x, y, z;
        cell_xyz(A, c, x, y, z);
        size_t cs[7];
        stencil7(I, x, y, z, cs);
#pragma unroll
        for (int j = 0; j < 7; ++j)
#pragma unroll
            for (int v = 0; v < 9; ++v) cp_async_r(S + (size_t)(9 * j + v) * ADJ_NT, A.u.p[v] + cs[j]);
    }
    cp_async_commit();
}
template <class R>
__device__ __forceinline__ void recon_issue_f(const AdjArgs<R>& A, const Idx<R>& I, R* S, size_t c) {
    if (c < I.n) {
#pragma unroll
        for (int k = 0; k < 54; ++k) cp_async_r(S + (size_t)(63 + k) * ADJ_NT, A.FSb + (size_t)k * I.n + c);
    }
    cp_async_commit();
}
// FSbar of the current cell from the slots; release() refills them with the next cell's
template <class R> struct FaceBarStaged {
    const AdjArgs<R>* A;
    const Idx<R>* I;
    R* S;
    size_t cnext;
    __device__ Q9<R> operator()(int k) const {
        Q9<R> q;
#pragma unroll
        for (int v = 0; v < 9; ++v) q.v[v] = S[(size_t)(63 + 9 * k + v) * ADJ_NT];
        return q;
    }
    __device__ void release() const {
        compiler_fence();
        recon_issue_f(*A, *I, S, cnext);
    }
};

template <class R> __global__ void __launch_bounds__(ADJ_NT, 3) adj_recon_staged_kernel(const AdjArgs<R> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* S = reinterpret_cast<R*>(smem_raw) + threadIdx.x;
    const Idx<R> I = idx_of(A);
    const size_t stride = (size_t)gridDim.x * ADJ_NT;
    const bool mm = A.recon == RECON_MINMOD;
    size_t c = (size_t)blockIdx.x * ADJ_NT + threadIdx.x;
    recon_issue_u(A, I, S, c);
    recon_issue_f(A, I, S, c);
    for (; c < I.n; c += stride) {
        cp_async_wait_group<1>();   // the stencil of cell c has landed
        CellRec<R> r;
        cell_rec_from(StencilStaged<R>{S}, A.K, A.dtdx, mm, r);
        compiler_fence();
        recon_issue_u(A, I, S, c + stride);
        cp_async_wait_group<1>();   // FSbar of cell c has landed
        adj_recon_core(A, I.n, c, r, FaceBarStaged<R>{&A, &I, S, c + stride});
    }
    cp_async_wait_all();
}

template <class K> static cudaError_t adj_smem_attr(K kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// FP32: passes 4 and 5 staged through shared memory (the FP64 passes keep the plain kernels)
template <int RIEM, bool DUALS, class R> static void launch_riemann_pass(const AdjArgs<R>& A, int nb, cudaStream_t s) {
    if constexpr (std::is_same<R, float>::value) {
        const size_t sm = (size_t)RS_SLOTS * ADJ_NT * sizeof(R);
        adj_smem_attr(adj_riemann_staged_kernel<RIEM, DUALS, R>, sm);
        adj_riemann_staged_kernel<RIEM, DUALS, R><<<nb, ADJ_NT, sm, s>>>(A);
    } else {
        adj_riemann_kernel<RIEM, DUALS, R><<<nb, 128, 0, s>>>(A);
    }
}
template <class R> static void launch_recon_pass(const AdjArgs<R>& A, int nb, cudaStream_t s) {
    if constexpr (std::is_same<R, float>::value) {
        const size_t sm = (size_t)RC_SLOTS * ADJ_NT * sizeof(R);
        adj_smem_attr(adj_recon_staged_kernel<R>, sm);
        adj_recon_staged_kernel<R><<<nb, ADJ_NT, sm, s>>>(A);
    } else {
        adj_recon_kernel<R><<<nb, 128, 0, s>>>(A);
    }
}

// ---- passes 1-3 as one tile march (record mode) -------------------------------------------------
// The forward step's own tile kernel with a scheme that, instead of writing the new state, stores
// every cell's six interface states (what pass 1 computes) and the adjoint of the update epilogue at
// the pre-epilogue state (pass 3), which it forms from the fluxes it has just solved (pass 2's
// product, which therefore never goes through memory).  The interface states are the forward
// step's own, in its evaluation order.
template <class R, int RECON, int RIEM> struct AdjRecordScheme : UnsplitScheme<R, RECON, RIEM> {
    static constexpr bool kRecord = true;
    static __device__ __forceinline__ void epilogue_adj(const Q9<R>& r1, const Consts<R>& K, R glm_fac, bool turb, R ax,
                                                        R ay, R az, R dt, const Q9<R>& ob, Q9<R>& rb, R ab[3]) {
        finish_update_adj(r1, K, glm_fac, turb, ax, ay, az, dt, ob, rb, ab);
    }
};
template <class R, int RECON, int RIEM, int MAXT, int MINB, int TOX, int TOY>
__global__ void __launch_bounds__(MAXT, MINB) adj_record_kernel(const __grid_constant__ UnsplitArgs<R> A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    scheme_tile<R, AdjRecordScheme<R, RECON, RIEM>, TOX, TOY, false, true>(A, step_vals(A), blockIdx.x, blockIdx.y,
                                                                            blockIdx.z, smem_raw);
}
template <class R, int RECON, int RIEM, int MAXT, int MINB, int TOX, int TOY>
static cudaError_t record_go(const UnsplitArgs<R>& A, cudaStream_t s) {
    auto k = adj_record_kernel<R, RECON, RIEM, MAXT, MINB, TOX, TOY>;
    static int configured[64] = {0};
    {
        cudaError_t e = configure_once(k, configured);
        if (e != cudaSuccess) return e;
    }
    const int nt = A.ox * A.oy;
    if (nt > MAXT || nt < 1) return cudaErrorInvalidConfiguration;
    dim3 grid(A.nx / A.ox, A.ny / A.oy, (A.nz + A.lz - 1) / A.lz);
    k<<<grid, nt, unsplit_smem_bytes<R>(A.ox, A.oy), s>>>(A);
    return cudaGetLastError();
}
template <class R, int RECON, int RIEM> static cudaError_t record_tile(const UnsplitArgs<R>& A, cudaStream_t s) {
    if (A.ox == 32 && A.oy == 16) return record_go<R, RECON, RIEM, 512, 1, 32, 16>(A, s);
    return record_go<R, RECON, RIEM, 512, 1, 0, 0>(A, s);
}
// passes 1-3 by the record tile, FP32, for PLM-MC / minmod with HLLD (also its LLF forms) or HLL;
// cudaErrorNotSupported otherwise (the caller then runs the per-cell passes).  In FP64 the three
// per-cell passes measured faster than the record tile (0.77 vs 0.95 ms for the whole adjoint step
// at 64^3): the FP64 tile holds 255 registers at 8 warps per SM.
template <class R> static cudaError_t launch_record(const UnsplitArgs<R>& A, int recon, int riem, cudaStream_t s) {
    if constexpr (std::is_same<R, float>::value) {
        if (recon == RECON_MC && riem == RIEM_HLLD) return record_tile<R, RECON_MC, RIEM_HLLD>(A, s);
        if (recon == RECON_MC && riem == RIEM_HLL) return record_tile<R, RECON_MC, RIEM_HLL>(A, s);
        if (recon == RECON_MINMOD && riem == RIEM_HLLD) return record_tile<R, RECON_MINMOD, RIEM_HLLD>(A, s);
        if (recon == RECON_MINMOD && riem == RIEM_HLL) return record_tile<R, RECON_MINMOD, RIEM_HLL>(A, s);
    }
    return cudaErrorNotSupported;
}

template <class R> cudaError_t launch_adjoint_t(const AdjArgs<R>& A, const UnsplitArgs<R>* rec, cudaStream_t s) {
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    const int nb = (int)std::min<size_t>((n + 127) / 128, 148 * 16);
    cudaError_t er = cudaErrorNotSupported;
    if (rec) er = launch_record(*rec, A.recon, A.riem, s);
    if (er == cudaErrorNotSupported) {
        adj_faces_kernel<R><<<nb, 128, 0, s>>>(A);
        if (A.riem == RIEM_HLL) adj_flux_kernel<RIEM_HLL, R><<<nb, 128, 0, s>>>(A);
        else if (A.riem == RIEM_LLF_BOUND) adj_flux_kernel<RIEM_LLF_BOUND, R><<<nb, 128, 0, s>>>(A);
        else adj_flux_kernel<RIEM_HLLD, R><<<nb, 128, 0, s>>>(A);
        adj_update_kernel<R><<<nb, 128, 0, s>>>(A);
    } else if (er != cudaSuccess) {
        return er;
    }
    const bool llf_switch = A.use_llf || A.K.llf_dmin > R(0) || A.K.llf_pmin > R(0);
    if (A.riem == RIEM_HLL) launch_riemann_pass<RIEM_HLL, false>(A, nb, s);
    else if (A.riem == RIEM_LLF_BOUND) launch_riemann_pass<RIEM_LLF_BOUND, true>(A, nb, s);
    else if (llf_switch) launch_riemann_pass<RIEM_HLLD, true>(A, nb, s);
    else launch_riemann_pass<RIEM_HLLD, false>(A, nb, s);
    launch_recon_pass(A, nb, s);
    adj_gather_kernel<R><<<nb, 128, 0, s>>>(A);
    return cudaGetLastError();
}

// one unit instantiates it per real type (gmt_adjoint.cu: double, gmt_adjoint_f32.cu: float)
template <class R> cudaError_t launch_adjoint(const AdjArgs<R>& A, const UnsplitArgs<R>* rec, cudaStream_t s) {
    return launch_adjoint_t(A, rec, s);
}

}  // namespace gmt
