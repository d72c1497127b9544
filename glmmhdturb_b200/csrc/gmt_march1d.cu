// gmt_march1d.cu -- transverse-free 1-D Hancock + HLL + Dedner step behind march_run_dev.
//
// Scheme of march_bridge/cu/spike_mhd.cu:227-302: per direction, full-slope MonCen on the
// primitive stencil i-2..i+2, a 1-D Hancock half step of cells i-1, i, i+1, face states
// mh +- s/2 (or Julia-form PPM edges + predictor shift, glmmhd_turb.jl:917-926), HLL with GLM
// cleaning, then u -= dt/dx * sum_d (F_hi - F_lo) and psi *= glmfac.  The update base is the
// state read from HBM (the spike adds the increment to a 16-bit tile copy instead).
#include "gmt_internal.h"

namespace gmt {

template <int D, class R>
__device__ __forceinline__ Q9<R> march_face(const Q9<R>& m2, const Q9<R>& m1, const Q9<R>& c0, const Q9<R>& p1,
                                            const Consts<R>& K, R dtdx, R ch, bool ppm) {
    Q9<R> sL = full_slope(m2, m1, c0), sR = full_slope(m1, c0, p1);
    Q9<R> mhL = hanc1d<D>(m1, sL, dtdx, K.gamma, K.smallr, K.smallp);
    Q9<R> mhR = hanc1d<D>(c0, sR, dtdx, K.gamma, K.smallr, K.smallp);
    Q9<R> L, Rr;
    if (ppm) {
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            R lo, hi;
            ppm_edges(m2.v[v], m1.v[v], c0.v[v], lo, hi);
            L.v[v] = hi + mhL.v[v] - m1.v[v];
            ppm_edges(m1.v[v], c0.v[v], p1.v[v], lo, hi);
            Rr.v[v] = lo + mhR.v[v] - c0.v[v];
        }
    } else {
        L = padd(mhL, sL, R(0.5));
        Rr = padd(mhR, sR, R(-0.5));
    }
    L.v[0] = rmax(L.v[0], K.smallr); L.v[4] = rmax(L.v[4], K.smallp);
    Rr.v[0] = rmax(Rr.v[0], K.smallr); Rr.v[4] = rmax(Rr.v[4], K.smallp);
    Q9<R> Lr = rot_to<D>(L), Rrr = rot_to<D>(Rr);
    R bns, psis;
    glm_pair(Lr.v[5], Rrr.v[5], Lr.v[8], Rrr.v[8], ch, bns, psis);
    Lr.v[5] = bns; Rrr.v[5] = bns;
    return rot_from<D>(hll_x(Lr, Rrr, K.gamma, bns, psis, ch * ch * bns));
}

template <class R>
__device__ __forceinline__ Q9<R> prim_at(const CPlanes<R>& u, size_t g, const Consts<R>& K) {
    Q9<R> c;
#pragma unroll
    for (int v = 0; v < 9; ++v) c.v[v] = u.p[v][g];
    return cons2prim(c, K.gamma, K.smallr, K.smallp);
}

template <int D, class R>
__device__ __forceinline__ void march_dir(const MarchArgs<R>& A, int x, int y, int z, Q9<R>& div) {
    auto at = [&](int s) {
        int xx = x + (D == 0 ? s : 0), yy = y + (D == 1 ? s : 0), zz = z + (D == 2 ? s : 0);
        return (size_t)wrapi(xx, A.nx) + (size_t)A.nx * ((size_t)wrapi(yy, A.ny) + (size_t)A.ny * wrapi(zz, A.nz));
    };
    Q9<R> cm2 = prim_at(A.u, at(-2), A.K), cm1 = prim_at(A.u, at(-1), A.K), c0 = prim_at(A.u, at(0), A.K);
    Q9<R> cp1 = prim_at(A.u, at(1), A.K), cp2 = prim_at(A.u, at(2), A.K);
    Q9<R> Fm = march_face<D>(cm2, cm1, c0, cp1, A.K, A.dtdx, A.ch, A.ppm != 0);
    Q9<R> Fp = march_face<D>(cm1, c0, cp1, cp2, A.K, A.dtdx, A.ch, A.ppm != 0);
#pragma unroll
    for (int v = 0; v < 9; ++v) div.v[v] = div.v[v] + (Fp.v[v] - Fm.v[v]);
}

template <class R>
__global__ void __launch_bounds__(128) march1d_kernel(const MarchArgs<R> A) {
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
        int x = (int)(g % A.nx), y = (int)((g / A.nx) % A.ny), z = (int)(g / ((size_t)A.nx * A.ny));
        Q9<R> div;
#pragma unroll
        for (int v = 0; v < 9; ++v) div.v[v] = R(0);
        march_dir<0>(A, x, y, z, div);
        march_dir<1>(A, x, y, z, div);
        march_dir<2>(A, x, y, z, div);
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            R u = A.u.p[v][g] - A.dtdx * div.v[v];
            if (v == 8) u = u * A.glm_fac;
            A.o.p[v][g] = u;
        }
    }
}

template <class R> static cudaError_t go(const MarchArgs<R>& A, cudaStream_t s) {
    size_t n = (size_t)A.nx * A.ny * A.nz;
    int nb = (int)std::min<size_t>((n + 127) / 128, (size_t)148 * 64);
    march1d_kernel<R><<<nb, 128, 0, s>>>(A);
    return cudaGetLastError();
}
cudaError_t launch_march1d(const MarchArgs<float>& A, cudaStream_t s) { return go(A, s); }
cudaError_t launch_march1d(const MarchArgs<double>& A, cudaStream_t s) { return go(A, s); }
int march1d_regs(int dtype_bytes) {
    cudaFuncAttributes fa{};
    cudaError_t e = dtype_bytes == 8 ? cudaFuncGetAttributes(&fa, march1d_kernel<double>)
                                     : cudaFuncGetAttributes(&fa, march1d_kernel<float>);
    return e == cudaSuccess ? fa.numRegs : -1;
}

}  // namespace gmt
