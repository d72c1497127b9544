// gmt_march1d.cu -- transverse-free 1-D Hancock + HLL + Dedner step behind march_run_dev.
//
// Scheme of march_bridge/cu/spike_mhd.cu:227-302: per direction, full-slope MonCen on the
// primitive stencil i-2..i+2, a 1-D Hancock half step of cells i-1, i, i+1, face states
// mh +- s/2 (or Julia-form PPM edges + predictor shift, glmmhd_turb.jl:917-926), HLL with GLM
// cleaning, then u -= dt/dx * sum_d (F_hi - F_lo) and psi *= glmfac.  The update base is the
// state read from HBM (the spike adds the increment to a 16-bit tile copy instead).
//
// Passive species (spike_mhd.cu:55-61, 128-139, 155-158, 218-221, 241-244, 278-296): planes hold
// rho*X; the fraction X = rho*X / max(rho, smallr) gets the same full MonCen slope, the predictor
// X - dt/(2dx) u_n dX and the faces X_h +- s/2 (or the PPM edge + predictor shift), and rides the
// face mass flux: F_X = F_rho X_L if F_rho >= 0, else F_rho X_R (consistent multi-fluid advection).
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

// species flux at the face between cells m1 and c0 (stencil m2, m1 | c0, p1 along the direction)
template <class R>
__device__ __forceinline__ R species_face(R xm2, R xm1, R xc0, R xp1, R un_m1, R un_c0, R h, R frho, bool ppm) {
    R sL = full_mc(xm2, xm1, xc0), sR = full_mc(xm1, xc0, xp1);
    R mhL = xm1 - h * un_m1 * sL;
    R mhR = xc0 - h * un_c0 * sR;
    R L, Rr;
    if (ppm) {
        R lo, hi;
        ppm_edges(xm2, xm1, xc0, lo, hi);
        L = hi + mhL - xm1;
        ppm_edges(xm1, xc0, xp1, lo, hi);
        Rr = lo + mhR - xc0;
    } else {
        L = mhL + R(0.5) * sL;
        Rr = mhR + R(-0.5) * sR;
    }
    return frho >= R(0) ? frho * L : frho * Rr;
}

template <class R>
__device__ __forceinline__ Q9<R> prim_at(const CPlanes<R>& u, size_t g, const Consts<R>& K) {
    Q9<R> c;
#pragma unroll
    for (int v = 0; v < 9; ++v) c.v[v] = u.p[v][g];
    return cons2prim(c, K.gamma, K.smallr, K.smallp);
}

template <int D, class R>
__device__ __forceinline__ void march_dir(const MarchArgs<R>& A, int x, int y, int z, Q9<R>& div, R* divs) {
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
    if (A.nsp > 0) {
        const size_t g[5] = {at(-2), at(-1), at(0), at(1), at(2)};
        const R rho[5] = {cm2.v[0], cm1.v[0], c0.v[0], cp1.v[0], cp2.v[0]};
        const R h = R(0.5) * A.dtdx;
#pragma unroll
        for (int s = 0; s < MAX_SPECIES; ++s) {
            if (s < A.nsp) {
                R X[5];
#pragma unroll
                for (int k = 0; k < 5; ++k) X[k] = A.su[s][g[k]] / rho[k];
                R fm = species_face(X[0], X[1], X[2], X[3], cm1.v[1 + D], c0.v[1 + D], h, Fm.v[0], A.ppm != 0);
                R fp = species_face(X[1], X[2], X[3], X[4], c0.v[1 + D], cp1.v[1 + D], h, Fp.v[0], A.ppm != 0);
                divs[s] = divs[s] + (fp - fm);
            }
        }
    }
}

template <class R>
__global__ void __launch_bounds__(128) march1d_kernel(const MarchArgs<R> A) {
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
        int x = (int)(g % A.nx), y = (int)((g / A.nx) % A.ny), z = (int)(g / ((size_t)A.nx * A.ny));
        Q9<R> div;
        R divs[MAX_SPECIES];
#pragma unroll
        for (int v = 0; v < 9; ++v) div.v[v] = R(0);
#pragma unroll
        for (int s = 0; s < MAX_SPECIES; ++s) divs[s] = R(0);
        march_dir<0>(A, x, y, z, div, divs);
        march_dir<1>(A, x, y, z, div, divs);
        march_dir<2>(A, x, y, z, div, divs);
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            R u = A.u.p[v][g] - A.dtdx * div.v[v];
            if (v == 8) u = u * A.glm_fac;
            A.o.p[v][g] = u;
        }
#pragma unroll
        for (int s = 0; s < MAX_SPECIES; ++s)
            if (s < A.nsp) A.so[s][g] = A.su[s][g] - A.dtdx * divs[s];
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
