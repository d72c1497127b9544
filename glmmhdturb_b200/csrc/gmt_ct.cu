// gmt_ct.cu -- constrained-transport MHD step (CTMHD.step!, ct_mhd.jl:174; ct_run, spike_ctm.cu:305).
//
// State: 5 cell-centred conserved planes + 3 face planes, bxf[i,j,k] = Bx at (i-1/2, j, k).
// Cell primitives use the face-averaged field (ct_mhd.jl:85-97).  Per direction the lower-face
// flux comes from full-slope MonCen (or Julia-form PPM) on the stencil i-2..i+1, the
// transverse-free 1-D Hancock predictor, the face normal field and HLL or HLLD (no GLM).  Edge
// EMFs: Balsara-Spicer average of the four face EMFs (ct_mhd.jl:139-154) or the upwind
// contact-mode EMF of Gardiner & Stone (2005).  Face B advances by the curl of the edge EMFs, so
// the face divergence is preserved to round-off; the hydro update takes the same epilogue as the
// GLM step (void floor, forcing kick).
//
// Three passes through a 27-plane scratch buffer: face fluxes -> edge EMFs -> update.
#include "gmt_internal.h"

namespace gmt {

template <class R> struct CTIdx {
    int nx, ny, nz;
    size_t n;
    __device__ __forceinline__ size_t at(int x, int y, int z) const {
        return (size_t)wrapi(x, nx) + (size_t)nx * ((size_t)wrapi(y, ny) + (size_t)ny * wrapi(z, nz));
    }
};

// cell primitive with the face-averaged field (psi slot 0)
template <class R>
__device__ __forceinline__ Q9<R> ct_prim(const CPlanes8<R>& q, const CTIdx<R>& I, int x, int y, int z,
                                         const Consts<R>& K) {
    size_t c = I.at(x, y, z);
    Q9<R> cu;
#pragma unroll
    for (int v = 0; v < 5; ++v) cu.v[v] = q.p[v][c];
    cu.v[5] = R(0.5) * (q.p[5][c] + q.p[5][I.at(x + 1, y, z)]);
    cu.v[6] = R(0.5) * (q.p[6][c] + q.p[6][I.at(x, y + 1, z)]);
    cu.v[7] = R(0.5) * (q.p[7][c] + q.p[7][I.at(x, y, z + 1)]);
    cu.v[8] = R(0);
    return cons2prim(cu, K.gamma, K.smallr, K.smallp);
}

template <int D, class R>
__device__ __forceinline__ Q9<R> ct_face_flux(const Q9<R>& m2, const Q9<R>& m1, const Q9<R>& c0, const Q9<R>& p1, R bn,
                                              const CTArgs<R>& A) {
    const Consts<R>& K = A.K;
    Q9<R> sL = full_slope(m2, m1, c0), sR = full_slope(m1, c0, p1);
    if (A.halfslope) {
#pragma unroll
        for (int v = 0; v < 9; ++v) { sL.v[v] = R(0.5) * sL.v[v]; sR.v[v] = R(0.5) * sR.v[v]; }
    }
    Q9<R> mhL = hanc1d<D>(m1, sL, A.dtdx, K.gamma, K.smallr, K.smallp);
    Q9<R> mhR = hanc1d<D>(c0, sR, A.dtdx, K.gamma, K.smallr, K.smallp);
    Q9<R> L, Rr;
    if (A.recon == RECON_PPM) {
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
    L.v[5 + D] = bn; Rr.v[5 + D] = bn;
    L.v[8] = R(0); Rr.v[8] = R(0);
    Q9<R> Lr = rot_to<D>(L), Rrr = rot_to<D>(Rr);
    Q9<R> f = A.riem == RIEM_HLLD ? hlld_x(Lr, Rrr, K.gamma, bn, R(0), R(0)) : hll_x(Lr, Rrr, K.gamma, bn, R(0), R(0));
    return rot_from<D>(f);
}

template <int D, class R>
__device__ __forceinline__ void ct_flux_dir(const CTArgs<R>& A, const CTIdx<R>& I, int x, int y, int z, size_t c) {
    auto P = [&](int s) {
        return ct_prim(A.q, I, x + (D == 0 ? s : 0), y + (D == 1 ? s : 0), z + (D == 2 ? s : 0), A.K);
    };
    Q9<R> m2 = P(-2), m1 = P(-1), c0 = P(0), p1 = P(1);
    Q9<R> f = ct_face_flux<D>(m2, m1, c0, p1, A.q.p[5 + D][c], A);
    R* F = A.scratch + (size_t)D * 8 * I.n;
#pragma unroll
    for (int v = 0; v < 8; ++v) F[(size_t)v * I.n + c] = f.v[v];
}

template <class R> __global__ void __launch_bounds__(128) ct_flux_kernel(const CTArgs<R> A) {
    CTIdx<R> I{A.nx, A.ny, A.nz, (size_t)A.nx * A.ny * A.nz};
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < I.n; c += (size_t)gridDim.x * blockDim.x) {
        int x = (int)(c % A.nx), y = (int)((c / A.nx) % A.ny), z = (int)(c / ((size_t)A.nx * A.ny));
        ct_flux_dir<0>(A, I, x, y, z, c);
        ct_flux_dir<1>(A, I, x, y, z, c);
        ct_flux_dir<2>(A, I, x, y, z, c);
    }
}

template <class R>
__device__ __forceinline__ R ct_ecc(const CTArgs<R>& A, const CTIdx<R>& I, size_t c, int x, int y, int z, int e) {
    Q9<R> q = ct_prim(A.q, I, x, y, z, A.K);
    R v;
    if (e == 0) v = q.v[2] * q.v[7] - q.v[3] * q.v[6];
    else if (e == 1) v = q.v[3] * q.v[5] - q.v[1] * q.v[7];
    else v = q.v[1] * q.v[6] - q.v[2] * q.v[5];
    (void)c;
    return -v;
}

template <class R> __device__ __forceinline__ R upwind(R flux, R minus, R plus) {
    return flux > R(0) ? minus : (flux < R(0) ? plus : R(0.5) * (minus + plus));
}

// edge EMFs; same corner formula and order as the oracle (cyclic axes (A,B,e))
template <class R> __global__ void __launch_bounds__(128) ct_emf_kernel(const CTArgs<R> A) {
    CTIdx<R> I{A.nx, A.ny, A.nz, (size_t)A.nx * A.ny * A.nz};
    const R* F = A.scratch;
    R* E = A.scratch + (size_t)24 * I.n;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < I.n; c += (size_t)gridDim.x * blockDim.x) {
        int x = (int)(c % A.nx), y = (int)((c / A.nx) % A.ny), z = (int)(c / ((size_t)A.nx * A.ny));
        for (int e = 0; e < 3; ++e) {
            const int Ax = (e + 1) % 3, Bx = (e + 2) % 3;
            int ia[3] = {0, 0, 0}, ib[3] = {0, 0, 0};
            ia[Ax] = 1; ib[Bx] = 1;
            auto atc = [&](int sa, int sb, int& xx, int& yy, int& zz) {
                xx = x - sa * ia[0] - sb * ib[0];
                yy = y - sa * ia[1] - sb * ib[1];
                zz = z - sa * ia[2] - sb * ib[2];
                return I.at(xx, yy, zz);
            };
            int x10, y10, z10, x01, y01, z01, x11, y11, z11, x00, y00, z00;
            size_t c00 = atc(0, 0, x00, y00, z00), c10 = atc(1, 0, x10, y10, z10);
            size_t c01 = atc(0, 1, x01, y01, z01), c11 = atc(1, 1, x11, y11, z11);
            const R* FA = F + (size_t)Ax * 8 * I.n;
            const R* FB = F + (size_t)Bx * 8 * I.n;
            R EaN = -FA[(size_t)(5 + Bx) * I.n + c00];
            R EaS = -FA[(size_t)(5 + Bx) * I.n + c01];
            R EbE = FB[(size_t)(5 + Ax) * I.n + c00];
            R EbW = FB[(size_t)(5 + Ax) * I.n + c10];
            R Ev = R(0.25) * (EbE + EbW + EaN + EaS);
            if (A.emf == 1) {
                R e00 = ct_ecc(A, I, c00, x00, y00, z00, e), e10 = ct_ecc(A, I, c10, x10, y10, z10, e);
                R e01 = ct_ecc(A, I, c01, x01, y01, z01, e), e11 = ct_ecc(A, I, c11, x11, y11, z11, e);
                R dN = upwind(FA[c00], e10 - EbW, e00 - EbE);
                R dS = upwind(FA[c01], EbW - e11, EbE - e01);
                R dE = upwind(FB[c00], e01 - EaS, e00 - EaN);
                R dW = upwind(FB[c10], EaS - e11, EaN - e10);
                Ev = Ev + R(0.25) * (dS - dN) + R(0.25) * (dW - dE);
            }
            E[(size_t)e * I.n + c00] = Ev;
        }
    }
}

template <class R> __global__ void __launch_bounds__(128) ct_update_kernel(const CTArgs<R> A) {
    CTIdx<R> I{A.nx, A.ny, A.nz, (size_t)A.nx * A.ny * A.nz};
    const R* F = A.scratch;
    const R* E = A.scratch + (size_t)24 * I.n;
    const R* ex = E;
    const R* ey = E + I.n;
    const R* ez = E + 2 * I.n;
    const bool turb = A.do_turb && A.btab != nullptr;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < I.n; c += (size_t)gridDim.x * blockDim.x) {
        int x = (int)(c % A.nx), y = (int)((c / A.nx) % A.ny), z = (int)(c / ((size_t)A.nx * A.ny));
        size_t cxp = I.at(x + 1, y, z), cyp = I.at(x, y + 1, z), czp = I.at(x, y, z + 1);
        const R dtdx = A.dtdx;
        A.o.p[5][c] = A.q.p[5][c] - dtdx * ((ez[cyp] - ez[c]) - (ey[czp] - ey[c]));
        A.o.p[6][c] = A.q.p[6][c] - dtdx * ((ex[czp] - ex[c]) - (ez[cxp] - ez[c]));
        A.o.p[7][c] = A.q.p[7][c] - dtdx * ((ey[cxp] - ey[c]) - (ex[cyp] - ex[c]));
        Q9<R> r;
#pragma unroll
        for (int v = 0; v < 5; ++v)
            r.v[v] = A.q.p[v][c] + dtdx * ((F[(size_t)v * I.n + c] - F[(size_t)v * I.n + cxp]) +
                                           (F[(size_t)(8 + v) * I.n + c] - F[(size_t)(8 + v) * I.n + cyp]) +
                                           (F[(size_t)(16 + v) * I.n + c] - F[(size_t)(16 + v) * I.n + czp]));
        Q9<R> pc = ct_prim(A.q, I, x, y, z, A.K);
        r.v[5] = pc.v[5]; r.v[6] = pc.v[6]; r.v[7] = pc.v[7]; r.v[8] = R(0);
        R ax = R(0), ay = R(0), az = R(0);
        if (turb) force_accel(A.btab + ((size_t)z * A.ny + y) * 24, A.trigx, A.nx, x, A.ramp, ax, ay, az);
        finish_update(r, A.K, R(1), turb, ax, ay, az, A.dt);
#pragma unroll
        for (int v = 0; v < 5; ++v) A.o.p[v][c] = r.v[v];
    }
}

template <class R> static cudaError_t go(const CTArgs<R>& A, cudaStream_t s) {
    size_t n = (size_t)A.nx * A.ny * A.nz;
    int nb = (int)std::min<size_t>((n + 127) / 128, (size_t)148 * 64);
    ct_flux_kernel<R><<<nb, 128, 0, s>>>(A);
    ct_emf_kernel<R><<<nb, 128, 0, s>>>(A);
    ct_update_kernel<R><<<nb, 128, 0, s>>>(A);
    return cudaGetLastError();
}
cudaError_t launch_ct(const CTArgs<float>& A, cudaStream_t s) { return go(A, s); }
cudaError_t launch_ct(const CTArgs<double>& A, cudaStream_t s) { return go(A, s); }
int ct_regs_of(int dtype_bytes) {
    cudaFuncAttributes fa{};
    cudaError_t e = dtype_bytes == 8 ? cudaFuncGetAttributes(&fa, ct_flux_kernel<double>)
                                     : cudaFuncGetAttributes(&fa, ct_flux_kernel<float>);
    return e == cudaSuccess ? fa.numRegs : -1;
}
size_t ct_smem_of(int, int, int) { return 0; }

}  // namespace gmt
