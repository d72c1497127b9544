// gmt_species.cuh -- passive species of the march scheme behind march_run_dev.
//
// The MHD part of the march step (spike_mhd.cu:227-302: per direction full-slope MonCen, a 1-D
// Hancock half step of each cell, HLL with GLM cleaning) runs in the tile march (MarchScheme,
// gmt_unsplit.cuh), which also stores every cell's lower-face mass fluxes when species are present.
//
// Passive species (spike_mhd.cu:55-61, 128-139, 155-158, 218-221, 241-244, 278-296): planes hold
// rho*X; the fraction X = rho*X / max(rho, smallr) gets the same full MonCen slope, the predictor
// X - dt/(2dx) u_n dX and the faces X_h +- s/2 (or the PPM edge + predictor shift), and rides the
// face mass flux: F_X = F_rho X_L if F_rho >= 0, else F_rho X_R (consistent multi-fluid advection).
#pragma once
#include <algorithm>

#include "gmt_internal.h"

namespace gmt {

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

// Passive species of one cell (one thread per cell), after the tiled march step: per direction
// the species flux at the cell's lower and upper faces from the stencil i-2..i+2, the normal
// velocities of the cells beside each face and the face mass flux the step stored.
template <class R>
__global__ void __launch_bounds__(128) species_kernel(const MarchArgs<R> A, const R* __restrict__ fmass) {
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    const R h = R(0.5) * A.dtdx;
    const size_t sxy = (size_t)A.nx * A.ny;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
        int x, y, z;
        if (n <= 0xffffffffu) {   // 32-bit divisions for every linear index below 2^32
            const unsigned gg = (unsigned)g, q = gg / (unsigned)A.nx;
            x = (int)(gg - q * (unsigned)A.nx);
            y = (int)(q % (unsigned)A.ny);
            z = (int)(q / (unsigned)A.ny);
        } else {
            x = (int)(g % A.nx); y = (int)((g / A.nx) % A.ny); z = (int)(g / sxy);
        }
        R divs[MAX_SPECIES];
#pragma unroll
        for (int s = 0; s < MAX_SPECIES; ++s) divs[s] = R(0);
#pragma unroll
        for (int D = 0; D < 3; ++D) {
            // the stencil g + (i - c) * stride along D, i the periodic image of c + k - 2
            const int c = D == 0 ? x : (D == 1 ? y : z), m = D == 0 ? A.nx : (D == 1 ? A.ny : A.nz);
            const size_t st = D == 0 ? 1 : (D == 1 ? (size_t)A.nx : sxy);
            size_t at[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                int i = c + k - 2;
                i = i < 0 ? i + m : (i >= m ? i - m : i);
                i = i < 0 ? i + m : (i >= m ? i - m : i);   // boxes narrower than the stencil
                at[k] = g + (size_t)((long long)(i - c) * (long long)st);
            }
            R rho[5], un[3];
#pragma unroll
            for (int k = 0; k < 5; ++k) rho[k] = rmax(A.u.p[0][at[k]], A.K.smallr);
#pragma unroll
            for (int k = 0; k < 3; ++k) un[k] = A.u.p[1 + D][at[k + 1]] * (R(1) / rho[k + 1]);
            const R Fm = fmass[(size_t)D * n + g], Fp = fmass[(size_t)D * n + at[3]];
#pragma unroll
            for (int s = 0; s < MAX_SPECIES; ++s) {
                if (s < A.nsp) {
                    R X[5];
#pragma unroll
                    for (int k = 0; k < 5; ++k) X[k] = A.su[s][at[k]] / rho[k];
                    const R fm = species_face(X[0], X[1], X[2], X[3], un[0], un[1], h, Fm, A.ppm != 0);
                    const R fp = species_face(X[1], X[2], X[3], X[4], un[1], un[2], h, Fp, A.ppm != 0);
                    divs[s] = divs[s] + (fp - fm);
                }
            }
        }
#pragma unroll
        for (int s = 0; s < MAX_SPECIES; ++s)
            if (s < A.nsp) A.so[s][g] = A.su[s][g] - A.dtdx * divs[s];
    }
}

// FP32 species pass, four cells x0..x0+3 (x0 = 4k) per thread: every plane is read as 16-byte
// quads (the x stencil from the quads at x0-4, x0, x0+4 of the row, periodic), the five x faces
// x0-1/2 .. x0+7/2 are each solved once, and the result is stored as one quad per species.  Same
// per-face and per-cell arithmetic as species_kernel.  Requires nx % 4 == 0, nx >= 8 and 16-byte
// aligned planes.
__device__ __forceinline__ float sq4(const float4& v, int j) { return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w)); }

template <int NSP> __global__ void __launch_bounds__(128) species_kernel4(const MarchArgs<float> A, const float* __restrict__ fmass) {
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const size_t n = (size_t)nx * ny * nz, nq = n / 4;
    const float h = 0.5f * A.dtdx;
    const bool ppm = A.ppm != 0;
    auto ld = [](const float* p, size_t i) { return __ldg(reinterpret_cast<const float4*>(p + i)); };
    auto wrap2 = [](int i, int m) {   // as species_kernel: boxes narrower than the stencil wrap twice
        i = i < 0 ? i + m : (i >= m ? i - m : i);
        return i < 0 ? i + m : (i >= m ? i - m : i);
    };
    for (size_t qd = (size_t)blockIdx.x * blockDim.x + threadIdx.x; qd < nq; qd += (size_t)gridDim.x * blockDim.x) {
        const size_t c = 4 * qd;
        int x, y, z;
        cell_coords(c, nx, ny, n, x, y, z);
        float divs[NSP][4];
#pragma unroll
        for (int sp = 0; sp < NSP; ++sp)
#pragma unroll
            for (int j = 0; j < 4; ++j) divs[sp][j] = 0.0f;
        // ---- x: the 8 cells x0-2 .. x0+5 from three quads
        {
            const size_t cm = x == 0 ? c + nx - 4 : c - 4, cp = x + 4 == nx ? c + 4 - nx : c + 4;
            float rho[8], un[6];
            {
                const float4 a = ld(A.u.p[0], cm), b = ld(A.u.p[0], c), d = ld(A.u.p[0], cp);
                const float r[8] = {a.z, a.w, b.x, b.y, b.z, b.w, d.x, d.y};
#pragma unroll
                for (int k = 0; k < 8; ++k) rho[k] = rmax(r[k], A.K.smallr);
            }
            {
                const float4 a = ld(A.u.p[1], cm), b = ld(A.u.p[1], c), d = ld(A.u.p[1], cp);
                const float m[6] = {a.w, b.x, b.y, b.z, b.w, d.x};   // cells x0-1 .. x0+4
#pragma unroll
                for (int k = 0; k < 6; ++k) un[k] = m[k] * (1.0f / rho[k + 1]);
            }
            const float4 f0 = ld(fmass, c), f1 = ld(fmass, cp);
            const float F[5] = {f0.x, f0.y, f0.z, f0.w, f1.x};   // faces x0-1/2 .. x0+7/2
#pragma unroll
            for (int sp = 0; sp < NSP; ++sp) {
                {
                    const float4 a = ld(A.su[sp], cm), b = ld(A.su[sp], c), d = ld(A.su[sp], cp);
                    const float v[8] = {a.z, a.w, b.x, b.y, b.z, b.w, d.x, d.y};
                    float X[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) X[k] = v[k] / rho[k];
                    float f[5];
#pragma unroll
                    for (int k = 0; k < 5; ++k)   // face x0+k-1/2: cells x0+k-2 .. x0+k+1 = X[k..k+3]
                        f[k] = species_face(X[k], X[k + 1], X[k + 2], X[k + 3], un[k], un[k + 1], h, F[k], ppm);
#pragma unroll
                    for (int j = 0; j < 4; ++j) divs[sp][j] = divs[sp][j] + (f[j + 1] - f[j]);
                }
            }
        }
        // ---- y and z: five rows (planes) of quads
#pragma unroll
        for (int D = 1; D < 3; ++D) {
            const int cc = D == 1 ? y : z, m = D == 1 ? ny : nz;
            const size_t st = D == 1 ? (size_t)nx : (size_t)nx * ny;
            size_t at[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) at[k] = c + (size_t)((long long)(wrap2(cc + k - 2, m) - cc) * (long long)st);
            float4 rho[5], un[3];
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                const float4 r = ld(A.u.p[0], at[k]);
                rho[k] = make_float4(rmax(r.x, A.K.smallr), rmax(r.y, A.K.smallr), rmax(r.z, A.K.smallr), rmax(r.w, A.K.smallr));
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float4 u = ld(A.u.p[1 + D], at[k + 1]);
                un[k] = make_float4(u.x * (1.0f / rho[k + 1].x), u.y * (1.0f / rho[k + 1].y), u.z * (1.0f / rho[k + 1].z),
                                    u.w * (1.0f / rho[k + 1].w));
            }
            const float4 Fm = ld(fmass + (size_t)D * n, c), Fp = ld(fmass + (size_t)D * n, at[3]);
#pragma unroll
            for (int sp = 0; sp < NSP; ++sp) {
                {
                    float4 X[5];
#pragma unroll
                    for (int k = 0; k < 5; ++k) {
                        const float4 v = ld(A.su[sp], at[k]);
                        X[k] = make_float4(v.x / rho[k].x, v.y / rho[k].y, v.z / rho[k].z, v.w / rho[k].w);
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float fm = species_face(sq4(X[0], j), sq4(X[1], j), sq4(X[2], j), sq4(X[3], j), sq4(un[0], j),
                                                      sq4(un[1], j), h, sq4(Fm, j), ppm);
                        const float fp = species_face(sq4(X[1], j), sq4(X[2], j), sq4(X[3], j), sq4(X[4], j), sq4(un[1], j),
                                                      sq4(un[2], j), h, sq4(Fp, j), ppm);
                        divs[sp][j] = divs[sp][j] + (fp - fm);
                    }
                }
            }
        }
#pragma unroll
        for (int sp = 0; sp < NSP; ++sp) {
            {
                const float4 u0 = ld(A.su[sp], c);
                *reinterpret_cast<float4*>(A.so[sp] + c) =
                    make_float4(u0.x - A.dtdx * divs[sp][0], u0.y - A.dtdx * divs[sp][1], u0.z - A.dtdx * divs[sp][2],
                                u0.w - A.dtdx * divs[sp][3]);
            }
        }
    }
}

// the 4-wide pass applies: FP32, nx a multiple of 4 and at least 8, every plane 16-byte aligned
inline bool species_quad_ok(const MarchArgs<float>& A, const float* fmass) {
    if (A.nx % 4 != 0 || A.nx < 8) return false;
    auto al = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
    if (!al(fmass) || !al(A.u.p[0]) || !al(A.u.p[1]) || !al(A.u.p[2]) || !al(A.u.p[3])) return false;
    for (int sp = 0; sp < A.nsp; ++sp)
        if (!al(A.su[sp]) || !al(A.so[sp])) return false;
    return true;
}

template <class R> static cudaError_t species_go(const MarchArgs<R>& A, const R* fmass, cudaStream_t s) {
    size_t n = (size_t)A.nx * A.ny * A.nz;
    if constexpr (std::is_same<R, float>::value) {
        if (species_quad_ok(A, fmass)) {
            const int nb4 = (int)std::min<size_t>((n / 4 + 127) / 128, (size_t)148 * 64);
            switch (A.nsp) {   // the species count is a template parameter (registers per species)
                case 1: species_kernel4<1><<<nb4, 128, 0, s>>>(A, fmass); break;
                case 2: species_kernel4<2><<<nb4, 128, 0, s>>>(A, fmass); break;
                case 3: species_kernel4<3><<<nb4, 128, 0, s>>>(A, fmass); break;
                case 4: species_kernel4<4><<<nb4, 128, 0, s>>>(A, fmass); break;
                default: species_kernel<R><<<(int)std::min<size_t>((n + 127) / 128, (size_t)148 * 64), 128, 0, s>>>(A, fmass);
            }
            return cudaGetLastError();
        }
    }
    int nb = (int)std::min<size_t>((n + 127) / 128, (size_t)148 * 64);
    species_kernel<R><<<nb, 128, 0, s>>>(A, fmass);
    return cudaGetLastError();
}

}  // namespace gmt
