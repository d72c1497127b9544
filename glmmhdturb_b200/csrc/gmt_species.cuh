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

template <class R> static cudaError_t species_go(const MarchArgs<R>& A, const R* fmass, cudaStream_t s) {
    size_t n = (size_t)A.nx * A.ny * A.nz;
    int nb = (int)std::min<size_t>((n + 127) / 128, (size_t)148 * 64);
    species_kernel<R><<<nb, 128, 0, s>>>(A, fmass);
    return cudaGetLastError();
}

}  // namespace gmt
