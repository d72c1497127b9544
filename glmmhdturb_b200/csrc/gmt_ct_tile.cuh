// gmt_ct_tile.cuh -- constrained-transport step as a z-marching tile kernel plus two short
// per-cell passes (CTMHD.step!, ct_mhd.jl:174; the fused march of spike_ctm.cu:250-298).
//
// Pass A (ct_tile_kernel): a block owns an OX x OY column tile over LZ planes, exactly like the
// GLM step.  Shared memory holds (9-variable arrays in the Lay layout of the GLM tile march: FP32
// cells as two 16-byte vectors and a scalar)
//   PR[3][(OX+4)(OY+4)]     cell primitives with the face-averaged field (ring of 3 planes),
//   FB[3][3][(OX+4)(OY+4)]  the lower-face fields bxf, byf, bzf of the same cells,
//   ST[4][(OX+2)(OY+2)]     in-plane interface states, overwritten by the face fluxes,
//   SG[9][(OY+5)][OX+8]     staging of plane k+2: 5 conserved, bxf, byf, bzf(k+2), bzf(k+3)
//   TS[OX][8], BS[OY][24]   FP32: the forcing kick's x table of the tile's columns and row table
//                           of its rows for the plane written next
// (SG has one more row and column than the ring, for the face averages of the outermost cells, at
// column offset 2; tiles clear of the box edges fill it by two TMA copies, the others by
// cp.async).  The write-out's old cell state is loaded before the z-face solve.  Per
// direction each cell gets a full (or ct_mhd.jl's half) MonCen slope, the transverse-free 1-D
// Hancock predictor and its two face states, whose normal component is the face field; every
// face is solved once (HLL or HLLD, no GLM).  The write-out does the hydro update with the
// floor/kick epilogue (on the old cell-centred field) and stores, per cell, the EMF data of its
// three lower faces and its cell-centre EMF: 12 planes of scratch.
// Pass B1 (ct_edge_kernel): the edge EMFs -- Balsara-Spicer average (ct_mhd.jl:139-154) or the
// upwind contact EMF of Gardiner & Stone (2005) -- from that scratch, in the oracle's order.
// Pass B2 (ct_face_kernel): face B advances by the curl of the edge EMFs (ct_mhd.jl:156-172), so
// the face divergence is preserved to round-off.
#pragma once
#include "gmt_internal.h"
#include "gmt_unsplit_inst.cuh"
#include <algorithm>

namespace gmt {

// scratch plane indices (each n reals)
enum CTScratch {
    CS_EZX = 0,   // -F_x[By]  on the lower x face   (E_z on an x face)
    CS_EYX,       // +F_x[Bz]                        (E_y on an x face)
    CS_MX,        //  F_x[rho]
    CS_EXY,       // -F_y[Bz]  on the lower y face   (E_x on a y face)
    CS_EZY,       // +F_y[Bx]                        (E_z on a y face)
    CS_MY,        //  F_y[rho]
    CS_EYZ,       // -F_z[Bx]  on the lower z face   (E_y on a z face)
    CS_EXZ,       // +F_z[By]                        (E_x on a z face)
    CS_MZ,        //  F_z[rho]
    CS_ECX,       // cell-centre E = -(v x B)
    CS_ECY,
    CS_ECZ,
    CS_EDX,       // edge EMFs ex (i, j-1/2, k-1/2), ey (i-1/2, j, k-1/2), ez (i-1/2, j-1/2, k)
    CS_EDY,
    CS_EDZ,
    CS_PLANES
};

// byte offset of the reduction / mbarrier words: after the real arrays, rounded up to 16 bytes
// staging plane: 128-byte aligned (a TMA destination), after the rings and the states
template <class R> __host__ __device__ inline size_t ct_tile_sg_offset(int ox, int oy) {
    size_t PN = (size_t)lay_n<R>((ox + 4) * (oy + 4)), RN = (size_t)lay_n<R>((ox + 2) * (oy + 2));
    return ((27 * PN + 9 * PN + 36 * RN) * sizeof(R) + 127) / 128 * 128;
}
template <class R> __host__ __device__ inline size_t ct_tile_words_offset(int ox, int oy) {
    size_t SN5 = (size_t)(ox + 8) * (oy + 5);
    return (ct_tile_sg_offset<R>(ox, oy) + 9 * SN5 * sizeof(R) + 15) / 16 * 16;
}
template <class R> __host__ __device__ inline size_t ct_tile_smem_bytes(int ox, int oy) {
    return ct_tile_words_offset<R>(ox, oy) + 40 * sizeof(double) + (sizeof(R) == 4 ? 32 * (size_t)ox + 96 * (size_t)oy : 0);
}

// stage plane kp: the conserved cell variables, the three face fields at kp and bzf at kp+1, on
// the region x0-2..x0+OX+2, y0-2..y0+OY+2.  SG rows have the pitch SW = OX + 8 and the region
// starts at column 2: the layout of the TMA box (x0-4, y0-2) of (OX+8) x (OY+5) cells.
template <class R>
__device__ __forceinline__ void ct_stage_plane(R* __restrict__ SG, const CPlanes8<R>& q, int PN5, int PW5, int SW,
                                               int SN5, int x0, int y0, int kp, int nx, int ny, int nz, int tid,
                                               int nt) {
    const size_t gz = (size_t)wrapi(kp, nz), gz1 = (size_t)wrapi(kp + 1, nz);
    for (int c = tid; c < PN5; c += nt) {
        const int lx = c % PW5, ly = c / PW5;
        const size_t gxy = (size_t)wrapi(x0 - 2 + lx, nx) + (size_t)nx * wrapi(y0 - 2 + ly, ny);
        const size_t g = gxy + (size_t)nx * ny * gz, g1 = gxy + (size_t)nx * ny * gz1;
        const int cs = ly * SW + lx + 2;
#pragma unroll
        for (int v = 0; v < 8; ++v) cp_async_r(SG + v * SN5 + cs, q.p[v] + g);
        cp_async_r(SG + 8 * SN5 + cs, q.p[7] + g1);
    }
    cp_async_commit();
}

// staged plane -> primitives with the face-averaged field (ct_mhd.jl:85-97) and the lower faces
template <class R>
__device__ __forceinline__ void ct_unstage_plane(R* __restrict__ PRs, R* __restrict__ FBs, const R* __restrict__ SG,
                                                 int PN, int PNc, int PW, int SN5, int SW, const Consts<R>& K, int tid,
                                                 int nt) {
    for (int c = tid; c < PNc; c += nt) {
        const int lx = c % PW, ly = c / PW;
        const int c5 = ly * SW + lx + 2;
        Q9<R> cu;
#pragma unroll
        for (int v = 0; v < 5; ++v) cu.v[v] = SG[v * SN5 + c5];
        const R bxl = SG[5 * SN5 + c5], byl = SG[6 * SN5 + c5], bzl = SG[7 * SN5 + c5];
        cu.v[5] = R(0.5) * (bxl + SG[5 * SN5 + c5 + 1]);
        cu.v[6] = R(0.5) * (byl + SG[6 * SN5 + c5 + SW]);
        cu.v[7] = R(0.5) * (bzl + SG[8 * SN5 + c5]);
        cu.v[8] = R(0);
        const Q9<R> q = cons2prim(cu, K.gamma, K.smallr, K.smallp);
        Lay<R>::put(PRs, PN, c, q);
        FBs[0 * PN + c] = bxl;
        FBs[1 * PN + c] = byl;
        FBs[2 * PN + c] = bzl;
    }
}

// one cell's slope and 1-D predictor along D (spike_ctm / ct_mhd.jl:40-80)
template <class R> struct CTCell {
    Q9<R> m0, s, mh;
};

template <int D, class R>
__device__ __forceinline__ void ct_neighbours(const R* PR, int PN, int PW, int c, int s0, int sm, int sp, Q9<R>& L,
                                              Q9<R>& Rr) {
    const R* PL = PR + (size_t)(D == 2 ? sm : s0) * 9 * PN;
    const R* PP = PR + (size_t)(D == 2 ? sp : s0) * 9 * PN;
    const int cl = D == 0 ? c - 1 : (D == 1 ? c - PW : c), cr = D == 0 ? c + 1 : (D == 1 ? c + PW : c);
    L = Lay<R>::get(PL, PN, cl);
    Rr = Lay<R>::get(PP, PN, cr);
}

template <int D, class R>
__device__ __forceinline__ void ct_prep(CTCell<R>& r, const R* PR, int PN, int PW, int c, int s0, int sm, int sp,
                                        const Consts<R>& K, R dtdx, int halfslope) {
    Q9<R> L, Rr;
    ct_neighbours<D>(PR, PN, PW, c, s0, sm, sp, L, Rr);
    r.s = full_slope(L, r.m0, Rr);
    if (halfslope) {
#pragma unroll
        for (int v = 0; v < 9; ++v) r.s.v[v] = R(0.5) * r.s.v[v];
    }
    r.mh = hanc1d<D>(r.m0, r.s, dtdx, K.gamma, K.smallr, K.smallp);
}

// face state on the SIGN side along D, floored, with the face normal field bn
template <int D, int SIGN, int RECON, class R>
__device__ __forceinline__ Q9<R> ct_state(const CTCell<R>& r, const R* PR, int PN, int PW, int c, int s0, int sm,
                                          int sp, const Consts<R>& K, R bn) {
    Q9<R> f;
    if (RECON == RECON_PPM) {
        Q9<R> L, Rr;
        ct_neighbours<D>(PR, PN, PW, c, s0, sm, sp, L, Rr);
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            R lo, hi;
            ppm_edges(L.v[v], r.m0.v[v], Rr.v[v], lo, hi);
            f.v[v] = (SIGN > 0 ? hi : lo) + r.mh.v[v] - r.m0.v[v];
        }
    } else {
        f = padd(r.mh, r.s, SIGN > 0 ? R(0.5) : R(-0.5));
    }
    f.v[0] = rmax(f.v[0], K.smallr);
    f.v[4] = rmax(f.v[4], K.smallp);
    f.v[5 + D] = bn;
    f.v[8] = R(0);
    return f;
}

template <int D, int RIEM, class R>
__device__ __forceinline__ Q9<R> ct_flux(const Q9<R>& L, const Q9<R>& Rr, const Consts<R>& K) {
    const Q9<R> Lr = rot_to<D>(L), Rrr = rot_to<D>(Rr);
    const R bn = Lr.v[5];
    return rot_from<D>(RIEM == RIEM_HLLD ? hlld_x(Lr, Rrr, K.gamma, bn, R(0), R(0))
                                         : hll_x(Lr, Rrr, K.gamma, bn, R(0), R(0)));
}

template <class R, int RECON, int RIEM, int TOX, int TOY>
__device__ __forceinline__ void ct_tile(const CTArgs<R>& A, int bx, int by, int bz, unsigned char* smem_raw) {
    const int OX = TOX > 0 ? TOX : A.ox, OY = TOY > 0 ? TOY : A.oy;
    const int PW = OX + 4, PN = lay_n<R>((OX + 4) * (OY + 4));   // padded array lengths (Lay layout)
    const int PNc = (OX + 4) * (OY + 4);                           // ring cells per plane
    const int PW5 = OX + 5, PN5 = (OX + 5) * (OY + 5);
    const int SW = OX + 8, SN5 = (OX + 8) * (OY + 5);
    const int RW = OX + 2, RN = lay_n<R>((OX + 2) * (OY + 2));
    R* PR = reinterpret_cast<R*>(smem_raw);
    R* FB = PR + 27 * PN;
    R* ST = FB + 9 * PN;
    R* SG = reinterpret_cast<R*>(smem_raw + ct_tile_sg_offset<R>(OX, OY));
    double* red = reinterpret_cast<double*>(smem_raw + ct_tile_words_offset<R>(OX, OY));
    // FP32 forcing tables of the tile: the x table of its columns (staged once) and the row table
    // of its rows for the plane written next (staged in the phase before that write-out)
    float* TS = reinterpret_cast<float*>(smem_raw + ct_tile_words_offset<R>(OX, OY) + 40 * sizeof(double));
    float* BS = TS + 8 * OX;

    const int tid = threadIdx.x, NT = OX * OY;
    const int tx = tid % OX, ty = tid / OX;
    const int x0 = bx * OX, y0 = by * OY;
    const int z0 = bz * A.lz, z1 = min(z0 + A.lz, A.nz);
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const size_t n = (size_t)nx * ny * nz;
    const Consts<R> K = A.K;
    const R dtdx = A.dtdx;
    const bool turb = A.do_turb && A.btab != nullptr;
    const int nhelp = 2 * (OX + OY);
    // staging skips the helper warps, the primitive conversion the boundary-face warps (the two
    // phases' barrier tails; as in the GLM tile march)
    const int oxp = 32 * ((OX + 31) / 32);   // boundary faces: y on [0, OX), x on [oxp, oxp + OY)
    const int hwarp = 32 * ((nhelp + 31) / 32), bwarp = oxp + 32 * ((OY + 31) / 32);
    const int stg0 = NT - hwarp >= 32 ? hwarp : 0;
    const int nunst = NT - bwarp >= 32 ? NT - bwarp : NT;
    R* S = A.scratch;

    // TMA staging (tiles whose region x0-4 .. x0+OX+3, y0-2 .. y0+OY+2 lies inside the box):
    // one copy of the 8 state variables of plane k+2 and one of bzf at k+3 per plane
    bool tma = false;
    {
        tma = A.use_tma && !A.wait_test && x0 >= 4 && x0 + OX + 4 <= nx && y0 >= 2 && y0 + OY + 3 <= ny;
        if ((unsigned)__cvta_generic_to_shared(SG) & 127u) tma = false;
    }
    const unsigned tma_bytes = (unsigned)(9 * SN5 * sizeof(R));

    if constexpr (std::is_same<R, float>::value) {
        if (A.trig8)
            for (int i = tid; i < 2 * OX; i += NT)
                reinterpret_cast<float4*>(TS)[i] = reinterpret_cast<const float4*>(A.trig8 + 8 * (size_t)x0)[i];
    }
    uint64_t* mbar = reinterpret_cast<uint64_t*>(red + 32);
    for (int j = 0; j < 3; ++j) {
        ct_stage_plane(SG, A.q, PN5, PW5, SW, SN5, x0, y0, z0 - 2 + j, nx, ny, nz, tid, NT);
        cp_async_wait_all();
        __syncthreads();
        ct_unstage_plane(PR + mod3(z0 - 2 + j) * 9 * PN, FB + mod3(z0 - 2 + j) * 3 * PN, SG, PN, PNc, PW, SN5, SW, K,
                         tid, NT);
        if (j == 2 && tid == 0) {
            mbar_init(mbar, tma ? 1u : (unsigned)NT);
            if (tma) fence_mbar_init();
        }
        __syncthreads();
    }

    Q9<R> pPz, Fzlo, Fxh, Fyh;
#pragma unroll
    for (int v = 0; v < 9; ++v) { pPz.v[v] = R(0); Fzlo.v[v] = R(0); Fxh.v[v] = R(0); Fyh.v[v] = R(0); }
    const int gx = x0 + tx, gy = y0 + ty;
    const int cown = (tx + 2) + PW * (ty + 2);
    const int rown = (tx + 1) + RW * (ty + 1);
    const int ixh = (tx + 2) + RW * (ty + 1);
    const int iyh = (tx + 1) + RW * (ty + 2);
    unsigned phase = 0;

    for (int kr = z0 - 1; kr <= z1; ++kr) {
        const bool first = kr == z0 - 1, last = kr == z1;
        const bool load = kr + 2 <= z1 + 1;
        const int s0 = mod3(kr), sm = mod3(kr - 1), sp = mod3(kr + 1);
        const R* FB0 = FB + (size_t)s0 * 3 * PN;
        if (load) {
            {
                if (tma && tid == 0) {
                    fence_proxy_async_smem();   // the previous plane's reads of SG come first
                    mbar_arrive_expect_tx(mbar, tma_bytes);
                    tma_load_4d(SG, &A.tmap8, x0 - 4, y0 - 2, wrapi(kr + 2, nz), 0, mbar);
                    tma_load_4d(SG + 8 * SN5, &A.tmap1, x0 - 4, y0 - 2, wrapi(kr + 3, nz), 7, mbar);
                }
            }
            if (!tma && !A.wait_test) {
                ct_stage_plane(SG, A.q, PN5, PW5, SW, SN5, x0, y0, kr + 2, nx, ny, nz, tid >= stg0 ? tid - stg0 : PN5,
                               NT - stg0);
                mbar_arrive_cp_async(mbar);
            }
        }
        {
            Q9<R> XY, Fxl, Fyl;
            if (kr - 1 >= z0) {
                Fxl = Lay<R>::get(ST + 1 * 9 * RN, RN, rown);
                Fyl = Lay<R>::get(ST + 3 * 9 * RN, RN, rown);
#pragma unroll
                for (int v = 0; v < 9; ++v) XY.v[v] = (Fxl.v[v] - Fxh.v[v]) + (Fyl.v[v] - Fyh.v[v]);
            }
            CTCell<R> r;
            r.m0 = Lay<R>::get(PR + (size_t)s0 * 9 * PN, PN, cown);
            if (!first && !last) {
                ct_prep<0>(r, PR, PN, PW, cown, s0, sm, sp, K, dtdx, A.halfslope);
                Lay<R>::put(ST + 0 * 9 * RN, RN, rown,
                       ct_state<0, +1, RECON>(r, PR, PN, PW, cown, s0, sm, sp, K, FB0[0 * PN + cown + 1]));
                Lay<R>::put(ST + 1 * 9 * RN, RN, rown,
                       ct_state<0, -1, RECON>(r, PR, PN, PW, cown, s0, sm, sp, K, FB0[0 * PN + cown]));
                ct_prep<1>(r, PR, PN, PW, cown, s0, sm, sp, K, dtdx, A.halfslope);
                Lay<R>::put(ST + 2 * 9 * RN, RN, rown,
                       ct_state<1, +1, RECON>(r, PR, PN, PW, cown, s0, sm, sp, K, FB0[1 * PN + cown + PW]));
                Lay<R>::put(ST + 3 * 9 * RN, RN, rown,
                       ct_state<1, -1, RECON>(r, PR, PN, PW, cown, s0, sm, sp, K, FB0[1 * PN + cown]));
            }
            ct_prep<2>(r, PR, PN, PW, cown, s0, sm, sp, K, dtdx, A.halfslope);
            const R* FBp = FB + (size_t)sp * 3 * PN;
            Q9<R> Pz = ct_state<2, +1, RECON>(r, PR, PN, PW, cown, s0, sm, sp, K, FBp[2 * PN + cown]);
            if (!first) {
                // the old cell state written out below, loaded before the z-face solve so that the
                // solve hides its latency
                const bool wr = kr - 1 >= z0;
                const int kf = kr - 1;
                const size_t g = (size_t)gx + (size_t)nx * ((size_t)gy + (size_t)ny * (wr ? kf : 0));
                R u0[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) u0[v] = wr ? __ldg(A.q.p[v] + g) : R(0);
                Q9<R> Mz = ct_state<2, -1, RECON>(r, PR, PN, PW, cown, s0, sm, sp, K, FB0[2 * PN + cown]);
                Q9<R> Fzhi = ct_flux<2, RIEM>(pPz, Mz, K);
                if (wr) {
                    const R* Pm = PR + (size_t)sm * 9 * PN;
                    Q9<R> q;
#pragma unroll
                    for (int v = 0; v < 5; ++v) q.v[v] = u0[v] + dtdx * (XY.v[v] + (Fzlo.v[v] - Fzhi.v[v]));
                    // the epilogue sees the old cell-centred field
                    const Q9<R> pm = Lay<R>::get(Pm, PN, cown);
                    const R vx = pm.v[1], vy = pm.v[2], vz = pm.v[3];
                    const R bxc = pm.v[5], byc = pm.v[6], bzc = pm.v[7];
                    q.v[5] = bxc; q.v[6] = byc; q.v[7] = bzc; q.v[8] = R(0);
                    R ax = R(0), ay = R(0), az = R(0);
                    if (turb) {
                        if constexpr (std::is_same<R, float>::value) {
                            if (A.trig8) force_accel_f32(BS + 24 * ty, TS, tx, A.ramp, ax, ay, az);
                            else force_accel(A.btab + ((size_t)kf * ny + gy) * 24, A.trigx, nx, gx, A.ramp, ax, ay, az);
                        } else {
                            force_accel(A.btab + ((size_t)kf * ny + gy) * 24, A.trigx, nx, gx, A.ramp, ax, ay, az);
                        }
                    }
                    finish_update(q, K, R(1), turb, ax, ay, az, A.dt);
#pragma unroll
                    for (int v = 0; v < 5; ++v) A.o.p[v][g] = q.v[v];
                    // EMF data of the three lower faces and the cell-centre EMF (-(v x B))
                    S[CS_EZX * n + g] = -Fxl.v[6];
                    S[CS_EYX * n + g] = Fxl.v[7];
                    S[CS_MX * n + g] = Fxl.v[0];
                    S[CS_EXY * n + g] = -Fyl.v[7];
                    S[CS_EZY * n + g] = Fyl.v[5];
                    S[CS_MY * n + g] = Fyl.v[0];
                    S[CS_EYZ * n + g] = -Fzlo.v[5];
                    S[CS_EXZ * n + g] = Fzlo.v[6];
                    S[CS_MZ * n + g] = Fzlo.v[0];
                    S[CS_ECX * n + g] = -(vy * bzc - vz * byc);
                    S[CS_ECY * n + g] = -(vz * bxc - vx * bzc);
                    S[CS_ECZ * n + g] = -(vx * byc - vy * bxc);
                }
                Fzlo = Fzhi;
            }
            pPz = Pz;
        }
        if (!first && !last) {
            // halo cells: the one interface state each contributes to the tile's faces
            for (int h = tid; h < nhelp; h += NT) {
                int rc, cc, which;
                if (h < OY) { rc = 0 + RW * (h + 1); cc = 1 + PW * (h + 2); which = 0; }
                else if (h < 2 * OY) { int f = h - OY; rc = (OX + 1) + RW * (f + 1); cc = (OX + 2) + PW * (f + 2); which = 1; }
                else if (h < 2 * OY + OX) { int f = h - 2 * OY; rc = (f + 1); cc = (f + 2) + PW * 1; which = 2; }
                else { int f = h - 2 * OY - OX; rc = (f + 1) + RW * (OY + 1); cc = (f + 2) + PW * (OY + 2); which = 3; }
                CTCell<R> r;
                r.m0 = Lay<R>::get(PR + (size_t)s0 * 9 * PN, PN, cc);
                Q9<R> f;
                if (which < 2) {
                    ct_prep<0>(r, PR, PN, PW, cc, s0, sm, sp, K, dtdx, A.halfslope);
                    if (which == 0) f = ct_state<0, +1, RECON>(r, PR, PN, PW, cc, s0, sm, sp, K, FB0[0 * PN + cc + 1]);
                    else f = ct_state<0, -1, RECON>(r, PR, PN, PW, cc, s0, sm, sp, K, FB0[0 * PN + cc]);
                } else {
                    ct_prep<1>(r, PR, PN, PW, cc, s0, sm, sp, K, dtdx, A.halfslope);
                    if (which == 2) f = ct_state<1, +1, RECON>(r, PR, PN, PW, cc, s0, sm, sp, K, FB0[1 * PN + cc + PW]);
                    else f = ct_state<1, -1, RECON>(r, PR, PN, PW, cc, s0, sm, sp, K, FB0[1 * PN + cc]);
                }
                Lay<R>::put(ST + which * 9 * RN, RN, rc, f);
            }
        }
        __syncthreads();
        if (!first && !last) {
            Fxh = ct_flux<0, RIEM>(Lay<R>::get(ST + 0 * 9 * RN, RN, rown), Lay<R>::get(ST + 1 * 9 * RN, RN, ixh), K);
            Lay<R>::put(ST + 1 * 9 * RN, RN, ixh, Fxh);
            Fyh = ct_flux<1, RIEM>(Lay<R>::get(ST + 2 * 9 * RN, RN, rown), Lay<R>::get(ST + 3 * 9 * RN, RN, iyh), K);
            Lay<R>::put(ST + 3 * 9 * RN, RN, iyh, Fyh);
            for (int h = NT - 1 - tid; h < oxp + OY; h += NT) {
                // y faces first, x faces from the next warp boundary (no warp runs both paths)
                if (h < OX) {
                    const int il = (h + 1), ir = (h + 1) + RW;
                    Lay<R>::put(ST + 3 * 9 * RN, RN, ir, ct_flux<1, RIEM>(Lay<R>::get(ST + 2 * 9 * RN, RN, il), Lay<R>::get(ST + 3 * 9 * RN, RN, ir), K));
                } else if (h >= oxp) {
                    const int f = h - oxp;
                    const int il = 0 + RW * (f + 1), ir = 1 + RW * (f + 1);
                    Lay<R>::put(ST + 1 * 9 * RN, RN, ir, ct_flux<0, RIEM>(Lay<R>::get(ST + 0 * 9 * RN, RN, il), Lay<R>::get(ST + 1 * 9 * RN, RN, ir), K));
                }
            }
        }
        // the forcing row table of the tile's rows for plane kr, written out in the next phase
        if constexpr (std::is_same<R, float>::value) {
            if (turb && A.trig8 && kr >= z0 && kr < z1)
                for (int i = tid; i < 6 * OY; i += NT)
                    reinterpret_cast<float4*>(BS)[i] =
                        reinterpret_cast<const float4*>(A.btab + ((size_t)kr * ny + y0) * 24)[i];
        }
        if (load) {
            mbar_wait(mbar, phase, A.err, A.wait_cycles);
            phase ^= 1u;
            ct_unstage_plane(PR + mod3(kr + 2) * 9 * PN, FB + mod3(kr + 2) * 3 * PN, SG, PN, PNc, PW, SN5, SW, K,
                             tid < nunst ? tid : PNc, nunst);
        }
        __syncthreads();
    }
    if (tid == 0) mbar_inval(mbar);
}

template <class R, int RECON, int RIEM, int MAXT, int MINB, int TOX = 0, int TOY = 0>
__global__ void __launch_bounds__(MAXT, MINB) ct_tile_kernel(const __grid_constant__ CTArgs<R> A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    ct_tile<R, RECON, RIEM, TOX, TOY>(A, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

template <class R> __device__ __forceinline__ R ct_upwind(R flux, R minus, R plus) {
    return flux > R(0) ? minus : (flux < R(0) ? plus : R(0.5) * (minus + plus));
}

// Pass B1: the three edge EMFs of cell (i,j,k) -- ez at (i-1/2, j-1/2, k), ex at (i, j-1/2, k-1/2),
// ey at (i-1/2, j, k-1/2) -- for the cyclic axes (A, B, e): on the A-face the face EMF is
// -F_A[B_B], on the B-face +F_B[B_A]; the same expressions and order as the oracle.
// All loads of a cell come first and all stores after them, so that a thread keeps its loads in
// flight together (the stores go to other scratch planes than the loads read).
template <class R, bool CONTACT> __global__ void __launch_bounds__(256) ct_edge_kernel(const CTArgs<R> A) {
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const size_t n = (size_t)nx * ny * nz;
    const R* S = A.scratch;
    R* W = A.scratch;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_coords(c, nx, ny, n, x, y, z);
        const size_t xm = (size_t)wrap1(x - 1, nx) + (size_t)nx * (y + (size_t)ny * z);
        const size_t ym = (size_t)x + (size_t)nx * (wrap1(y - 1, ny) + (size_t)ny * z);
        const size_t zm = (size_t)x + (size_t)nx * (y + (size_t)ny * wrap1(z - 1, nz));
        // per edge e: EaN, EaS, EbE, EbW, then (contact) e00, e10, e01, e11, maN, maS, mbE, mbW
        R v[3][12];
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            // A = (e+1)%3, B = (e+2)%3; c10 = one step back along A, c01 along B, c11 along both
            size_t c10, c01, c11;
            int ea, eb, ma, mb, ec;
            if (e == 2) {        // (A,B) = (x,y)
                c10 = xm; c01 = ym;
                c11 = (size_t)wrap1(x - 1, nx) + (size_t)nx * (wrap1(y - 1, ny) + (size_t)ny * z);
                ea = CS_EZX; eb = CS_EZY; ma = CS_MX; mb = CS_MY; ec = CS_ECZ;
            } else if (e == 0) { // (A,B) = (y,z)
                c10 = ym; c01 = zm;
                c11 = (size_t)x + (size_t)nx * (wrap1(y - 1, ny) + (size_t)ny * wrap1(z - 1, nz));
                ea = CS_EXY; eb = CS_EXZ; ma = CS_MY; mb = CS_MZ; ec = CS_ECX;
            } else {             // (A,B) = (z,x)
                c10 = zm; c01 = xm;
                c11 = (size_t)wrap1(x - 1, nx) + (size_t)nx * (y + (size_t)ny * wrap1(z - 1, nz));
                ea = CS_EYZ; eb = CS_EYX; ma = CS_MZ; mb = CS_MX; ec = CS_ECY;
            }
            v[e][0] = S[ea * n + c];
            v[e][1] = S[ea * n + c01];
            v[e][2] = S[eb * n + c];
            v[e][3] = S[eb * n + c10];
            if (CONTACT) {
                v[e][4] = S[ec * n + c];
                v[e][5] = S[ec * n + c10];
                v[e][6] = S[ec * n + c01];
                v[e][7] = S[ec * n + c11];
                v[e][8] = S[ma * n + c];
                v[e][9] = S[ma * n + c01];
                v[e][10] = S[mb * n + c];
                v[e][11] = S[mb * n + c10];
            }
        }
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            const R EaN = v[e][0], EaS = v[e][1], EbE = v[e][2], EbW = v[e][3];
            R E = R(0.25) * (EbE + EbW + EaN + EaS);
            if (CONTACT) {
                const R e00 = v[e][4], e10 = v[e][5], e01 = v[e][6], e11 = v[e][7];
                const R dN = ct_upwind(v[e][8], e10 - EbW, e00 - EbE);
                const R dS = ct_upwind(v[e][9], EbW - e11, EbE - e01);
                const R dE = ct_upwind(v[e][10], e01 - EaS, e00 - EaN);
                const R dW = ct_upwind(v[e][11], EaS - e11, EaN - e10);
                E = E + R(0.25) * (dS - dN) + R(0.25) * (dW - dE);
            }
            W[(CS_EDX + e) * n + c] = E;
        }
    }
}

// Pass B2: face B by the curl of the edge EMFs
template <class R> __global__ void __launch_bounds__(256) ct_face_kernel(const CTArgs<R> A) {
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const size_t n = (size_t)nx * ny * nz;
    const R* ex = A.scratch + CS_EDX * n;
    const R* ey = A.scratch + CS_EDY * n;
    const R* ez = A.scratch + CS_EDZ * n;
    const R dtdx = A.dtdx;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_coords(c, nx, ny, n, x, y, z);
        const size_t cxp = (size_t)wrap1(x + 1, nx) + (size_t)nx * (y + (size_t)ny * z);
        const size_t cyp = (size_t)x + (size_t)nx * (wrap1(y + 1, ny) + (size_t)ny * z);
        const size_t czp = (size_t)x + (size_t)nx * (y + (size_t)ny * wrap1(z + 1, nz));
        // every load before the first store (the outputs may share an allocation with the inputs)
        const R exc = ex[c], eyc = ey[c], ezc = ez[c];
        const R ezy = ez[cyp], eyz = ey[czp], exz = ex[czp], ezx = ez[cxp], eyx = ey[cxp], exy = ex[cyp];
        const R b5 = A.q.p[5][c], b6 = A.q.p[6][c], b7 = A.q.p[7][c];
        A.o.p[5][c] = b5 - dtdx * ((ezy - ezc) - (eyz - eyc));
        A.o.p[6][c] = b6 - dtdx * ((exz - exc) - (ezx - ezc));
        A.o.p[7][c] = b7 - dtdx * ((eyx - eyc) - (exy - exc));
    }
}

// FP32 passes B1 and B2 four cells per thread (x0 = 4k): every plane is read as one 16-byte load
// per thread, and a neighbour one cell back (forward) in x as the same quad shifted by one cell,
// its outside value read separately (from the other end of the row at the periodic boundary).
// Requires nx % 4 == 0 and 16-byte aligned planes; the per-cell arithmetic is the scalar passes'.
struct CTQuad {
    const float* S;
    size_t n;
    int x, nx;
    __device__ __forceinline__ float4 at(int plane, size_t base) const {
        return __ldg(reinterpret_cast<const float4*>(S + (size_t)plane * n + base));
    }
    // cells base-1 .. base+2 (base is the first cell of a quad at column x of its row)
    __device__ __forceinline__ float4 back(int plane, size_t base) const {
        const float4 q = at(plane, base);
        const float w = __ldg(S + (size_t)plane * n + (x == 0 ? base + nx - 1 : base - 1));
        return make_float4(w, q.x, q.y, q.z);
    }
};
__device__ __forceinline__ float q4(const float4& v, int j) { return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w)); }

// three blocks per SM (at most 85 registers, a 40-byte spill): 2.8 % faster for the whole CT step than
// two blocks at 92 registers, the pass being bound by loads in flight
template <bool CONTACT> __global__ void __launch_bounds__(256, 3) ct_edge_kernel4(const CTArgs<float> A) {
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const size_t n = (size_t)nx * ny * nz, nq = n / 4;
    float* W = A.scratch;
    for (size_t qd = (size_t)blockIdx.x * blockDim.x + threadIdx.x; qd < nq; qd += (size_t)gridDim.x * blockDim.x) {
        const size_t c = 4 * qd;
        int x, y, z;
        cell_coords(c, nx, ny, n, x, y, z);
        const CTQuad Q{A.scratch, n, x, nx};
        const size_t ym = (size_t)x + (size_t)nx * (wrap1(y - 1, ny) + (size_t)ny * z);
        const size_t zm = (size_t)x + (size_t)nx * (y + (size_t)ny * wrap1(z - 1, nz));
        const size_t yzm = (size_t)x + (size_t)nx * (wrap1(y - 1, ny) + (size_t)ny * wrap1(z - 1, nz));
        // per edge e as in ct_edge_kernel: EaN, EaS, EbE, EbW, then e00, e10, e01, e11, maN, maS, mbE, mbW
        float4 v[3][CONTACT ? 12 : 4];
        // e = 0: (A,B) = (y,z), c10 = y-1, c01 = z-1
        v[0][0] = Q.at(CS_EXY, c); v[0][1] = Q.at(CS_EXY, zm); v[0][2] = Q.at(CS_EXZ, c); v[0][3] = Q.at(CS_EXZ, ym);
        // e = 1: (A,B) = (z,x), c10 = z-1, c01 = x-1
        v[1][0] = Q.at(CS_EYZ, c); v[1][1] = Q.back(CS_EYZ, c); v[1][2] = Q.at(CS_EYX, c); v[1][3] = Q.at(CS_EYX, zm);
        // e = 2: (A,B) = (x,y), c10 = x-1, c01 = y-1
        v[2][0] = Q.at(CS_EZX, c); v[2][1] = Q.at(CS_EZX, ym); v[2][2] = Q.at(CS_EZY, c); v[2][3] = Q.back(CS_EZY, c);
        if constexpr (CONTACT) {
            v[0][4] = Q.at(CS_ECX, c); v[0][5] = Q.at(CS_ECX, ym); v[0][6] = Q.at(CS_ECX, zm); v[0][7] = Q.at(CS_ECX, yzm);
            v[0][8] = Q.at(CS_MY, c); v[0][9] = Q.at(CS_MY, zm); v[0][10] = Q.at(CS_MZ, c); v[0][11] = Q.at(CS_MZ, ym);
            v[1][4] = Q.at(CS_ECY, c); v[1][5] = Q.at(CS_ECY, zm); v[1][6] = Q.back(CS_ECY, c); v[1][7] = Q.back(CS_ECY, zm);
            v[1][8] = Q.at(CS_MZ, c); v[1][9] = Q.back(CS_MZ, c); v[1][10] = Q.at(CS_MX, c); v[1][11] = Q.at(CS_MX, zm);
            v[2][4] = Q.at(CS_ECZ, c); v[2][5] = Q.back(CS_ECZ, c); v[2][6] = Q.at(CS_ECZ, ym); v[2][7] = Q.back(CS_ECZ, ym);
            v[2][8] = Q.at(CS_MX, c); v[2][9] = Q.at(CS_MX, ym); v[2][10] = Q.at(CS_MY, c); v[2][11] = Q.back(CS_MY, c);
        }
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            float out[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float EaN = q4(v[e][0], j), EaS = q4(v[e][1], j), EbE = q4(v[e][2], j), EbW = q4(v[e][3], j);
                float E = 0.25f * (EbE + EbW + EaN + EaS);
                if constexpr (CONTACT) {
                    const float e00 = q4(v[e][4], j), e10 = q4(v[e][5], j), e01 = q4(v[e][6], j), e11 = q4(v[e][7], j);
                    const float dN = ct_upwind(q4(v[e][8], j), e10 - EbW, e00 - EbE);
                    const float dS = ct_upwind(q4(v[e][9], j), EbW - e11, EbE - e01);
                    const float dE = ct_upwind(q4(v[e][10], j), e01 - EaS, e00 - EaN);
                    const float dW = ct_upwind(q4(v[e][11], j), EaS - e11, EaN - e10);
                    E = E + 0.25f * (dS - dN) + 0.25f * (dW - dE);
                }
                out[j] = E;
            }
            *reinterpret_cast<float4*>(W + (size_t)(CS_EDX + e) * n + c) = make_float4(out[0], out[1], out[2], out[3]);
        }
    }
}

template <class R> __global__ void __launch_bounds__(256) ct_face_kernel4(const CTArgs<R> A) {
    static_assert(std::is_same<R, float>::value, "the 4-wide CT passes are FP32");
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const size_t n = (size_t)nx * ny * nz, nq = n / 4;
    const float* ex = A.scratch + CS_EDX * n;
    const float* ey = A.scratch + CS_EDY * n;
    const float* ez = A.scratch + CS_EDZ * n;
    const float dtdx = A.dtdx;
    for (size_t qd = (size_t)blockIdx.x * blockDim.x + threadIdx.x; qd < nq; qd += (size_t)gridDim.x * blockDim.x) {
        const size_t c = 4 * qd;
        int x, y, z;
        cell_coords(c, nx, ny, n, x, y, z);
        const size_t cyp = (size_t)x + (size_t)nx * (wrap1(y + 1, ny) + (size_t)ny * z);
        const size_t czp = (size_t)x + (size_t)nx * (y + (size_t)ny * wrap1(z + 1, nz));
        const size_t cxn = x + 4 == nx ? c + 4 - nx : c + 4;   // first cell of the next quad of the row
        auto ld = [](const float* p, size_t i) { return __ldg(reinterpret_cast<const float4*>(p + i)); };
        // every load before the first store (the outputs may share an allocation with the inputs)
        const float4 exc = ld(ex, c), eyc = ld(ey, c), ezc = ld(ez, c);
        const float4 ezy = ld(ez, cyp), eyz = ld(ey, czp), exz = ld(ex, czp), exy = ld(ex, cyp);
        const float4 ezq = ezc, eyq = eyc;
        const float ezn = __ldg(ez + cxn), eyn = __ldg(ey + cxn);
        const float4 ezx = make_float4(ezq.y, ezq.z, ezq.w, ezn), eyx = make_float4(eyq.y, eyq.z, eyq.w, eyn);
        // the face field through the coherent path: its planes are the outputs' counterparts (the
        // read-only cache is for data this kernel does not write)
        auto ldc = [](const float* p, size_t i) { return *reinterpret_cast<const float4*>(p + i); };
        const float4 b5 = ldc(A.q.p[5], c), b6 = ldc(A.q.p[6], c), b7 = ldc(A.q.p[7], c);
        float o5[4], o6[4], o7[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            o5[j] = q4(b5, j) - dtdx * ((q4(ezy, j) - q4(ezc, j)) - (q4(eyz, j) - q4(eyc, j)));
            o6[j] = q4(b6, j) - dtdx * ((q4(exz, j) - q4(exc, j)) - (q4(ezx, j) - q4(ezc, j)));
            o7[j] = q4(b7, j) - dtdx * ((q4(eyx, j) - q4(eyc, j)) - (q4(exy, j) - q4(exc, j)));
        }
        *reinterpret_cast<float4*>(A.o.p[5] + c) = make_float4(o5[0], o5[1], o5[2], o5[3]);
        *reinterpret_cast<float4*>(A.o.p[6] + c) = make_float4(o6[0], o6[1], o6[2], o6[3]);
        *reinterpret_cast<float4*>(A.o.p[7] + c) = make_float4(o7[0], o7[1], o7[2], o7[3]);
    }
}

// the 4-wide passes apply: FP32, nx a multiple of 4, every plane they touch 16-byte aligned
template <class R> inline bool ct_quad_ok(const CTArgs<R>& A) {
    if (sizeof(R) != 4 || A.nx % 4 != 0) return false;
    auto al = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
    if (!al(A.scratch) || ((size_t)A.nx * A.ny * A.nz) % 4 != 0) return false;
    for (int v = 5; v < 8; ++v)
        if (!al(A.q.p[v]) || !al(A.o.p[v])) return false;
    return true;
}

// launch: pass A (tile kernel), then B1 and B2; nt <= 0 in A configures the kernel only
template <class R, int RECON, int RIEM, int MAXT, int MINB, int TOX = 0, int TOY = 0>
static cudaError_t ct_go(const CTArgs<R>& A, cudaStream_t s, bool configure_only) {
    auto k = ct_tile_kernel<R, RECON, RIEM, MAXT, MINB, TOX, TOY>;
    static int configured[64] = {0};
    {
        cudaError_t e = configure_once(k, configured);
        if (e != cudaSuccess) return e;
    }
    if (configure_only) return cudaSuccess;
    const int nt = A.ox * A.oy;
    if (nt > MAXT || nt < 1) return cudaErrorInvalidConfiguration;
    dim3 grid(A.nx / A.ox, A.ny / A.oy, (A.nz + A.lz - 1) / A.lz);
    k<<<grid, nt, ct_tile_smem_bytes<R>(A.ox, A.oy), s>>>(A);
    const size_t n = (size_t)A.nx * A.ny * A.nz;
    if constexpr (std::is_same<R, float>::value) {
        if (ct_quad_ok(A)) {
            const int nb4 = (int)std::min<size_t>((n / 4 + 255) / 256, (size_t)148 * 16);
            if (A.emf == 1) ct_edge_kernel4<true><<<nb4, 256, 0, s>>>(A);
            else ct_edge_kernel4<false><<<nb4, 256, 0, s>>>(A);
            ct_face_kernel4<R><<<nb4, 256, 0, s>>>(A);
            return cudaGetLastError();
        }
    }
    const int nb = (int)std::min<size_t>((n + 255) / 256, (size_t)148 * 16);
    if (A.emf == 1) ct_edge_kernel<R, true><<<nb, 256, 0, s>>>(A);
    else ct_edge_kernel<R, false><<<nb, 256, 0, s>>>(A);
    ct_face_kernel<R><<<nb, 256, 0, s>>>(A);
    return cudaGetLastError();
}

template <class R, int MAXT, int MINB>
static cudaError_t ct_dispatch_t(const CTArgs<R>& A, int recon, int riem, cudaStream_t s, bool configure_only) {
    const bool ppm = recon == RECON_PPM, hlld = riem == RIEM_HLLD;
    if (ppm && hlld) return ct_go<R, RECON_PPM, RIEM_HLLD, MAXT, MINB>(A, s, configure_only);
    if (ppm) return ct_go<R, RECON_PPM, RIEM_HLL, MAXT, MINB>(A, s, configure_only);
    if (hlld) return ct_go<R, RECON_MC, RIEM_HLLD, MAXT, MINB>(A, s, configure_only);
    return ct_go<R, RECON_MC, RIEM_HLL, MAXT, MINB>(A, s, configure_only);
}

template <class R, int MAXT, int MINB> static cudaError_t ct_configure_all_t() {
    CTArgs<R> none{};
    cudaError_t e = cudaSuccess;
    for (int rc = 0; e == cudaSuccess && rc < 2; ++rc)
        for (int rm = 0; e == cudaSuccess && rm < 2; ++rm)
            e = ct_dispatch_t<R, MAXT, MINB>(none, rc ? RECON_PPM : RECON_MC, rm ? RIEM_HLL : RIEM_HLLD, 0, true);
    return e;
}

template <class R, int MAXT, int MINB> static int ct_regs_of_t(int recon, int riem) {
    cudaFuncAttributes fa{};
    const bool ppm = recon == RECON_PPM, hlld = riem == RIEM_HLLD;
    cudaError_t e;
    if (ppm && hlld) e = cudaFuncGetAttributes(&fa, ct_tile_kernel<R, RECON_PPM, RIEM_HLLD, MAXT, MINB>);
    else if (ppm) e = cudaFuncGetAttributes(&fa, ct_tile_kernel<R, RECON_PPM, RIEM_HLL, MAXT, MINB>);
    else if (hlld) e = cudaFuncGetAttributes(&fa, ct_tile_kernel<R, RECON_MC, RIEM_HLLD, MAXT, MINB>);
    else e = cudaFuncGetAttributes(&fa, ct_tile_kernel<R, RECON_MC, RIEM_HLL, MAXT, MINB>);
    return e == cudaSuccess ? fa.numRegs : -1;
}

}  // namespace gmt
