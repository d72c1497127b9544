// gmt_unsplit.cuh -- fused unsplit GLM-MHD step: PLM(MC|minmod)/PPM + MUSCL-Hancock +
// HLLD|HLL|LLF + Dedner GLM + void floor + psi damping + mode-sum forcing kick (+ next-step CFL).
//
// Layout.  A block owns an OX x OY column tile of the periodic box over a chunk of LZ planes and
// marches z.  Shared memory holds (9-variable arrays in the Lay layout below: FP32 cells as two
// 16-byte vectors and a scalar)
//   PR[3][(OX+4)(OY+4)]     primitive ring (planes k-1, k, k+1; 2-cell in-plane halo),
//   ST[4][(OX+2)(OY+2)]     in-plane interface states +x,-x,+y,-y of the reconstruction region,
//                           overwritten in place by the face fluxes,
//   SG[9][(OY+4)][OX+8]     conserved staging plane k+2 (the ring region at column offset 2),
//                           filled while plane k computes,
//   TS[OX][8], BS[OY][24]   FP32: the forcing kick's x table of the tile's columns and row table
//                           of its rows for the plane written next.
// Each owned thread keeps its column's z-face work in registers (the +z state of plane k-1 and
// F_z at its lower face) plus its own x/y face fluxes, so every face is solved once, every cell is
// read from HBM once and written once, and a plane costs two block barriers.  The next conserved
// plane streams in by one TMA copy (tiles clear of the box edges) or by per-thread cp.async,
// and completes on an mbarrier (bounded wait, error flag).
//
// Reference semantics: integrator_tiled!/integrator_plm!/integrator_plm_ppm!
// (glmmhd_turb.jl:608-743, 782-864, 931-1014) -- one reconstruction per cell, one Riemann solve
// per face, revert unphysical interface states (iflo, :618), update with floor, psi *= glm_fac,
// forcing kick; the streaming order follows integrator_stream! (:1842-1946).
#pragma once
#include "gmt_common.cuh"

namespace gmt {

template <class R> struct Rec {
    Q9<R> m0, mh, s[3];
    bool up;
    bool check;   // some lane of the warp may revert an interface state (warp-uniform)
};

// Shared-memory layout of the 9-variable arrays (the primitive ring, the interface states): an
// array of n cells, padded to lay_n(n) cells.  FP32: per cell the variables 0-3 and 4-7 as two
// 16-byte vectors and variable 8 alone ([A: float4 x n][B: float4 x n][C: float x n]), so one
// cell's 9 values take two 128-bit and one 32-bit access (a warp's 32 consecutive cells read
// 512 contiguous bytes per vector, conflict-free).  FP64: 9 scalar planes ([v][n]).
template <class R> __host__ __device__ constexpr int lay_n(int n) { return sizeof(R) == 4 ? (n + 3) & ~3 : n; }
template <class R> struct Lay {
    static __device__ __forceinline__ Q9<R> get(const R* __restrict__ S, int n, int c) {
        Q9<R> q;
#pragma unroll
        for (int v = 0; v < 9; ++v) q.v[v] = S[v * n + c];
        return q;
    }
    static __device__ __forceinline__ void put(R* __restrict__ S, int n, int c, const Q9<R>& q) {
#pragma unroll
        for (int v = 0; v < 9; ++v) S[v * n + c] = q.v[v];
    }
    static __device__ __forceinline__ R get1(const R* __restrict__ S, int n, int c, int v) { return S[v * n + c]; }
};
template <> struct Lay<float> {
    static __device__ __forceinline__ Q9<float> get(const float* __restrict__ S, int n, int c) {
        const float4 a = reinterpret_cast<const float4*>(S)[c];
        const float4 b = reinterpret_cast<const float4*>(S)[n + c];
        return Q9<float>{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, S[8 * n + c]}};
    }
    static __device__ __forceinline__ void put(float* __restrict__ S, int n, int c, const Q9<float>& q) {
        reinterpret_cast<float4*>(S)[c] = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
        reinterpret_cast<float4*>(S)[n + c] = make_float4(q.v[4], q.v[5], q.v[6], q.v[7]);
        S[8 * n + c] = q.v[8];
    }
    static __device__ __forceinline__ float get1(const float* __restrict__ S, int n, int c, int v) {
        return v < 8 ? S[4 * (v < 4 ? c : n + c) + (v & 3)] : S[8 * n + c];
    }
};

template <class R, int RECON>
__device__ __forceinline__ void recon_prims(const R* __restrict__ PR, int PN, int PW, int c, int s0, int sm, int sp,
                                            const Consts<R>& K, R dtdx, Rec<R>& r) {
    const R* P0 = PR + (size_t)s0 * 9 * PN;
    const R* Pm = PR + (size_t)sm * 9 * PN;
    const R* Pp = PR + (size_t)sp * 9 * PN;
    Q9<R> L, Rr;
    constexpr bool MM = RECON == RECON_MINMOD;
    bool up = true;
    r.m0 = Lay<R>::get(P0, PN, c);
    L = Lay<R>::get(P0, PN, c - 1);
    Rr = Lay<R>::get(P0, PN, c + 1);
    r.s[0] = half_slope<MM>(L, r.m0, Rr);
    if (RECON == RECON_PPM) up = up && !spj(L.v[4], r.m0.v[4], Rr.v[4]);
    L = Lay<R>::get(P0, PN, c - PW);
    Rr = Lay<R>::get(P0, PN, c + PW);
    r.s[1] = half_slope<MM>(L, r.m0, Rr);
    if (RECON == RECON_PPM) up = up && !spj(L.v[4], r.m0.v[4], Rr.v[4]);
    L = Lay<R>::get(Pm, PN, c);
    Rr = Lay<R>::get(Pp, PN, c);
    r.s[2] = half_slope<MM>(L, r.m0, Rr);
    if (RECON == RECON_PPM) up = up && !spj(L.v[4], r.m0.v[4], Rr.v[4]);
    r.up = up;
    r.mh = cons2prim(hancock(r.m0, r.s[0], r.s[1], r.s[2], dtdx, K.gamma), K.gamma, K.smallr, K.pfl);
    if (r.mh.v[0] <= K.smallr || r.mh.v[4] <= K.pfl) r.mh = r.m0;
    // PLM states are mh +- s_d, so some state of the cell has rho < smallr or p < pfl exactly when
    // mh - max_d |s_d| does (mh - |s| is the smaller state, rounded alike); one warp vote then
    // decides whether the per-state revert checks run at all.  PPM states are checked one by one.
    bool bad = RECON == RECON_PPM;
    if (RECON != RECON_PPM) {
        const R dr = rmax(rmax(rabs(r.s[0].v[0]), rabs(r.s[1].v[0])), rabs(r.s[2].v[0]));
        const R dp = rmax(rmax(rabs(r.s[0].v[4]), rabs(r.s[1].v[4])), rabs(r.s[2].v[4]));
        bad = r.mh.v[0] - dr < K.smallr || r.mh.v[4] - dp < K.pfl;
    }
    r.check = __any_sync(__activemask(), bad);
}

// interface state of the reconstructed cell on the SIGN side of axis D
template <class R, int RECON, int D, int SIGN>
__device__ __forceinline__ Q9<R> face_state(const Rec<R>& r, const R* __restrict__ PR, int PN, int PW, int c,
                                            int s0, int sm, int sp, const Consts<R>& K, int iflo) {
    Q9<R> f;
    if (RECON == RECON_PPM && r.up) {
        const R* PL;
        const R* PRr;
        int cl, cr;
        if (D == 0) { PL = PRr = PR + (size_t)s0 * 9 * PN; cl = c - 1; cr = c + 1; }
        else if (D == 1) { PL = PRr = PR + (size_t)s0 * 9 * PN; cl = c - PW; cr = c + PW; }
        else { PL = PR + (size_t)sm * 9 * PN; PRr = PR + (size_t)sp * 9 * PN; cl = c; cr = c; }
        const Q9<R> qm = Lay<R>::get(PL, PN, cl), qp = Lay<R>::get(PRr, PN, cr);
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            R lo, hi;
            ppm_edges(qm.v[v], r.m0.v[v], qp.v[v], lo, hi);
            f.v[v] = r.mh.v[v] + (SIGN > 0 ? hi : lo) - r.m0.v[v];
        }
    } else {
        f = padd(r.mh, r.s[D], SIGN > 0 ? R(1) : R(-1));
    }
    // revert an unphysical state to the cell value; the revert is rare, so the checks are skipped
    // when no lane of the warp can need them
    if (iflo && r.check) {
        const bool bad = f.v[0] < K.smallr || f.v[4] < K.pfl;
        if (bad) f = r.m0;
    }
    return f;
}

// 9 scalar planes of RN cells (the CT tile's state arrays)
template <class R> __device__ __forceinline__ void st_put(R* __restrict__ S, int RN, int idx, const Q9<R>& q) {
#pragma unroll
    for (int v = 0; v < 9; ++v) S[v * RN + idx] = q.v[v];
}
template <class R> __device__ __forceinline__ Q9<R> st_get(const R* __restrict__ S, int RN, int idx) {
    Q9<R> q;
#pragma unroll
    for (int v = 0; v < 9; ++v) q.v[v] = S[v * RN + idx];
    return q;
}

__device__ __forceinline__ int mod3(int k) {
    int m = k % 3;
    return m < 0 ? m + 3 : m;
}

// The staging plane SG holds the conserved variables of the ring region (x0-2.., y0-2..) with a
// row pitch SW = OX + 8 and the region starting at column 2: exactly the box (x0-4, y0-2) of
// (OX+8) x (OY+4) cells that one TMA copy delivers (its first column 16-byte aligned).
template <class R>
__device__ __forceinline__ void stage_plane(R* __restrict__ SG, const CPlanes<R>& u, int PN, int PW, int SW, int SN,
                                            int x0, int y0, int kp, int nx, int ny, int nz, int tid, int nt) {
    const int gz = wrapi(kp, nz);
    for (int c = tid; c < PN; c += nt) {
        int lx = c % PW, ly = c / PW;
        int gx = wrapi(x0 - 2 + lx, nx), gy = wrapi(y0 - 2 + ly, ny);
        size_t g = (size_t)gx + (size_t)nx * ((size_t)gy + (size_t)ny * gz);
        const int cs = ly * SW + lx + 2;
#pragma unroll
        for (int v = 0; v < 9; ++v) cp_async_r(SG + v * SN + cs, u.p[v] + g);
    }
    cp_async_commit();
}

// PN: the ring's padded array length (the layout stride); PNc: the ring cells to convert
template <class R>
__device__ __forceinline__ void unstage_plane(R* __restrict__ PRs, const R* __restrict__ SG, int PN, int PNc, int PW,
                                              int SW, int SN, const Consts<R>& K, R pfloor, int tid, int nt) {
    for (int c = tid; c < PNc; c += nt) {
        const int cs = (c / PW) * SW + c % PW + 2;
        Q9<R> q;
#pragma unroll
        for (int v = 0; v < 9; ++v) q.v[v] = SG[v * SN + cs];
        q = cons2prim(q, K.gamma, K.smallr, pfloor);
        Lay<R>::put(PRs, PN, c, q);
    }
}

// shared-memory layout of the tile march: PR ring, ST states, then (128-byte aligned, as a TMA
// destination) the staging plane SG, then (16-byte aligned) the reduction and mbarrier words and,
// in FP32, the tile's forcing tables (8 floats per column, 24 per row)
template <class R> __host__ __device__ inline size_t unsplit_sg_offset(int ox, int oy) {
    size_t PN = (size_t)lay_n<R>((ox + 4) * (oy + 4)), RN = (size_t)lay_n<R>((ox + 2) * (oy + 2));
    return ((27 * PN + 36 * RN) * sizeof(R) + 127) / 128 * 128;
}
template <class R> __host__ __device__ inline size_t unsplit_red_offset(int ox, int oy) {
    size_t SN = (size_t)(ox + 8) * (oy + 4);
    return (unsplit_sg_offset<R>(ox, oy) + 9 * SN * sizeof(R) + 15) / 16 * 16;
}
template <class R> __host__ __device__ inline size_t unsplit_smem_bytes(int ox, int oy) {
    return unsplit_red_offset<R>(ox, oy) + 40 * sizeof(double) + (sizeof(R) == 4 ? 32 * (size_t)ox + 96 * (size_t)oy : 0);
}

// adjoint record mode: interface state k (+x, -x, +y, -y, +z, -z) of cell g
template <class R> __device__ __forceinline__ void rec_put(const UnsplitArgs<R>& A, size_t n, int k, size_t g,
                                                          const Q9<R>& f) {
#pragma unroll
    for (int v = 0; v < 9; ++v) A.rec_fs[(size_t)(k * 9 + v) * n + g] = f.v[v];
}

// The two schemes that share the tile march.  A scheme supplies the primitive floor of the
// staged planes, the reconstruction of a cell (recon, then prep<D> before the states of
// direction D), its interface states, the face flux and the update epilogue.
//
// Unsplit (integrator_tiled!/plm!/plm_ppm!): one MUSCL-Hancock predictor over all three
// directions, iflo revert, HLLD/HLL/LLF + GLM, void floor, psi damping and forcing kick.
template <class R, int RECON, int RIEM> struct UnsplitScheme {
    using Cell = Rec<R>;
    static constexpr bool kRecord = false;   // adjoint record mode (AdjRecordScheme)
    // load the write-out's old state before the z-face solve: it pays in FP32 with HLLD, whose
    // long solve hides the load; with HLL, and in FP64 (255 registers), it measured slower
    static constexpr bool kEarlyOld = std::is_same<R, float>::value && RIEM == RIEM_HLLD;
    static __device__ __forceinline__ R prim_floor(const Consts<R>& K) { return K.pfl; }
    static __device__ __forceinline__ void recon(const R* PR, int PN, int PW, int c, int s0, int sm, int sp,
                                                 const Consts<R>& K, R dtdx, Cell& r) {
        recon_prims<R, RECON>(PR, PN, PW, c, s0, sm, sp, K, dtdx, r);
    }
    template <int D>
    static __device__ __forceinline__ void prep(Cell&, const R*, int, int, int, int, int, int, const Consts<R>&, R) {}
    template <int D, int SIGN>
    static __device__ __forceinline__ Q9<R> state(const Cell& r, const R* PR, int PN, int PW, int c, int s0, int sm,
                                                  int sp, const Consts<R>& K, int iflo) {
        return face_state<R, RECON, D, SIGN>(r, PR, PN, PW, c, s0, sm, sp, K, iflo);
    }
    template <int D>
    static __device__ __forceinline__ Q9<R> flux(const Q9<R>& L, const Q9<R>& Rr, const Consts<R>& K, R ch, bool llf) {
        return riemann_glm<D, RIEM>(L, Rr, K, ch, llf);
    }
    static __device__ __forceinline__ void finish(Q9<R>& q, const Consts<R>& K, R glm_fac, bool turb, R ax, R ay, R az,
                                                  R dt) {
        finish_update(q, K, glm_fac, turb, ax, ay, az, dt);
    }
};

// March (spike_mhd.cu:65-223, 257-299): per direction a full MonCen slope and a transverse-free
// 1-D Hancock half step of the cell, faces at mh -+ s/2 (or the Julia-form PPM edge plus the
// predictor shift), floors rho >= smallr and p >= smallp, HLL with GLM cleaning; the update is
// u - dt/dx sum_d (F_hi - F_lo) and psi *= glm_fac.  The unsplit tile's update
// u + dt/dx ((F_xlo - F_xhi) + (F_ylo - F_yhi) + (F_zlo - F_zhi)) is the same IEEE value, since
// negation is exact and round-to-nearest is sign-symmetric.
template <class R> struct MarchCell {
    Q9<R> m0, s, mh;   // cell primitives; slope and 1-D predictor of the direction being prepared
};
template <class R, int RECON> struct MarchScheme {
    using Cell = MarchCell<R>;
    static constexpr bool kRecord = false;
    static constexpr bool kEarlyOld = std::is_same<R, float>::value;   // 9.31 -> 9.15 ms at 512^3
    static __device__ __forceinline__ R prim_floor(const Consts<R>& K) { return K.smallp; }
    static __device__ __forceinline__ void recon(const R* PR, int PN, int, int c, int s0, int, int, const Consts<R>&, R,
                                                 Cell& r) {
        r.m0 = Lay<R>::get(PR + (size_t)s0 * 9 * PN, PN, c);
    }
    template <int D>
    static __device__ __forceinline__ void neighbours(const R* PR, int PN, int PW, int c, int s0, int sm, int sp,
                                                      Q9<R>& L, Q9<R>& Rr) {
        const R* PL = PR + (size_t)(D == 2 ? sm : s0) * 9 * PN;
        const R* PP = PR + (size_t)(D == 2 ? sp : s0) * 9 * PN;
        const int cl = D == 0 ? c - 1 : (D == 1 ? c - PW : c), cr = D == 0 ? c + 1 : (D == 1 ? c + PW : c);
        L = Lay<R>::get(PL, PN, cl);
        Rr = Lay<R>::get(PP, PN, cr);
    }
    template <int D>
    static __device__ __forceinline__ void prep(Cell& r, const R* PR, int PN, int PW, int c, int s0, int sm, int sp,
                                                const Consts<R>& K, R dtdx) {
        Q9<R> L, Rr;
        neighbours<D>(PR, PN, PW, c, s0, sm, sp, L, Rr);
        r.s = full_slope(L, r.m0, Rr);
        r.mh = hanc1d<D>(r.m0, r.s, dtdx, K.gamma, K.smallr, K.smallp);
    }
    template <int D, int SIGN>
    static __device__ __forceinline__ Q9<R> state(const Cell& r, const R* PR, int PN, int PW, int c, int s0, int sm,
                                                  int sp, const Consts<R>& K, int) {
        Q9<R> f;
        if (RECON == RECON_PPM) {
            Q9<R> L, Rr;
            neighbours<D>(PR, PN, PW, c, s0, sm, sp, L, Rr);
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
        return f;
    }
    template <int D>
    static __device__ __forceinline__ Q9<R> flux(const Q9<R>& L, const Q9<R>& Rr, const Consts<R>& K, R ch, bool) {
        Q9<R> Lr = rot_to<D>(L), Rrr = rot_to<D>(Rr);
        R bns, psis;
        glm_pair(Lr.v[5], Rrr.v[5], Lr.v[8], Rrr.v[8], ch, bns, psis);
        Lr.v[5] = bns;
        Rrr.v[5] = bns;
        return rot_from<D>(hll_x(Lr, Rrr, K.gamma, bns, psis, ch * ch * bns));
    }
    static __device__ __forceinline__ void finish(Q9<R>& q, const Consts<R>&, R glm_fac, bool, R, R, R, R) {
        q.v[8] = q.v[8] * glm_fac;
    }
};

// One tile (bx, by) x z-chunk bz of one box.  TOX, TOY > 0 fix the tile at compile time
// (constant shared-memory offsets); 0 = runtime tile.  Used by the single-box kernel (one tile per
// block) and by the ensemble kernel (a queue of tiles over many boxes).
// TMA: the kernel's A is a grid-constant parameter, so A.tmap can be handed to the TMA unit
// (the ensemble kernel copies its arguments from global memory and keeps the cp.async path).
template <class R, class S, int TOX, int TOY, bool OVERHANG = false, bool TMA = false>
__device__ __forceinline__ void scheme_tile(const UnsplitArgs<R>& A, const StepVals<R>& V, int bx, int by, int bz,
                                            unsigned char* smem_raw) {
    const int OX = TOX > 0 ? TOX : A.ox, OY = TOY > 0 ? TOY : A.oy;
    const int PW = OX + 4, PN = lay_n<R>((OX + 4) * (OY + 4));     // padded array lengths
    const int RW = OX + 2, RN = lay_n<R>((OX + 2) * (OY + 2));
    const int PNc = (OX + 4) * (OY + 4);                             // ring cells per plane
    const int SW = OX + 8, SN = (OX + 8) * (OY + 4);
    R* PR = reinterpret_cast<R*>(smem_raw);
    R* ST = PR + 27 * PN;
    R* SG = reinterpret_cast<R*>(smem_raw + unsplit_sg_offset<R>(OX, OY));
    double* red = reinterpret_cast<double*>(smem_raw + unsplit_red_offset<R>(OX, OY));
    // FP32 forcing tables of the tile: the x table of its columns (staged once) and the row table
    // of its rows for the plane written next (staged in the phase before that write-out)
    float* TS = reinterpret_cast<float*>(smem_raw + unsplit_red_offset<R>(OX, OY) + 40 * sizeof(double));
    float* BS = TS + 8 * OX;

    const int tid = threadIdx.x, NT = OX * OY;
    const int tx = tid % OX, ty = tid / OX;
    const int x0 = bx * OX, y0 = by * OY;
    const int z0 = bz * A.lz, z1 = min(z0 + A.lz, A.nz);
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const Consts<R> K = A.K;
    const R dtdx = V.dtdx, ch = V.ch;
    const bool turb = A.do_turb && A.btab != nullptr;
    const int nhelp = 2 * (OX + OY);
    // The extra work of a plane is packed into whole warps: halo reconstructions on the first
    // warps (phase R), boundary faces on the last ones (phase F).  The plane's staging copies skip
    // the helper warps and its primitive conversion skips the boundary-face warps, so both
    // phases' barrier tails shrink by that share (when at least one other warp remains).
    const int oxp = 32 * ((OX + 31) / 32);   // boundary faces: y on [0, OX), x on [oxp, oxp + OY)
    const int hwarp = 32 * ((nhelp + 31) / 32), bwarp = oxp + 32 * ((OY + 31) / 32);
    const int stg0 = NT - hwarp >= 32 ? hwarp : 0;                 // first staging thread
    const int nunst = NT - bwarp >= 32 ? NT - bwarp : NT;          // unstaging threads [0, nunst)

    // a tile whose staged region (x0-4 .. x0+OX+3, y0-2 .. y0+OY+1) lies inside the box stages its
    // planes by one TMA copy each (the tensor map addresses no periodic images); the others, and
    // every tile when the caller supplied no map, by per-thread cp.async
    bool tma = false;
    if constexpr (TMA) {
        tma = A.use_tma && !A.wait_test && x0 >= 4 && x0 + OX + 4 <= nx && y0 >= 2 && y0 + OY + 2 <= ny;
        // a TMA destination must be 128-byte aligned; otherwise stay on cp.async
        if ((unsigned)__cvta_generic_to_shared(SG) & 127u) tma = false;
    }
    const unsigned tma_bytes = (unsigned)(9 * SN * sizeof(R));

    // (the ensemble kernel, OVERHANG, keeps the tables in global memory: staged there it measured
    // 2 % slower, its 128 registers already spilling)
    if constexpr (std::is_same<R, float>::value && !OVERHANG) {
        if (A.trig8)
            for (int i = tid; i < 2 * OX; i += NT)
                reinterpret_cast<float4*>(TS)[i] = reinterpret_cast<const float4*>(A.trig8 + 8 * (size_t)x0)[i];
    }
    // prologue: primitives of planes z0-2, z0-1, z0
    uint64_t* mbar = reinterpret_cast<uint64_t*>(red + 32);
    for (int j = 0; j < 3; ++j) {
        stage_plane(SG, A.u, PNc, PW, SW, SN, x0, y0, z0 - 2 + j, nx, ny, nz, tid, NT);
        cp_async_wait_all();
        __syncthreads();
        unstage_plane(PR + mod3(z0 - 2 + j) * 9 * PN, SG, PN, PNc, PW, SW, SN, K, S::prim_floor(K), tid, NT);
        if (j == 2 && tid == 0) {
            mbar_init(mbar, tma ? 1u : (unsigned)NT);
            if (tma) fence_mbar_init();
        }
        __syncthreads();
    }

    // registers carried along the column: +z state of the previous plane, F_z at its lower face,
    // and this thread's own x/y face fluxes of the previous plane
    Q9<R> pPz, Fzlo, Fxh, Fyh;
#pragma unroll
    for (int v = 0; v < 9; ++v) { pPz.v[v] = R(0); Fzlo.v[v] = R(0); Fxh.v[v] = R(0); Fyh.v[v] = R(0); }
    R cmax = R(0), smax = R(0);   // exact maxima in R, widened to FP64 once per block
    double damp = 0.0;            // record mode: this thread's share of dL/d(forcing amplitude)
    // OVERHANG: a tile may overhang the box (an ensemble box narrower than a tile multiple); the
    // overhanging columns recompute the periodic images of cells at the start of the row, bit for
    // bit the same values, so their duplicate writes (and CFL maxima) are harmless
    int gx = x0 + tx, gy = y0 + ty;
    if (OVERHANG) {
        gx = gx < nx ? gx : gx - nx;
        gy = gy < ny ? gy : gy - ny;
    }
    const int cown = (tx + 2) + PW * (ty + 2);     // ring-local index of the owned cell
    const int rown = (tx + 1) + RW * (ty + 1);     // recon-local index of the owned cell
    const int ixh = (tx + 2) + RW * (ty + 1);      // slot of the +x neighbour
    const int iyh = (tx + 1) + RW * (ty + 2);      // slot of the +y neighbour
    unsigned phase = 0;

    // Two barriers per plane:
    //  [R] issue the load of plane kr+2; x/y divergence of plane kr-1 (own fluxes in registers,
    //      lower-face fluxes from the own slot); reconstruct plane kr; F_z at kr-1/2; write out kr-1
    //  [F] x/y Riemann solves of plane kr; convert plane kr+2 into the primitive ring
    for (int kr = z0 - 1; kr <= z1; ++kr) {
        const bool first = kr == z0 - 1, last = kr == z1;
        const bool load = kr + 2 <= z1 + 1;
        const int s0 = mod3(kr), sm = mod3(kr - 1), sp = mod3(kr + 1);
        if (load) {
            if constexpr (TMA) {
                if (tma) {
                    if (tid == 0) {
                        fence_proxy_async_smem();   // the previous plane's reads of SG come first
                        mbar_arrive_expect_tx(mbar, tma_bytes);
                        tma_load_4d(SG, &A.tmap, x0 - 4, y0 - 2, wrapi(kr + 2, nz), 0, mbar);
                    }
                }
            }
            if (!tma && !A.wait_test) {
                stage_plane(SG, A.u, PNc, PW, SW, SN, x0, y0, kr + 2, nx, ny, nz, tid >= stg0 ? tid - stg0 : PNc,
                            NT - stg0);
                mbar_arrive_cp_async(mbar);
            }
        }
        {
            Q9<R> XY;
            R fmx = R(0), fmy = R(0);   // lower-face mass fluxes, kept when A.fmass is set
            if (kr - 1 >= z0) {
                const Q9<R> Fxl = Lay<R>::get(ST + 1 * 9 * RN, RN, rown), Fyl = Lay<R>::get(ST + 3 * 9 * RN, RN, rown);
#pragma unroll
                for (int v = 0; v < 9; ++v) XY.v[v] = (Fxl.v[v] - Fxh.v[v]) + (Fyl.v[v] - Fyh.v[v]);
                if (A.fmass) {
                    fmx = Fxl.v[0];
                    fmy = Fyl.v[0];
                }
            }
            typename S::Cell r;
            S::recon(PR, PN, PW, cown, s0, sm, sp, K, dtdx, r);
            // record mode: interface state k of the own cell of plane kr, written only for a plane of
            // this chunk (z0 <= kr < z1)
            const size_t ncell = (size_t)nx * ny * nz;
            auto record = [&](int k, const Q9<R>& f) {
                if constexpr (S::kRecord) {
                    if (kr >= z0 && kr < z1)
                        rec_put(A, ncell, k, (size_t)gx + (size_t)nx * ((size_t)gy + (size_t)ny * (size_t)kr), f);
                }
            };
            if (!first && !last) {
                S::template prep<0>(r, PR, PN, PW, cown, s0, sm, sp, K, dtdx);
                {
                    const Q9<R> f = S::template state<0, +1>(r, PR, PN, PW, cown, s0, sm, sp, K, A.iflo);
                    Lay<R>::put(ST + 0 * 9 * RN, RN, rown, f);
                    record(0, f);
                }
                {
                    const Q9<R> f = S::template state<0, -1>(r, PR, PN, PW, cown, s0, sm, sp, K, A.iflo);
                    Lay<R>::put(ST + 1 * 9 * RN, RN, rown, f);
                    record(1, f);
                }
                S::template prep<1>(r, PR, PN, PW, cown, s0, sm, sp, K, dtdx);
                {
                    const Q9<R> f = S::template state<1, +1>(r, PR, PN, PW, cown, s0, sm, sp, K, A.iflo);
                    Lay<R>::put(ST + 2 * 9 * RN, RN, rown, f);
                    record(2, f);
                }
                {
                    const Q9<R> f = S::template state<1, -1>(r, PR, PN, PW, cown, s0, sm, sp, K, A.iflo);
                    Lay<R>::put(ST + 3 * 9 * RN, RN, rown, f);
                    record(3, f);
                }
            }
            S::template prep<2>(r, PR, PN, PW, cown, s0, sm, sp, K, dtdx);
            Q9<R> Pz = S::template state<2, +1>(r, PR, PN, PW, cown, s0, sm, sp, K, A.iflo);
            if (!first && !last) record(4, Pz);
            if (!first) {
                // the old state of the cell written out below, loaded before the z-face solve so that
                // the solve hides its latency (S::kEarlyOld), else at the write-out; the ensemble
                // kernel (OVERHANG) measured 7 % slower with the early load
                const bool wr = kr - 1 >= z0;
                const int kf = kr - 1;
                const size_t g = (size_t)gx + (size_t)nx * ((size_t)gy + (size_t)ny * (wr ? kf : 0));
                Q9<R> u0;
                if constexpr (S::kEarlyOld && !OVERHANG) {
#pragma unroll
                    for (int v = 0; v < 9; ++v) u0.v[v] = wr ? __ldg(A.u.p[v] + g) : R(0);
                }
                Q9<R> Mz = S::template state<2, -1>(r, PR, PN, PW, cown, s0, sm, sp, K, A.iflo);
                if (!last) record(5, Mz);
                Q9<R> Fzhi = S::template flux<2>(pPz, Mz, K, ch, A.use_llf != 0);
                if (wr) {
                    Q9<R> q;
#pragma unroll
                    for (int v = 0; v < 9; ++v)
                        q.v[v] = ((S::kEarlyOld && !OVERHANG) ? u0.v[v] : A.u.p[v][g]) + dtdx * (XY.v[v] + (Fzlo.v[v] - Fzhi.v[v]));
                    R ax = R(0), ay = R(0), az = R(0);
                    if (turb) {
                        if constexpr (std::is_same<R, float>::value && !OVERHANG) {
                            if (A.trig8) force_accel_f32(BS + 24 * ty, TS, tx, V.ramp, ax, ay, az);
                            else force_accel(A.btab + ((size_t)kf * ny + gy) * 24, A.trigx, nx, gx, V.ramp, ax, ay, az);
                        } else {
                            force_accel(A.btab + ((size_t)kf * ny + gy) * 24, A.trigx, nx, gx, V.ramp, ax, ay, az);
                        }
                    }
                    if constexpr (S::kRecord) {
                        // the epilogue's adjoint at the pre-epilogue state q; R1bar and the identity
                        // part of ubar, and this cell's share of dL/d(amplitude)
                        Q9<R> ob, rb;
#pragma unroll
                        for (int v = 0; v < 9; ++v) ob.v[v] = A.rec_ubn[(size_t)v * ncell + g];
                        R ab[3];
                        S::epilogue_adj(q, K, V.glm_fac, turb, ax, ay, az, V.dt, ob, rb, ab);
#pragma unroll
                        for (int v = 0; v < 9; ++v) {
                            A.rec_r1b[(size_t)v * ncell + g] = rb.v[v];
                            A.rec_ub[(size_t)v * ncell + g] = rb.v[v];
                        }
                        if (turb && A.rec_amp != R(0))
                            damp += ((double)ab[0] * ax + (double)ab[1] * ay + (double)ab[2] * az) / (double)A.rec_amp;
                    } else {
                        S::finish(q, K, V.glm_fac, turb, ax, ay, az, V.dt);
#pragma unroll
                        for (int v = 0; v < 9; ++v) A.o.p[v][g] = q.v[v];
                        if (A.fmass) {
                            A.fmass[g] = fmx;
                            A.fmass[ncell + g] = fmy;
                            A.fmass[2 * ncell + g] = Fzlo.v[0];
                        }
                        if (A.cfl_out) {
                            R ct, sg;
                            cfl_speeds(q, K, ct, sg);
                            cmax = fmax(cmax, ct);
                            smax = fmax(smax, sg);
                        }
                    }
                }
                Fzlo = Fzhi;
            }
            pPz = Pz;
        }
        if (!first && !last) {
            // halo reconstructions: only the one interface state each halo cell contributes
            for (int h = tid; h < nhelp; h += NT) {
                int rc, cc, which;
                if (h < OY) { rc = 0 + RW * (h + 1); cc = 1 + PW * (h + 2); which = 0; }
                else if (h < 2 * OY) { int f = h - OY; rc = (OX + 1) + RW * (f + 1); cc = (OX + 2) + PW * (f + 2); which = 1; }
                else if (h < 2 * OY + OX) { int f = h - 2 * OY; rc = (f + 1); cc = (f + 2) + PW * 1; which = 2; }
                else { int f = h - 2 * OY - OX; rc = (f + 1) + RW * (OY + 1); cc = (f + 2) + PW * (OY + 2); which = 3; }
                typename S::Cell r;
                S::recon(PR, PN, PW, cc, s0, sm, sp, K, dtdx, r);
                Q9<R> f;
                if (which < 2) {
                    S::template prep<0>(r, PR, PN, PW, cc, s0, sm, sp, K, dtdx);
                    if (which == 0) f = S::template state<0, +1>(r, PR, PN, PW, cc, s0, sm, sp, K, A.iflo);
                    else f = S::template state<0, -1>(r, PR, PN, PW, cc, s0, sm, sp, K, A.iflo);
                } else {
                    S::template prep<1>(r, PR, PN, PW, cc, s0, sm, sp, K, dtdx);
                    if (which == 2) f = S::template state<1, +1>(r, PR, PN, PW, cc, s0, sm, sp, K, A.iflo);
                    else f = S::template state<1, -1>(r, PR, PN, PW, cc, s0, sm, sp, K, A.iflo);
                }
                Lay<R>::put(ST + which * 9 * RN, RN, rc, f);
            }
        }
        __syncthreads();
        if (!first && !last) {
            // own faces at x+1/2 and y+1/2: flux kept in registers and written over the right state,
            // where the neighbour reads it as its lower-face flux
            Fxh = S::template flux<0>(Lay<R>::get(ST + 0 * 9 * RN, RN, rown), Lay<R>::get(ST + 1 * 9 * RN, RN, ixh), K, ch,
                                      A.use_llf != 0);
            Lay<R>::put(ST + 1 * 9 * RN, RN, ixh, Fxh);
            Fyh = S::template flux<1>(Lay<R>::get(ST + 2 * 9 * RN, RN, rown), Lay<R>::get(ST + 3 * 9 * RN, RN, iyh), K, ch,
                                      A.use_llf != 0);
            Lay<R>::put(ST + 3 * 9 * RN, RN, iyh, Fyh);
            for (int h = NT - 1 - tid; h < oxp + OY; h += NT) {
                // boundary faces on the low x and low y side of the tile, taken by the last threads:
                // the y faces first, the x faces from the next warp boundary, so that no warp runs
                // both solver paths one after the other
                if (h < OX) {
                    const int il = (h + 1), ir = (h + 1) + RW;
                    Q9<R> F = S::template flux<1>(Lay<R>::get(ST + 2 * 9 * RN, RN, il), Lay<R>::get(ST + 3 * 9 * RN, RN, ir), K,
                                                  ch, A.use_llf != 0);
                    Lay<R>::put(ST + 3 * 9 * RN, RN, ir, F);
                } else if (h >= oxp) {
                    const int f = h - oxp;
                    const int il = 0 + RW * (f + 1), ir = 1 + RW * (f + 1);
                    Q9<R> F = S::template flux<0>(Lay<R>::get(ST + 0 * 9 * RN, RN, il), Lay<R>::get(ST + 1 * 9 * RN, RN, ir), K,
                                                  ch, A.use_llf != 0);
                    Lay<R>::put(ST + 1 * 9 * RN, RN, ir, F);
                }
            }
        }
        // the forcing row table of the tile's rows for plane kr, written out in the next phase R
        if constexpr (std::is_same<R, float>::value && !OVERHANG) {
            if (turb && A.trig8 && kr >= z0 && kr < z1)
                for (int i = tid; i < 6 * OY; i += NT)
                    reinterpret_cast<float4*>(BS)[i] =
                        reinterpret_cast<const float4*>(A.btab + ((size_t)kr * ny + y0) * 24)[i];
        }
        if (load) {
            mbar_wait(mbar, phase, A.err, A.wait_cycles);
            phase ^= 1u;
            unstage_plane(PR + mod3(kr + 2) * 9 * PN, SG, PN, PNc, PW, SW, SN, K, S::prim_floor(K), tid < nunst ? tid : PNc,
                          nunst);
        }
        __syncthreads();
    }
    if (tid == 0) mbar_inval(mbar);
    if constexpr (S::kRecord) {
        // block sum of the amplitude partials (red[0..31]; the mbarrier word sits at red[32])
        double v = damp;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((tid & 31) == 0) red[tid >> 5] = v;
        __syncthreads();
        if (tid < 32) {
            double x = tid < (NT + 31) / 32 ? red[tid] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (tid == 0 && x != 0.0 && A.rec_damp) atomicAdd(A.rec_damp, x);
        }
        __syncthreads();   // red is free again for a following tile of the same block
    } else {
        (void)damp;
    }
    if (A.cfl_out) {
        block_max_atomic((double)cmax, A.cfl_out, red);
        __syncthreads();
        block_max_atomic((double)smax, A.cfl_out + 1, red);
    }
}

template <class R, int RECON, int RIEM, int TOX, int TOY, bool OVERHANG = false, bool TMA = false>
__device__ __forceinline__ void unsplit_tile(const UnsplitArgs<R>& A, const StepVals<R>& V, int bx, int by, int bz,
                                             unsigned char* smem_raw) {
    scheme_tile<R, UnsplitScheme<R, RECON, RIEM>, TOX, TOY, OVERHANG, TMA>(A, V, bx, by, bz, smem_raw);
}

// A tile = (box, bx, by, bz) work item of the ensemble kernel.
struct EnsItem { int box, bx, by, bz; };

// Persistent ensemble step: each block takes work items from a global queue (one atomic per
// item) until the queue is drained; every box has its own arguments, step values and CFL slot.
template <class R, int RECON, int RIEM, int TOX, int TOY, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) ensemble_kernel(const UnsplitArgs<R>* __restrict__ boxes,
                                                              const EnsItem* __restrict__ items, int nitems,
                                                              unsigned* queue) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ int item_s;
    for (;;) {
        if (threadIdx.x == 0) item_s = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int it = item_s;
        __syncthreads();
        if (it >= nitems) break;
        const EnsItem w = items[it];
        const UnsplitArgs<R> A = boxes[w.box];
        unsplit_tile<R, RECON, RIEM, TOX, TOY, true>(A, step_vals(A), w.bx, w.by, w.bz, smem_raw);
        __syncthreads();
    }
}

template <class R, int RECON, int RIEM, int MAXT, int MINB, int TOX = 0, int TOY = 0>
__global__ void __launch_bounds__(MAXT, MINB) unsplit_kernel(const __grid_constant__ UnsplitArgs<R> A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsplit_tile<R, RECON, RIEM, TOX, TOY, false, true>(A, step_vals(A), blockIdx.x, blockIdx.y,
                                                                                 blockIdx.z, smem_raw);
}

// Tiled march step (the scheme behind march_run_dev); RECON is RECON_MC or RECON_PPM.
template <class R, int RECON, int MAXT, int MINB, int TOX = 0, int TOY = 0>
__global__ void __launch_bounds__(MAXT, MINB) march_tile_kernel(const __grid_constant__ UnsplitArgs<R> A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    scheme_tile<R, MarchScheme<R, RECON>, TOX, TOY, false, true>(
        A, step_vals(A), blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

}  // namespace gmt
