// gmt_adjoint.cuh -- per-cell passes of the discrete adjoint of the unsplit GLM step (PLM-MC /
// minmod, any Riemann solver, GLM, void floor, psi damping, forcing kick) with dt frozen.
//
// Given the step's input state u and the adjoint ubar' = dL/du' of its output, the passes form
// ubar = (du'/du)^T ubar' and dL/d(forcing amplitude) of the step (periodic wrap):
//   1 faces    forward reconstruction of every cell -> its 6 interface states FS
//   2 fluxes   forward Riemann solve at every cell's +x,+y,+z face -> FL
//   3 update   r1 = u + dt/dx * sum(F_lo - F_hi); adjoint of the epilogue (floor, psi damping,
//              forcing kick) -> R1bar; ubar = R1bar (identity part); kick amplitude partials
//   4 riemann  Fbar = dt/dx (R1bar[c+d] - R1bar[c]) -> adjoint interface states FSbar
//   5 recon    faces -> (mh, m0, slopes) bars; the Hancock block mh = c2p(p2c(m0) - dt/2dx sum_d
//              [F_d(m0+s_d) - F_d(m0-s_d)]) by one vector-Jacobian product per flux; limiter
//              derivatives split each slope bar onto the three cells of its stencil
//   6 gather   qbar(c) = own + neighbours' slope terms; ubar += (dq/du)^T qbar
// The Riemann solves (HLLD, HLL), the directional fluxes, prim2cons and cons2prim have hand-written
// reverse sweeps (gmt_riemann_adj.cuh); the exact-speed LLF paths and the update epilogue are
// differentiated by running the forward physics functions on forward-mode duals seeded in chunks
// (the seeds are selects on a chunk offset, so no tangent is ever indexed dynamically).  The
// limiter derivative, the face/revert structure, the Hancock sum and the flux-difference identity
// are written out.  At a limiter kink, an HLLD fan switch, a floor or an interface-state revert the
// derivative of the branch that was taken is used (a subgradient).
//
// Every pass is a host-device function of one cell, so the same code also runs on the host.
#pragma once
#include "gmt_dual.cuh"
#include "gmt_internal.h"
#include "gmt_riemann_adj.cuh"

namespace gmt {


constexpr int NCH = 3;   // tangents per dual pass

template <class R> GMT_HD void q9_add(Q9<R>& a, const Q9<R>& b, R s = R(1)) {
#pragma unroll
    for (int v = 0; v < 9; ++v) a.v[v] += s * b.v[v];
}
template <class R> GMT_HD Q9<R> q9_zero() {
    Q9<R> a;
#pragma unroll
    for (int v = 0; v < 9; ++v) a.v[v] = R(0);
    return a;
}

template <class R> struct Idx {
    int nx, ny, nz;
    size_t n;
    // periodic index of (x, y, z), each coordinate at most one cell outside the box
    GMT_HD static int wrap1(int i, int m) { return i < 0 ? i + m : (i >= m ? i - m : i); }
    GMT_HD size_t at(int x, int y, int z) const {
        return (size_t)wrap1(x, nx) + (size_t)nx * ((size_t)wrap1(y, ny) + (size_t)ny * wrap1(z, nz));
    }
};

template <class R> GMT_HD Q9<R> load_u(const CPlanes<R>& u, size_t c) {
    Q9<R> q;
#pragma unroll
    for (int v = 0; v < 9; ++v) q.v[v] = u.p[v][c];
    return q;
}

// the six interface states of one cell (recon_prims + face_state of the forward kernel)
template <class R> struct CellRec {
    Q9<R> m0, uh, mh, s[3], L[3], Rr[3];
    bool hrev;        // the predictor reverted to m0
    bool bad[6];      // the face state reverted to m0
};

// the seven cells of the reconstruction stencil of (x, y, z), in the order c, x-, x+, y-, y+, z-, z+
template <class R> GMT_HD void stencil7(const Idx<R>& I, int x, int y, int z, size_t (&cs)[7]) {
    cs[0] = I.at(x, y, z);
    cs[1] = I.at(x - 1, y, z);
    cs[2] = I.at(x + 1, y, z);
    cs[3] = I.at(x, y - 1, z);
    cs[4] = I.at(x, y + 1, z);
    cs[5] = I.at(x, y, z - 1);
    cs[6] = I.at(x, y, z + 1);
}

// reconstruction of one cell from the conserved states of its stencil; U(j) returns stencil cell j
template <class R, class U>
GMT_HD void cell_rec_from(const U& u, const Consts<R>& K, R dtdx, bool mm, CellRec<R>& r) {
    r.m0 = cons2prim(u(0), K.gamma, K.smallr, K.pfl);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        r.L[d] = cons2prim(u(1 + 2 * d), K.gamma, K.smallr, K.pfl);
        r.Rr[d] = cons2prim(u(2 + 2 * d), K.gamma, K.smallr, K.pfl);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            R dl = r.m0.v[v] - r.L[d].v[v], dr = r.Rr[d].v[v] - r.m0.v[v];
            r.s[d].v[v] = mm ? R(0.5) * minmod(dl, dr) : R(0.5) * moncen(dl, dr);
        }
    r.uh = hancock(r.m0, r.s[0], r.s[1], r.s[2], dtdx, K.gamma);
    r.mh = cons2prim(r.uh, K.gamma, K.smallr, K.pfl);
    r.hrev = r.mh.v[0] <= K.smallr || r.mh.v[4] <= K.pfl;
    if (r.hrev) r.mh = r.m0;
}

// stencil source reading the conserved planes
template <class R> struct StencilGlobal {
    const CPlanes<R>& u;
    size_t cs[7];
    GMT_HD Q9<R> operator()(int j) const { return load_u(u, cs[j]); }
};

template <class R>
GMT_HD void cell_rec(const CPlanes<R>& u, const Idx<R>& I, int x, int y, int z, const Consts<R>& K,
                                         R dtdx, int, bool mm, CellRec<R>& r) {
    StencilGlobal<R> src{u, {}};
    stencil7(I, x, y, z, src.cs);
    cell_rec_from(src, K, dtdx, mm, r);
}

template <class R>
GMT_HD Q9<R> rec_face(const CellRec<R>& r, int k, const Consts<R>& K, int iflo, bool& bad) {
    const int d = k >> 1;
    Q9<R> f = padd(r.mh, r.s[d], (k & 1) ? R(-1) : R(1));
    bad = iflo && (f.v[0] < K.smallr || f.v[4] < K.pfl);
    return bad ? r.m0 : f;
}

// derivatives of the half slope g(dl, dr) (MonCen or minmod) w.r.t. dl and dr
template <class R> GMT_HD void slope_deriv(R dl, R dr, bool mm, R& gl, R& gr) {
    gl = R(0);
    gr = R(0);
    if (dl * dr <= R(0)) return;
    if (mm) {
        if (rabs(dl) < rabs(dr)) gl = R(0.5); else gr = R(0.5);
        return;
    }
    R dc = R(0.5) * (dl + dr);
    R m2 = R(2) * rmin(rabs(dl), rabs(dr));
    if (m2 <= rabs(dc)) {                          // rmin(m2, |dc|) picks m2
        if (rabs(dl) <= rabs(dr)) gl = R(1); else gr = R(1);
    } else {
        gl = R(0.25);
        gr = R(0.25);
    }
}

// the cyclic rotation that makes direction d the x normal, and its inverse, for a runtime d
// (rot_to / rot_from of the physics, glmmhd_turb.jl:118-138): a Jacobian evaluated in the x
// frame serves all three directions, J_d^T v = rot_from_d(J_x^T rot_to_d(v))
template <class R> GMT_HD Q9<R> rot_to_d(const Q9<R>& q, int d) {
    if (d == 0) return q;
    Q9<R> r;
    if (d == 1) {
        r.v[0] = q.v[0]; r.v[1] = q.v[2]; r.v[2] = q.v[3]; r.v[3] = q.v[1]; r.v[4] = q.v[4];
        r.v[5] = q.v[6]; r.v[6] = q.v[7]; r.v[7] = q.v[5]; r.v[8] = q.v[8];
    } else {
        r.v[0] = q.v[0]; r.v[1] = q.v[3]; r.v[2] = q.v[1]; r.v[3] = q.v[2]; r.v[4] = q.v[4];
        r.v[5] = q.v[7]; r.v[6] = q.v[5]; r.v[7] = q.v[6]; r.v[8] = q.v[8];
    }
    return r;
}
template <class R> GMT_HD Q9<R> rot_from_d(const Q9<R>& f, int d) {
    if (d == 0) return f;
    Q9<R> r;
    if (d == 1) {
        r.v[0] = f.v[0]; r.v[1] = f.v[3]; r.v[2] = f.v[1]; r.v[3] = f.v[2]; r.v[4] = f.v[4];
        r.v[5] = f.v[7]; r.v[6] = f.v[5]; r.v[7] = f.v[6]; r.v[8] = f.v[8];
    } else {
        r.v[0] = f.v[0]; r.v[1] = f.v[2]; r.v[2] = f.v[3]; r.v[3] = f.v[1]; r.v[4] = f.v[4];
        r.v[5] = f.v[6]; r.v[6] = f.v[7]; r.v[7] = f.v[5]; r.v[8] = f.v[8];
    }
    return r;
}

// the flux at a face of direction d: riemann_glm<d> = rot_from_d . riemann_glm<0> . rot_to_d
template <int RIEM, class R>
GMT_HD Q9<R> riemann_dir(const Q9<R>& L, const Q9<R>& Rr, int d, const Consts<R>& K, R ch, bool use_llf) {
    return rot_from_d(riemann_glm<0, RIEM>(rot_to_d(L, d), rot_to_d(Rr, d), K, ch, use_llf), d);
}

// Lbar, Rbar = J^T Fbar of the Riemann solve at a face of direction d (18 inputs in chunks of NCH,
// evaluated in the x frame)
// DUALS: whether the exact-speed LLF paths can occur (LLF-bound solver, use_llf, or the density /
// pressure LLF switch); without them every face takes the hand-written reverse sweep and the
// dual-number code is not compiled in
template <int RIEM, bool DUALS, class R>
GMT_HD void riemann_adj(const Q9<R>& L, const Q9<R>& Rr, const Q9<R>& Fb, int d, const Consts<R>& K, R ch,
                        bool use_llf, Q9<R>& Lb, Q9<R>& Rb) {
    using DD = Dual<R, NCH>;
    const Q9<R> Lx = rot_to_d(L, d), Rx = rot_to_d(Rr, d), Fbx = rot_to_d(Fb, d);
    Q9<R> Lbx = q9_zero<R>(), Rbx = q9_zero<R>();
    // hand-written reverse sweep (HLLD, HLL); the exact-speed LLF paths go through dual numbers
    if (riemann_x_adj<RIEM>(Lx, Rx, Fbx, K, ch, use_llf, Lbx, Rbx) || !DUALS) {
        Lb = rot_from_d(Lbx, d);
        Rb = rot_from_d(Rbx, d);
        return;
    }
    const Consts<DD> KD = dual_consts<R, NCH>(K);
#pragma unroll 1
    for (int c0 = 0; c0 < 18; c0 += NCH) {
        Q9<DD> Ld, Rd;
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            Ld.v[v] = DD(Lx.v[v]);
            Rd.v[v] = DD(Rx.v[v]);
#pragma unroll
            for (int j = 0; j < NCH; ++j) {
                Ld.v[v].d[j] = (c0 + j == v) ? R(1) : R(0);
                Rd.v[v].d[j] = (c0 + j == 9 + v) ? R(1) : R(0);
            }
        }
        Q9<DD> F = riemann_glm<0, RIEM>(Ld, Rd, KD, DD(ch), use_llf);
#pragma unroll
        for (int j = 0; j < NCH; ++j) {
            R acc = R(0);
#pragma unroll
            for (int v = 0; v < 9; ++v) acc += Fbx.v[v] * F.v[v].d[j];
#pragma unroll
            for (int v = 0; v < 9; ++v) {
                if (c0 + j == v) Lbx.v[v] = acc;
                if (c0 + j == 9 + v) Rbx.v[v] = acc;
            }
        }
    }
    Lb = rot_from_d(Lbx, d);
    Rb = rot_from_d(Rbx, d);
}

template <class R> GMT_HD void cell_xyz(const AdjArgs<R>& A, size_t c, int& x, int& y, int& z) {
    if (c <= 0xffffffffu) {   // 32-bit divisions for every linear index below 2^32
        const unsigned cc = (unsigned)c, nx = (unsigned)A.nx, ny = (unsigned)A.ny;
        const unsigned q = cc / nx;
        x = (int)(cc - q * nx);
        y = (int)(q % ny);
        z = (int)(q / ny);
        return;
    }
    x = (int)(c % A.nx);
    y = (int)((c / A.nx) % A.ny);
    z = (int)(c / ((size_t)A.nx * A.ny));
}
template <class R> GMT_HD Idx<R> idx_of(const AdjArgs<R>& A) {
    return Idx<R>{A.nx, A.ny, A.nz, (size_t)A.nx * A.ny * A.nz};
}
template <class R> GMT_HD Q9<R> fs_get(const R* FS, size_t n, size_t c, int k) {
    Q9<R> q;
#pragma unroll
    for (int v = 0; v < 9; ++v) q.v[v] = FS[(size_t)(k * 9 + v) * n + c];
    return q;
}

// pass 1: the six interface states of cell c
template <class R> GMT_HD void adj_faces_store(const AdjArgs<R>& A, size_t n, size_t c, const CellRec<R>& r) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        bool bad;
        Q9<R> f = rec_face(r, k, A.K, A.iflo, bad);
#pragma unroll
        for (int v = 0; v < 9; ++v) A.FS[(size_t)(k * 9 + v) * n + c] = f.v[v];
    }
}
template <class R> GMT_HD void adj_faces_cell(const AdjArgs<R>& A, size_t c) {
    const Idx<R> I = idx_of(A);
    int x, y, z;
    cell_xyz(A, c, x, y, z);
    CellRec<R> r;
    cell_rec(A.u, I, x, y, z, A.K, A.dtdx, A.iflo, A.recon == RECON_MINMOD, r);
    adj_faces_store(A, I.n, c, r);
}

// pass 2: the fluxes at the +x, +y, +z faces of cell c
template <int RIEM, class R> GMT_HD void adj_flux_cell(const AdjArgs<R>& A, size_t c) {
    const Idx<R> I = idx_of(A);
    const bool ul = A.use_llf != 0;
    int x, y, z;
    cell_xyz(A, c, x, y, z);
#pragma unroll 1
    for (int d = 0; d < 3; ++d) {
        const size_t cp = d == 0 ? I.at(x + 1, y, z) : (d == 1 ? I.at(x, y + 1, z) : I.at(x, y, z + 1));
        const Q9<R> F = riemann_dir<RIEM>(fs_get(A.FS, I.n, c, 2 * d), fs_get(A.FS, I.n, cp, 2 * d + 1), d, A.K, A.ch, ul);
#pragma unroll
        for (int v = 0; v < 9; ++v) A.FL[(size_t)(9 * d + v) * I.n + c] = F.v[v];
    }
}

// pass 3: the update and its epilogue; returns this cell's part of dL/d(amplitude)
template <class R> GMT_HD double adj_update_cell(const AdjArgs<R>& A, size_t c) {
    const Idx<R> I = idx_of(A);
    const bool turb = A.do_turb && A.btab != nullptr;
    int x, y, z;
    cell_xyz(A, c, x, y, z);
    const size_t cxm = I.at(x - 1, y, z), cym = I.at(x, y - 1, z), czm = I.at(x, y, z - 1);
    Q9<R> r1;
#pragma unroll
    for (int v = 0; v < 9; ++v) {
        R fxl = A.FL[(size_t)v * I.n + cxm], fxh = A.FL[(size_t)v * I.n + c];
        R fyl = A.FL[(size_t)(9 + v) * I.n + cym], fyh = A.FL[(size_t)(9 + v) * I.n + c];
        R fzl = A.FL[(size_t)(18 + v) * I.n + czm], fzh = A.FL[(size_t)(18 + v) * I.n + c];
        r1.v[v] = A.u.p[v][c] + A.dtdx * (((fxl - fxh) + (fyl - fyh)) + (fzl - fzh));
    }
    R a3[3] = {R(0), R(0), R(0)};
    if (turb) force_accel(A.btab + ((size_t)z * A.ny + y) * 24, A.trigx, A.nx, x, A.ramp, a3[0], a3[1], a3[2]);
    const Q9<R> ob = load_u(A.ubn, c);
    Q9<R> rb;
    R abar[3];
    finish_update_adj(r1, A.K, A.glm_fac, turb, a3[0], a3[1], a3[2], A.dt, ob, rb, abar);
#pragma unroll
    for (int v = 0; v < 9; ++v) {
        A.R1b[(size_t)v * I.n + c] = rb.v[v];
        A.ub.p[v][c] = rb.v[v];
    }
    if (turb && A.amp != R(0))
        return ((double)abar[0] * a3[0] + (double)abar[1] * a3[1] + (double)abar[2] * a3[2]) / (double)A.amp;
    return 0.0;
}

// the same epilogue adjoint by forward-mode dual numbers over the 12 inputs (9 state, 3
// accelerations); the reference the hand-written sweep is checked against
template <class R>
GMT_HD void finish_update_adj_dual(const Q9<R>& r1, const Consts<R>& K, R glm_fac, bool turb, const R a3[3], R dt,
                                   const Q9<R>& ob, Q9<R>& rb, R abar[3]) {
    constexpr int NU = 6;
    using DD = Dual<R, NU>;
    const Consts<DD> KD = dual_consts<R, NU>(K);
#pragma unroll
    for (int c0 = 0; c0 < 12; c0 += NU) {   // two passes: the 9 state inputs, then the 3 accelerations
        Q9<DD> q;
        DD ad[3];
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            q.v[v] = DD(r1.v[v]);
#pragma unroll
            for (int j = 0; j < NU; ++j) q.v[v].d[j] = (c0 + j == v) ? R(1) : R(0);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            ad[i] = DD(a3[i]);
#pragma unroll
            for (int j = 0; j < NU; ++j) ad[i].d[j] = (c0 + j == 9 + i) ? R(1) : R(0);
        }
        finish_update(q, KD, DD(glm_fac), turb, ad[0], ad[1], ad[2], DD(dt));
#pragma unroll
        for (int j = 0; j < NU; ++j) {
            R acc = R(0);
#pragma unroll
            for (int v = 0; v < 9; ++v) acc += ob.v[v] * q.v[v].d[j];
            const int i = c0 + j;
            if (i < 9) rb.v[i] = acc;
            else if (i < 12) abar[i - 9] = acc;
        }
    }
}

// pass 4: adjoint of the Riemann solves at the +x, +y, +z faces of cell c
// one face c | cp of direction d: its two interface states and the flux adjoint -> FSbar
template <int RIEM, bool DUALS, class R>
GMT_HD void adj_riemann_face(const AdjArgs<R>& A, size_t n, size_t c, size_t cp, int d, const Q9<R>& L,
                             const Q9<R>& Rr, const Q9<R>& Fb, bool ul) {
    Q9<R> Lb, Rb;
    riemann_adj<RIEM, DUALS>(L, Rr, Fb, d, A.K, A.ch, ul, Lb, Rb);
#pragma unroll
    for (int v = 0; v < 9; ++v) {
        A.FSb[(size_t)((2 * d) * 9 + v) * n + c] = Lb.v[v];
        A.FSb[(size_t)((2 * d + 1) * 9 + v) * n + cp] = Rb.v[v];
    }
}
template <int RIEM, bool DUALS, class R> GMT_HD void adj_riemann_cell(const AdjArgs<R>& A, size_t c) {
    const Idx<R> I = idx_of(A);
    const bool ul = A.use_llf != 0;
    int x, y, z;
    cell_xyz(A, c, x, y, z);
#pragma unroll 1
    for (int d = 0; d < 3; ++d) {
        const size_t cp = d == 0 ? I.at(x + 1, y, z) : (d == 1 ? I.at(x, y + 1, z) : I.at(x, y, z + 1));
        Q9<R> Fb;
#pragma unroll
        for (int v = 0; v < 9; ++v) Fb.v[v] = A.dtdx * (A.R1b[(size_t)v * I.n + cp] - A.R1b[(size_t)v * I.n + c]);
        adj_riemann_face<RIEM, DUALS>(A, I.n, c, cp, d, fs_get(A.FS, I.n, c, 2 * d), fs_get(A.FS, I.n, cp, 2 * d + 1),
                                      Fb, ul);
    }
}

// pass 5: adjoint of the reconstruction of cell c
// FSbar source reading the scratch planes
template <class R> struct FaceBarGlobal {
    const R* FSb;
    size_t n, c;
    GMT_HD Q9<R> operator()(int k) const { return fs_get(FSb, n, c, k); }
    GMT_HD void release() const {}
};

// the reconstruction adjoint of cell c from its reconstruction r and the adjoints of its six
// interface states (FB(k), k = +x, -x, +y, -y, +z, -z); FB(k) is called once per face, in face order,
// and FB.release() once all six have been read
template <class R, class FB>
GMT_HD void adj_recon_core(const AdjArgs<R>& A, size_t n, size_t c, const CellRec<R>& r, const FB& fbar) {
    const bool mm = A.recon == RECON_MINMOD;
    // faces: f = mh +- s_d, or m0 where reverted
    Q9<R> m0b = q9_zero<R>(), mhb = q9_zero<R>(), sb[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) sb[d] = q9_zero<R>();
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        bool bad;
        (void)rec_face(r, k, A.K, A.iflo, bad);
        const Q9<R> fb = fbar(k);
        if (bad) {
            q9_add(m0b, fb);
        } else {
            q9_add(mhb, fb);
            q9_add(sb[k >> 1], fb, (k & 1) ? R(-1) : R(1));
        }
    }
    fbar.release();   // every interface-state adjoint has been read
    // predictor: mh = c2p(p2c(m0) - h sum_d [F_d(m0 + s_d) - F_d(m0 - s_d)]), or m0 if reverted
    if (r.hrev) {
        q9_add(m0b, mhb);
    } else {
        Q9<R> uhb = q9_zero<R>();
        cons2prim_adj(r.uh, A.K.gamma, A.K.smallr, A.K.pfl, mhb, uhb);
        prim2cons_adj(r.m0, A.K.gamma, uhb, m0b);
        Q9<R> Fb;
        const R h = R(0.5) * A.dtdx;
#pragma unroll
        for (int v = 0; v < 9; ++v) Fb.v[v] = -h * uhb.v[v];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            // dir_flux<d> = rot_from_d . phys_flux_x . rot_to_d
            const Q9<R> Fbx = rot_to_d(Fb, d);
            Q9<R> jpx = q9_zero<R>(), jmx = q9_zero<R>();
            phys_flux_x_adj(rot_to_d(padd(r.m0, r.s[d], R(1)), d), A.K.gamma, Fbx, jpx);
            phys_flux_x_adj(rot_to_d(padd(r.m0, r.s[d], R(-1)), d), A.K.gamma, Fbx, jmx);
            const Q9<R> jp = rot_from_d(jpx, d), jm = rot_from_d(jmx, d);
#pragma unroll
            for (int v = 0; v < 9; ++v) {
                m0b.v[v] += jp.v[v] - jm.v[v];
                sb[d].v[v] += jp.v[v] + jm.v[v];
            }
        }
    }
    // limiter: s_d = g(m0 - L_d, R_d - m0); m0 gets (gl - gr) sbar, the neighbours -gl sbar, +gr sbar
#pragma unroll
    for (int v = 0; v < 9; ++v) {
        R own = m0b.v[v];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            R gl, gr;
            slope_deriv(r.m0.v[v] - r.L[d].v[v], r.Rr[d].v[v] - r.m0.v[v], mm, gl, gr);
            const R Ad = sb[d].v[v] * gl, Bd = sb[d].v[v] * gr;
            own += Ad - Bd;
            A.QB[(size_t)(9 + 9 * d + v) * n + c] = Ad;
            A.QB[(size_t)(36 + 9 * d + v) * n + c] = Bd;
        }
        A.QB[(size_t)v * n + c] = own;
    }
}
template <class R> GMT_HD void adj_recon_cell(const AdjArgs<R>& A, size_t c) {
    const Idx<R> I = idx_of(A);
    int x, y, z;
    cell_xyz(A, c, x, y, z);
    CellRec<R> r;
    cell_rec(A.u, I, x, y, z, A.K, A.dtdx, A.iflo, A.recon == RECON_MINMOD, r);
    adj_recon_core(A, I.n, c, r, FaceBarGlobal<R>{A.FSb, I.n, c});
}

// pass 6: gather the primitive adjoint of cell c and map it through cons2prim
template <class R> GMT_HD void adj_gather_cell(const AdjArgs<R>& A, size_t c) {
    const Idx<R> I = idx_of(A);
    int x, y, z;
    cell_xyz(A, c, x, y, z);
    const size_t cp[3] = {I.at(x + 1, y, z), I.at(x, y + 1, z), I.at(x, y, z + 1)};
    const size_t cm[3] = {I.at(x - 1, y, z), I.at(x, y - 1, z), I.at(x, y, z - 1)};
    // all 63 scratch loads (and the 9 state loads) are issued before any use, so a thread keeps
    // them in flight together: the pass is bound by memory latency, not by arithmetic
    const R* __restrict__ QB = A.QB;
    R own[9], ap[27], bm[27];
#pragma unroll
    for (int v = 0; v < 9; ++v) own[v] = QB[(size_t)v * I.n + c];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            ap[9 * d + v] = QB[(size_t)(9 + 9 * d + v) * I.n + cp[d]];
            bm[9 * d + v] = QB[(size_t)(36 + 9 * d + v) * I.n + cm[d]];
        }
    const Q9<R> u0 = load_u(A.u, c);
    Q9<R> qb;
#pragma unroll
    for (int v = 0; v < 9; ++v) {
        R s = own[v];
#pragma unroll
        for (int d = 0; d < 3; ++d) s += -ap[9 * d + v] + bm[9 * d + v];
        qb.v[v] = s;
    }
    Q9<R> ubq = q9_zero<R>();
    cons2prim_adj(u0, A.K.gamma, A.K.smallr, A.K.pfl, qb, ubq);
#pragma unroll
    for (int v = 0; v < 9; ++v) A.ub.p[v][c] += ubq.v[v];
}

}  // namespace gmt
