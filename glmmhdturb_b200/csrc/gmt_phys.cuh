// gmt_phys.cuh -- device physics of the GLM-MHD step, templated on the real type.
//
// Ideal GLM-MHD in the x-normal frame with compile-time cyclic rotations, the MonCen/minmod
// limiters, the unsplit MUSCL-Hancock predictor, PPM edges, and the HLLD / HLL / LLF Riemann
// solvers with Dedner cleaning.  Every expression keeps the left-to-right order of the
// reference's Julia source so that a build without FMA contraction reproduces an IEEE
// evaluation of the same formulas bit for bit.
//
// Reference (GLMMHDTurb): glmmhd_turb.jl:68-354 (physics), :917-926 (PPM),
// march_bridge/cu/spike_mhd.cu:65-223 (1-D Hancock, full-slope MonCen).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define GMT_HD __host__ __device__ __forceinline__

namespace gmt {

template <class R> struct Q9 { R v[9]; };

template <class R> GMT_HD R rmax(R a, R b);
template <> GMT_HD float rmax(float a, float b) { return fmaxf(a, b); }
template <> GMT_HD double rmax(double a, double b) { return fmax(a, b); }
template <class R> GMT_HD R rmin(R a, R b);
template <> GMT_HD float rmin(float a, float b) { return fminf(a, b); }
template <> GMT_HD double rmin(double a, double b) { return fmin(a, b); }
template <class R> GMT_HD R rabs(R a);
template <> GMT_HD float rabs(float a) { return fabsf(a); }
template <> GMT_HD double rabs(double a) { return fabs(a); }
template <class R> GMT_HD R rsqrt_ieee(R a);
template <> GMT_HD float rsqrt_ieee(float a) { return sqrtf(a); }
template <> GMT_HD double rsqrt_ieee(double a) { return sqrt(a); }

// Physical constants of one step, in working precision.
template <class R> struct Consts {
    R gamma, smallr, pfl, smallc, smallp, llf_dmin, llf_pmin, turb_min_rho;
};

// cons2prim (glmmhd_turb.jl:68-77); `pf` is the pressure floor (pfl, or SMALLP for the march)
template <class R> GMT_HD Q9<R> cons2prim(const Q9<R>& c, R gamma, R smallr, R pf) {
    Q9<R> q;
    R rho = rmax(c.v[0], smallr);
    R ir = R(1) / rho;
    q.v[0] = rho;
    q.v[1] = c.v[1] * ir; q.v[2] = c.v[2] * ir; q.v[3] = c.v[3] * ir;
    R bx = c.v[5], by = c.v[6], bz = c.v[7];
    R ekin = R(0.5) * (c.v[1] * c.v[1] + c.v[2] * c.v[2] + c.v[3] * c.v[3]) * ir;
    R emag = R(0.5) * (bx * bx + by * by + bz * bz);
    q.v[4] = rmax((gamma - R(1)) * (c.v[4] - ekin - emag), pf);
    q.v[5] = bx; q.v[6] = by; q.v[7] = bz; q.v[8] = c.v[8];
    return q;
}

// prim2cons (glmmhd_turb.jl:79-86)
template <class R> GMT_HD Q9<R> prim2cons(const Q9<R>& q, R gamma) {
    Q9<R> c;
    R rho = q.v[0], vx = q.v[1], vy = q.v[2], vz = q.v[3], p = q.v[4];
    R bx = q.v[5], by = q.v[6], bz = q.v[7];
    R ekin = R(0.5) * rho * (vx * vx + vy * vy + vz * vz);
    R emag = R(0.5) * (bx * bx + by * by + bz * bz);
    c.v[0] = rho; c.v[1] = rho * vx; c.v[2] = rho * vy; c.v[3] = rho * vz;
    c.v[4] = p / (gamma - R(1)) + ekin + emag;
    c.v[5] = bx; c.v[6] = by; c.v[7] = bz; c.v[8] = q.v[8];
    return c;
}

// fast magnetosonic speed with normal field bn (glmmhd_turb.jl:89-95)
template <class R> GMT_HD R fast_speed(const Q9<R>& q, R gamma, R bn) {
    R rho = q.v[0];
    R c2 = gamma * q.v[4] / rho;
    R b2 = (q.v[5] * q.v[5] + q.v[6] * q.v[6] + q.v[7] * q.v[7]) / rho;
    R d2 = R(0.5) * (b2 + c2);
    return rsqrt_ieee(d2 + rsqrt_ieee(rmax(d2 * d2 - c2 * bn * bn / rho, R(0))));
}

// ideal-MHD x flux; F[Bx] and F[psi] are left 0 (glmmhd_turb.jl:98-115)
template <class R> GMT_HD Q9<R> phys_flux_x(const Q9<R>& q, R gamma) {
    Q9<R> f;
    R rho = q.v[0], vx = q.v[1], vy = q.v[2], vz = q.v[3], p = q.v[4];
    R bx = q.v[5], by = q.v[6], bz = q.v[7];
    R b2 = bx * bx + by * by + bz * bz;
    R ptot = p + R(0.5) * b2;
    R ekin = R(0.5) * rho * (vx * vx + vy * vy + vz * vz);
    R E = p / (gamma - R(1)) + ekin + R(0.5) * b2;
    R vdotb = vx * bx + vy * by + vz * bz;
    f.v[0] = rho * vx;
    f.v[1] = rho * vx * vx + ptot - bx * bx;
    f.v[2] = rho * vx * vy - bx * by;
    f.v[3] = rho * vx * vz - bx * bz;
    f.v[4] = (E + ptot) * vx - bx * vdotb;
    f.v[5] = R(0);
    f.v[6] = vx * by - vy * bx;
    f.v[7] = vx * bz - vz * bx;
    f.v[8] = R(0);
    return f;
}

// cyclic rotations (glmmhd_turb.jl:118-138); D is the sweep axis
template <int D, class R> GMT_HD Q9<R> rot_to(const Q9<R>& q) {
    if (D == 0) return q;
    Q9<R> r;
    r.v[0] = q.v[0]; r.v[4] = q.v[4]; r.v[8] = q.v[8];
    if (D == 1) {
        r.v[1] = q.v[2]; r.v[2] = q.v[3]; r.v[3] = q.v[1];
        r.v[5] = q.v[6]; r.v[6] = q.v[7]; r.v[7] = q.v[5];
    } else {
        r.v[1] = q.v[3]; r.v[2] = q.v[1]; r.v[3] = q.v[2];
        r.v[5] = q.v[7]; r.v[6] = q.v[5]; r.v[7] = q.v[6];
    }
    return r;
}
template <int D, class R> GMT_HD Q9<R> rot_from(const Q9<R>& f) {
    if (D == 0) return f;
    Q9<R> r;
    r.v[0] = f.v[0]; r.v[4] = f.v[4]; r.v[8] = f.v[8];
    if (D == 1) {
        r.v[1] = f.v[3]; r.v[2] = f.v[1]; r.v[3] = f.v[2];
        r.v[5] = f.v[7]; r.v[6] = f.v[5]; r.v[7] = f.v[6];
    } else {
        r.v[1] = f.v[2]; r.v[2] = f.v[3]; r.v[3] = f.v[1];
        r.v[5] = f.v[6]; r.v[6] = f.v[7]; r.v[7] = f.v[5];
    }
    return r;
}
template <int D, class R> GMT_HD Q9<R> dir_flux(const Q9<R>& q, R gamma) {
    return rot_from<D>(phys_flux_x(rot_to<D>(q), gamma));
}

// MonCen half-slope (glmmhd_turb.jl:145-155) and minmod half-slope (:300-303)
template <class R> GMT_HD R moncen(R dl, R dr) {
    R dc = R(0.5) * (dl + dr);
    R sgn = dc >= R(0) ? R(1) : R(-1);
    R val = sgn * rmin(R(2) * rmin(rabs(dl), rabs(dr)), rabs(dc));
    return dl * dr <= R(0) ? R(0) : val;
}
template <class R> GMT_HD R minmod(R a, R b) {
    return a * b <= R(0) ? R(0) : (rabs(a) < rabs(b) ? a : b);
}
// FP32 MonCen half slope with the scalings folded: 0.5*sgn(dc)*min(2 min(|dl|,|dr|), |dc|) =
// copysign(min(min(|dl|,|dr|), |dl+dr|/4), dl+dr); equal to moncen() up to the sign of zero.
GMT_HD float moncen_half_fast(float dl, float dr) {
    float a = dl + dr;
    float m = fminf(fminf(fabsf(dl), fabsf(dr)), 0.25f * fabsf(a));
    return dl * dr <= 0.f ? 0.f : copysignf(m, a);
}
template <bool MM, class R> GMT_HD R half_slope1(R dl, R dr) {
    return MM ? R(0.5) * minmod(dl, dr) : R(0.5) * moncen(dl, dr);
}
template <> GMT_HD float half_slope1<false, float>(float dl, float dr) { return moncen_half_fast(dl, dr); }
template <bool MM, class R> GMT_HD Q9<R> half_slope(const Q9<R>& L, const Q9<R>& M, const Q9<R>& Rr) {
    Q9<R> s;
#pragma unroll
    for (int i = 0; i < 9; ++i) s.v[i] = half_slope1<MM, R>(M.v[i] - L.v[i], Rr.v[i] - M.v[i]);
    return s;
}
// spike_mhd.cu:118-123 full-slope MonCen: sgn(dl)*min(|dc|, 2|dl|, 2|dr|), dc = (c-a)/2
template <class R> GMT_HD R full_mc(R a, R b, R c) {
    R dl = b - a, dr = c - b, dc = R(0.5) * (c - a);
    if (dl * dr <= R(0)) return R(0);
    R s = dl > R(0) ? R(1) : R(-1);
    return s * rmin(rabs(dc), rmin(R(2) * rabs(dl), R(2) * rabs(dr)));
}
template <class R> GMT_HD Q9<R> full_slope(const Q9<R>& a, const Q9<R>& b, const Q9<R>& c) {
    Q9<R> s;
#pragma unroll
    for (int i = 0; i < 9; ++i) s.v[i] = full_mc(a.v[i], b.v[i], c.v[i]);
    return s;
}
template <class R> GMT_HD Q9<R> padd(const Q9<R>& q, const Q9<R>& s, R a) {
    Q9<R> r;
#pragma unroll
    for (int i = 0; i < 9; ++i) r.v[i] = q.v[i] + a * s.v[i];
    return r;
}

// unsplit MUSCL-Hancock predictor (glmmhd_turb.jl:165-172)
template <class R>
GMT_HD Q9<R> hancock(const Q9<R>& m0, const Q9<R>& sx, const Q9<R>& sy, const Q9<R>& sz, R dtdx, R gamma) {
    Q9<R> u0 = prim2cons(m0, gamma);
    R h = R(0.5) * dtdx;
    Q9<R> fxp = dir_flux<0>(padd(m0, sx, R(1)), gamma);
    Q9<R> fxm = dir_flux<0>(padd(m0, sx, R(-1)), gamma);
    Q9<R> dx, dy;
#pragma unroll
    for (int i = 0; i < 9; ++i) dx.v[i] = fxp.v[i] - fxm.v[i];
    Q9<R> fyp = dir_flux<1>(padd(m0, sy, R(1)), gamma);
    Q9<R> fym = dir_flux<1>(padd(m0, sy, R(-1)), gamma);
#pragma unroll
    for (int i = 0; i < 9; ++i) dy.v[i] = fyp.v[i] - fym.v[i];
    Q9<R> fzp = dir_flux<2>(padd(m0, sz, R(1)), gamma);
    Q9<R> fzm = dir_flux<2>(padd(m0, sz, R(-1)), gamma);
    Q9<R> r;
#pragma unroll
    for (int i = 0; i < 9; ++i) r.v[i] = u0.v[i] - h * ((dx.v[i] + dy.v[i]) + (fzp.v[i] - fzm.v[i]));
    return r;
}

// transverse-free 1-D Hancock half step of a cell centre, full slope s (spike_mhd.cu:149-161)
template <int D, class R>
GMT_HD Q9<R> hanc1d(const Q9<R>& c0, const Q9<R>& s, R dtdx, R gamma, R smallr, R smallp) {
    Q9<R> FL = dir_flux<D>(padd(c0, s, R(-0.5)), gamma);
    Q9<R> FR = dir_flux<D>(padd(c0, s, R(0.5)), gamma);
    Q9<R> U = prim2cons(c0, gamma);
    R h = R(0.5) * dtdx;
#pragma unroll
    for (int v = 0; v < 9; ++v) U.v[v] = U.v[v] - h * (FR.v[v] - FL.v[v]);
    return cons2prim(U, gamma, smallr, smallp);
}

// PPM edges (glmmhd_turb.jl:917-926): exact parabola edge + CW84 monotonisation
template <class R> GMT_HD void ppm_edges(R qm, R q0, R qp, R& lo, R& hi) {
    R sl = R(0.25) * (qp - qm);
    R curve = (qm - R(2) * q0 + qp) / R(12);
    R ql = q0 - sl + curve, qr = q0 + sl + curve;
    R dq = qr - ql;
    R diff = (q0 - R(0.5) * (ql + qr)) * dq;
    if ((qr - q0) * (q0 - ql) <= R(0)) { lo = q0; hi = q0; }
    else if (diff > dq * dq / R(6)) { lo = R(3) * q0 - R(2) * qr; hi = qr; }
    else if (diff < -(dq * dq / R(6))) { lo = ql; hi = R(3) * q0 - R(2) * ql; }
    else { lo = ql; hi = qr; }
}
template <class R> GMT_HD bool spj(R a, R b, R c) {
    R hi = rmax(a, rmax(b, c));
    R lo = rmax(rmin(a, rmin(b, c)), R(1e-20));
    return hi / lo > R(2);
}

// ---------------------------------------------------------------------------------------
// Riemann solvers in the x-normal frame (inputs already rotated, floored, bn cleaned)
// ---------------------------------------------------------------------------------------
template <class R> GMT_HD void glm_pair(R bnL, R bnR, R psiL, R psiR, R ch, R& bns, R& psis) {
    bns = R(0.5) * (bnL + bnR) - R(0.5) * (psiR - psiL) / ch;
    psis = R(0.5) * (psiL + psiR) - R(0.5) * ch * (bnR - bnL);
}

template <bool BOUND, class R>
GMT_HD Q9<R> llf_x(const Q9<R>& L, const Q9<R>& Rr, R gamma, R ch, R fbn, R fpsi) {
    Q9<R> fL = phys_flux_x(L, gamma), fR = phys_flux_x(Rr, gamma);
    Q9<R> uL = prim2cons(L, gamma), uR = prim2cons(Rr, gamma);
    R sL, sR;
    if (BOUND) {  // fast_speed_bound (glmmhd_turb.jl:307-310)
        R irL = R(1) / L.v[0], irR = R(1) / Rr.v[0];
        sL = rabs(L.v[1]) + rsqrt_ieee((gamma * L.v[4] + L.v[5] * L.v[5] + L.v[6] * L.v[6] + L.v[7] * L.v[7]) * irL);
        sR = rabs(Rr.v[1]) + rsqrt_ieee((gamma * Rr.v[4] + Rr.v[5] * Rr.v[5] + Rr.v[6] * Rr.v[6] + Rr.v[7] * Rr.v[7]) * irR);
    } else {
        sL = rabs(L.v[1]) + fast_speed(L, gamma, L.v[5]);
        sR = rabs(Rr.v[1]) + fast_speed(Rr, gamma, Rr.v[5]);
    }
    R smax = rmax(rmax(sL, sR), ch);
    Q9<R> f;
#pragma unroll
    for (int i = 0; i < 9; ++i) f.v[i] = R(0.5) * (fL.v[i] + fR.v[i]) - R(0.5) * smax * (uR.v[i] - uL.v[i]);
    f.v[5] = fbn; f.v[8] = fpsi;
    return f;
}

template <class R> GMT_HD Q9<R> hll_x(const Q9<R>& L, const Q9<R>& Rr, R gamma, R bn, R fbn, R fpsi) {
    R cfL = fast_speed(L, gamma, bn), cfR = fast_speed(Rr, gamma, bn);
    R SL = rmin(rmin(L.v[1] - cfL, Rr.v[1] - cfR), R(0));
    R SR = rmax(rmax(L.v[1] + cfL, Rr.v[1] + cfR), R(0));
    Q9<R> fL = phys_flux_x(L, gamma), fR = phys_flux_x(Rr, gamma);
    Q9<R> uL = prim2cons(L, gamma), uR = prim2cons(Rr, gamma);
    R ihd = R(1) / (SR - SL);
    Q9<R> f;
#pragma unroll
    for (int i = 0; i < 9; ++i) f.v[i] = (SR * fL.v[i] - SL * fR.v[i] + SL * SR * (uR.v[i] - uL.v[i])) * ihd;
    f.v[5] = fbn; f.v[8] = fpsi;
    return f;
}

// Miyoshi & Kusano (2005) HLLD (glmmhd_turb.jl:193-272)
template <class R>
GMT_HD void hlld_star(R d, R u, R v, R w, R by, R bz, R S, R SM, R bn, R& vy, R& vz, R& byS, R& bzS) {
    R denK = d * (S - u) * (S - SM) - bn * bn;
    if (rabs(denK) < R(1e-12)) {
        vy = v; vz = w; byS = by; bzS = bz;
    } else {
        R fac = bn * (SM - u) / denK;
        vy = v - by * fac;
        vz = w - bz * fac;
        byS = by * (d * (S - u) * (S - u) - bn * bn) / denK;
        bzS = bz * (d * (S - u) * (S - u) - bn * bn) / denK;
    }
}

template <class R> GMT_HD Q9<R> hlld_x(const Q9<R>& L, const Q9<R>& Rr, R gamma, R bn, R fbn, R fpsi) {
    const R tiny = R(1e-12);
    R dL = L.v[0], uL = L.v[1], vL = L.v[2], wL = L.v[3], pL = L.v[4], byL = L.v[6], bzL = L.v[7];
    R dR = Rr.v[0], uR = Rr.v[1], vR = Rr.v[2], wR = Rr.v[3], pR = Rr.v[4], byR = Rr.v[6], bzR = Rr.v[7];
    R b2L = bn * bn + byL * byL + bzL * bzL;
    R b2R = bn * bn + byR * byR + bzR * bzR;
    R ptL = pL + R(0.5) * b2L;
    R ptR = pR + R(0.5) * b2R;
    R EL = pL / (gamma - R(1)) + R(0.5) * dL * (uL * uL + vL * vL + wL * wL) + R(0.5) * b2L;
    R ER = pR / (gamma - R(1)) + R(0.5) * dR * (uR * uR + vR * vR + wR * wR) + R(0.5) * b2R;
    R cfL = fast_speed(L, gamma, bn);
    R cfR = fast_speed(Rr, gamma, bn);
    R SL = rmin(rmin(uL, uR) - rmax(cfL, cfR), R(0));
    R SR = rmax(rmax(uL, uR) + rmax(cfL, cfR), R(0));
    R den = (SR - uR) * dR - (SL - uL) * dL;
    R SM = ((SR - uR) * dR * uR - (SL - uL) * dL * uL - ptR + ptL) / den;
    R pts = ((SR - uR) * dR * ptL - (SL - uL) * dL * ptR + dL * dR * (SR - uR) * (SL - uL) * (uR - uL)) / den;
    R dLs = rmax(dL * (SL - uL) / (SL - SM), tiny);
    R dRs = rmax(dR * (SR - uR) / (SR - SM), tiny);
    R sqdLs = rsqrt_ieee(dLs), sqdRs = rsqrt_ieee(dRs);
    R SLs = SM - rabs(bn) / sqdLs;
    R SRs = SM + rabs(bn) / sqdRs;
    Q9<R> f;
    // The flux of the sampled region only needs the states on its side of the fan.
    if (SLs >= R(0)) {
        // F = FL + SL*(UL* - UL)
        R vyLs, vzLs, byLs, bzLs;
        hlld_star(dL, uL, vL, wL, byL, bzL, SL, SM, bn, vyLs, vzLs, byLs, bzLs);
        R vdotbL = uL * bn + vL * byL + wL * bzL;
        R vdotbLs = SM * bn + vyLs * byLs + vzLs * bzLs;
        R ELs = ((SL - uL) * EL - ptL * uL + pts * SM + bn * (vdotbL - vdotbLs)) / (SL - SM);
        Q9<R> FL = phys_flux_x(Q9<R>{{dL, uL, vL, wL, pL, bn, byL, bzL, R(0)}}, gamma);
        R ULs[9] = {dLs, dLs * SM, dLs * vyLs, dLs * vzLs, ELs, bn, byLs, bzLs, R(0)};
        R UL[9] = {dL, dL * uL, dL * vL, dL * wL, EL, bn, byL, bzL, R(0)};
#pragma unroll
        for (int i = 0; i < 9; ++i) f.v[i] = FL.v[i] + SL * (ULs[i] - UL[i]);
    } else if (SRs < R(0)) {
        R vyRs, vzRs, byRs, bzRs;
        hlld_star(dR, uR, vR, wR, byR, bzR, SR, SM, bn, vyRs, vzRs, byRs, bzRs);
        R vdotbR = uR * bn + vR * byR + wR * bzR;
        R vdotbRs = SM * bn + vyRs * byRs + vzRs * bzRs;
        R ERs = ((SR - uR) * ER - ptR * uR + pts * SM + bn * (vdotbR - vdotbRs)) / (SR - SM);
        Q9<R> FR = phys_flux_x(Q9<R>{{dR, uR, vR, wR, pR, bn, byR, bzR, R(0)}}, gamma);
        R URs[9] = {dRs, dRs * SM, dRs * vyRs, dRs * vzRs, ERs, bn, byRs, bzRs, R(0)};
        R UR[9] = {dR, dR * uR, dR * vR, dR * wR, ER, bn, byR, bzR, R(0)};
#pragma unroll
        for (int i = 0; i < 9; ++i) f.v[i] = FR.v[i] + SR * (URs[i] - UR[i]);
    } else {
        // inner fan: both star states and the double-star state
        R vyLs, vzLs, byLs, bzLs, vyRs, vzRs, byRs, bzRs;
        hlld_star(dL, uL, vL, wL, byL, bzL, SL, SM, bn, vyLs, vzLs, byLs, bzLs);
        hlld_star(dR, uR, vR, wR, byR, bzR, SR, SM, bn, vyRs, vzRs, byRs, bzRs);
        R vdotbL = uL * bn + vL * byL + wL * bzL;
        R vdotbLs = SM * bn + vyLs * byLs + vzLs * bzLs;
        R ELs = ((SL - uL) * EL - ptL * uL + pts * SM + bn * (vdotbL - vdotbLs)) / (SL - SM);
        R vdotbR = uR * bn + vR * byR + wR * bzR;
        R vdotbRs = SM * bn + vyRs * byRs + vzRs * bzRs;
        R ERs = ((SR - uR) * ER - ptR * uR + pts * SM + bn * (vdotbR - vdotbRs)) / (SR - SM);
        R sgn = bn >= R(0) ? R(1) : R(-1);
        R invsum = R(1) / (sqdLs + sqdRs);
        R vyss = (sqdLs * vyLs + sqdRs * vyRs + (byRs - byLs) * sgn) * invsum;
        R vzss = (sqdLs * vzLs + sqdRs * vzRs + (bzRs - bzLs) * sgn) * invsum;
        R byss = (sqdLs * byRs + sqdRs * byLs + sqdLs * sqdRs * (vyRs - vyLs) * sgn) * invsum;
        R bzss = (sqdLs * bzRs + sqdRs * bzLs + sqdLs * sqdRs * (vzRs - vzLs) * sgn) * invsum;
        R vdotbss = SM * bn + vyss * byss + vzss * bzss;
        if (SM >= R(0)) {
            R ELss = ELs - sqdLs * (vdotbLs - vdotbss) * sgn;
            Q9<R> FL = phys_flux_x(Q9<R>{{dL, uL, vL, wL, pL, bn, byL, bzL, R(0)}}, gamma);
            R ULss[9] = {dLs, dLs * SM, dLs * vyss, dLs * vzss, ELss, bn, byss, bzss, R(0)};
            R ULs[9] = {dLs, dLs * SM, dLs * vyLs, dLs * vzLs, ELs, bn, byLs, bzLs, R(0)};
            R UL[9] = {dL, dL * uL, dL * vL, dL * wL, EL, bn, byL, bzL, R(0)};
#pragma unroll
            for (int i = 0; i < 9; ++i) f.v[i] = FL.v[i] + SLs * ULss[i] - (SLs - SL) * ULs[i] - SL * UL[i];
        } else {
            R ERss = ERs + sqdRs * (vdotbRs - vdotbss) * sgn;
            Q9<R> FR = phys_flux_x(Q9<R>{{dR, uR, vR, wR, pR, bn, byR, bzR, R(0)}}, gamma);
            R URss[9] = {dRs, dRs * SM, dRs * vyss, dRs * vzss, ERss, bn, byss, bzss, R(0)};
            R URs[9] = {dRs, dRs * SM, dRs * vyRs, dRs * vzRs, ERs, bn, byRs, bzRs, R(0)};
            R UR[9] = {dR, dR * uR, dR * vR, dR * wR, ER, bn, byR, bzR, R(0)};
#pragma unroll
            for (int i = 0; i < 9; ++i) f.v[i] = FR.v[i] + SRs * URss[i] - (SRs - SR) * URs[i] - SR * UR[i];
        }
    }
    f.v[5] = fbn; f.v[8] = fpsi;
    return f;
}

enum { RIEM_HLLD = 0, RIEM_HLL = 1, RIEM_LLF = 2, RIEM_LLF_BOUND = 3 };
enum { RECON_MC = 0, RECON_MINMOD = 1, RECON_PPM = 2 };

// GLM Riemann dispatch in direction D (glmmhd_turb.jl:275-292, 313-354).  RIEM_HLLD also
// covers the exact-speed LLF (use_llf) and the density/pressure LLF switch.
template <int D, int RIEM, class R>
GMT_HD Q9<R> riemann_glm(const Q9<R>& Lq, const Q9<R>& Rq, const Consts<R>& K, R ch, bool use_llf) {
    Q9<R> L = rot_to<D>(Lq), Rr = rot_to<D>(Rq);
    L.v[0] = rmax(L.v[0], K.smallr); L.v[4] = rmax(L.v[4], K.pfl);
    Rr.v[0] = rmax(Rr.v[0], K.smallr); Rr.v[4] = rmax(Rr.v[4], K.pfl);
    R bns, psis;
    glm_pair(L.v[5], Rr.v[5], L.v[8], Rr.v[8], ch, bns, psis);
    R fbn = psis, fpsi = ch * ch * bns;
    L.v[5] = bns; Rr.v[5] = bns;
    Q9<R> f;
    if (RIEM == RIEM_HLL) {
        f = hll_x(L, Rr, K.gamma, bns, fbn, fpsi);
    } else if (RIEM == RIEM_LLF_BOUND) {
        f = llf_x<true>(L, Rr, K.gamma, ch, fbn, fpsi);
    } else {
        bool uself = (K.llf_dmin > R(0) && rmin(L.v[0], Rr.v[0]) < K.llf_dmin) ||
                     (K.llf_pmin > R(0) && rmin(L.v[4], Rr.v[4]) < K.llf_pmin) || use_llf;
        if (uself) f = llf_x<false>(L, Rr, K.gamma, ch, fbn, fpsi);
        else f = hlld_x(L, Rr, K.gamma, bns, fbn, fpsi);
    }
    return rot_from<D>(f);
}

// Update epilogue: void floor, psi damping, forcing kick (glmmhd_turb.jl:447-475, tiled :849-858)
template <class R>
GMT_HD void finish_update(Q9<R>& r, const Consts<R>& K, R glm_fac, bool turb, R ax, R ay, R az, R dt) {
    if (r.v[0] < K.smallr) {
        R emag = R(0.5) * (r.v[5] * r.v[5] + r.v[6] * r.v[6] + r.v[7] * r.v[7]);
        r.v[0] = K.smallr; r.v[1] = R(0); r.v[2] = R(0); r.v[3] = R(0);
        r.v[4] = K.pfl / (K.gamma - R(1)) + emag;
    }
    r.v[8] = r.v[8] * glm_fac;
    if (turb && r.v[0] >= K.turb_min_rho) {
        R rhom = rmax(r.v[0], K.smallr);
        R sc2 = K.smallc * K.smallc;
        R rho = r.v[0];
        R e = r.v[4];
        R fl = rho * sc2;
        e = rmax(e - R(0.5) * r.v[1] * r.v[1] / rhom, fl);
        e = rmax(e - R(0.5) * r.v[2] * r.v[2] / rhom, fl);
        e = rmax(e - R(0.5) * r.v[3] * r.v[3] / rhom, fl);
        R m2 = r.v[1] + rhom * ax * dt;
        R m3 = r.v[2] + rhom * ay * dt;
        R m4 = r.v[3] + rhom * az * dt;
        e = rmax(e + R(0.5) * m2 * m2 / rhom, fl);
        e = rmax(e + R(0.5) * m3 * m3 / rhom, fl);
        e = rmax(e + R(0.5) * m4 * m4 / rhom, fl);
        r.v[1] = m2; r.v[2] = m3; r.v[3] = m4; r.v[4] = e;
    }
}

}  // namespace gmt
