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

#include <type_traits>

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
template <class R> GMT_HD R sqrt_r(R a);
template <> GMT_HD float sqrt_r(float a) { return sqrtf(a); }
template <> GMT_HD double sqrt_r(double a) { return sqrt(a); }

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
    return sqrt_r(d2 + sqrt_r(rmax(d2 * d2 - c2 * bn * bn / rho, R(0))));
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

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000) && defined(GMT_PACKED_F32)
// Packed FP32 pairs for the fast FP32 build on sm_100: one f32x2 FMA / add / multiply does the same
// operation on two states, here the m0+s and m0-s states whose flux difference the Hancock
// predictor needs.
struct F2 { float2 v; };
__device__ __forceinline__ F2 splat2(float a) { return {make_float2(a, a)}; }
__device__ __forceinline__ F2 add2(F2 a, F2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 mul2(F2 a, F2 b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }

// phys_flux_x of two states at once (F[Bx] = F[psi] = 0)
__device__ __forceinline__ void phys_flux_x2(const F2* q, F2 igm1, F2* f) {
    const F2 half = splat2(0.5f), m1 = splat2(-1.0f);
    const F2 rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4], bx = q[5], by = q[6], bz = q[7];
    const F2 b2 = fma2(bx, bx, fma2(by, by, mul2(bz, bz)));
    const F2 ptot = fma2(half, b2, p);
    const F2 vsq = fma2(vx, vx, fma2(vy, vy, mul2(vz, vz)));
    const F2 E = fma2(p, igm1, fma2(mul2(half, rho), vsq, mul2(half, b2)));
    const F2 vdotb = fma2(vx, bx, fma2(vy, by, mul2(vz, bz)));
    const F2 nbx = mul2(bx, m1);
    const F2 f0 = mul2(rho, vx);
    f[0] = f0;
    f[1] = fma2(f0, vx, fma2(nbx, bx, ptot));
    f[2] = fma2(f0, vy, mul2(nbx, by));
    f[3] = fma2(f0, vz, mul2(nbx, bz));
    f[4] = fma2(add2(E, ptot), vx, mul2(nbx, vdotb));
    f[6] = fma2(vx, by, mul2(nbx, vy));
    f[7] = fma2(vx, bz, mul2(nbx, vz));
}

// F_D(m0 + a s) - F_D(m0 - a s), the two fluxes evaluated as one packed pair
template <int D> __device__ __forceinline__ void flux_pair_diff(const Q9<float>& m0, const Q9<float>& s, F2 igm1,
                                                               float* d, float a = 1.0f) {
    // the two states m0 + a s and m0 - a s, each formed by one scalar FMA straight into its half of
    // the pair (the same single rounding as a packed FMA of splatted operands, without the copies)
    F2 q[9];
#pragma unroll
    for (int v = 0; v < 9; ++v) q[v] = {make_float2(fmaf(a, s.v[v], m0.v[v]), fmaf(-a, s.v[v], m0.v[v]))};
    // rotate so that D is the x normal (rot_to): the velocity and field triples cycle
    constexpr int i1 = D == 0 ? 1 : (D == 1 ? 2 : 3), i2 = D == 0 ? 2 : (D == 1 ? 3 : 1), i3 = D == 0 ? 3 : (D == 1 ? 1 : 2);
    F2 r[9] = {q[0], q[i1], q[i2], q[i3], q[4], q[i1 + 4], q[i2 + 4], q[i3 + 4], q[8]};
    F2 f[9];
    phys_flux_x2(r, igm1, f);
    float fd[9];
#pragma unroll
    for (int v = 0; v < 9; ++v) fd[v] = (v == 5 || v == 8) ? 0.0f : f[v].v.x - f[v].v.y;
    // rotate back (rot_from): component i1 of the state was placed at 1, and so on
    d[0] = fd[0]; d[4] = fd[4]; d[8] = 0.0f;
    d[i1] = fd[1]; d[i2] = fd[2]; d[i3] = fd[3];
    d[i1 + 4] = fd[5]; d[i2 + 4] = fd[6]; d[i3 + 4] = fd[7];
}

__device__ __forceinline__ Q9<float> hancock_packed(const Q9<float>& m0, const Q9<float>& sx, const Q9<float>& sy,
                                                    const Q9<float>& sz, float dtdx, float gamma) {
    const Q9<float> u0 = prim2cons(m0, gamma);
    const F2 igm1 = splat2(1.0f / (gamma - 1.0f));
    const float h = 0.5f * dtdx;
    float dx[9], dy[9], dz[9];
    flux_pair_diff<0>(m0, sx, igm1, dx);
    flux_pair_diff<1>(m0, sy, igm1, dy);
    flux_pair_diff<2>(m0, sz, igm1, dz);
    Q9<float> r;
#pragma unroll
    for (int i = 0; i < 9; ++i) r.v[i] = u0.v[i] - h * ((dx[i] + dy[i]) + dz[i]);
    return r;
}
#endif

// unsplit MUSCL-Hancock predictor (glmmhd_turb.jl:165-172)
template <class R>
GMT_HD Q9<R> hancock(const Q9<R>& m0, const Q9<R>& sx, const Q9<R>& sy, const Q9<R>& sz, R dtdx, R gamma) {
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000) && defined(GMT_PACKED_F32)
    if constexpr (std::is_same<R, float>::value) return hancock_packed(m0, sx, sy, sz, dtdx, gamma);
#endif
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
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000) && defined(GMT_PACKED_F32)
    if constexpr (std::is_same<R, float>::value) {
        float df[9];
        flux_pair_diff<D>(c0, s, splat2(1.0f / (gamma - 1.0f)), df, 0.5f);
        Q9<float> U = prim2cons(c0, gamma);
        const float h = 0.5f * dtdx;
#pragma unroll
        for (int v = 0; v < 9; ++v) U.v[v] = U.v[v] - h * df[v];
        return cons2prim(U, gamma, smallr, smallp);
    }
#endif
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
        sL = rabs(L.v[1]) + sqrt_r((gamma * L.v[4] + L.v[5] * L.v[5] + L.v[6] * L.v[6] + L.v[7] * L.v[7]) * irL);
        sR = rabs(Rr.v[1]) + sqrt_r((gamma * Rr.v[4] + Rr.v[5] * Rr.v[5] + Rr.v[6] * Rr.v[6] + Rr.v[7] * Rr.v[7]) * irR);
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

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000) && defined(GMT_PACKED_F32)
// FP32 HLLD for the fast build: the same Miyoshi-Kusano states, sampled with fewer operations.
//  - The sampled region lies on the side of the sign of SM in all four regions (SL* >= 0 implies
//    SM >= 0, SR* < 0 implies SM < 0), so one side's star state is formed, and the other side's only
//    for the double-star regions.
//  - Every region's flux equals the physical flux of its sampled state with normal velocity SM and
//    total pressure pT* (F_L + S_L (U*_L - U_L) = F(U*_L) and F*_L + S*_L (U**_L - U*_L) = F(U**_L)
//    hold exactly in exact arithmetic, S_L clamped or not, since the star states solve those jump
//    conditions; pT* = pT_L + rho_L (S_L - u_L)(SM - u_L) equals the symmetric form used here), so
//    the flux is one evaluation F(rho*, SM, v*, w*, B*, E*, pT*) instead of F_side + S (U* - U).
//    In the degenerate star branch (|denK| < 1e-12, where B_t vanishes) F(U*)[B_t] and the jump
//    form differ by B_t (SM - u), which is zero with B_t.
//  - The reciprocals of rho, of the HLL denominator and of S - SM are formed once.
__device__ __forceinline__ Q9<float> hlld_x_f32(const Q9<float>& L, const Q9<float>& Rr, float gamma, float bn,
                                               float fbn, float fpsi) {
    const float tiny = 1e-12f;
    const float igm1 = 1.0f / (gamma - 1.0f);
    const float dL = L.v[0], uL = L.v[1], vL = L.v[2], wL = L.v[3], pL = L.v[4], byL = L.v[6], bzL = L.v[7];
    const float dR = Rr.v[0], uR = Rr.v[1], vR = Rr.v[2], wR = Rr.v[3], pR = Rr.v[4], byR = Rr.v[6], bzR = Rr.v[7];
    const float bn2 = bn * bn;
    const float b2L = fmaf(byL, byL, fmaf(bzL, bzL, bn2)), b2R = fmaf(byR, byR, fmaf(bzR, bzR, bn2));
    const float ptL = fmaf(0.5f, b2L, pL), ptR = fmaf(0.5f, b2R, pR);
    const float irL = 1.0f / dL, irR = 1.0f / dR;
    // fast speeds with the common normal field (fast_speed)
    const float c2L = gamma * pL * irL, c2R = gamma * pR * irR;
    const float d2L = 0.5f * fmaf(b2L, irL, c2L), d2R = 0.5f * fmaf(b2R, irR, c2R);
    const float cfL = sqrtf(d2L + sqrtf(fmaxf(fmaf(d2L, d2L, -c2L * bn2 * irL), 0.0f)));
    const float cfR = sqrtf(d2R + sqrtf(fmaxf(fmaf(d2R, d2R, -c2R * bn2 * irR), 0.0f)));
    const float cmax = fmaxf(cfL, cfR);
    const float SL = fminf(fminf(uL, uR) - cmax, 0.0f);
    const float SR = fmaxf(fmaxf(uL, uR) + cmax, 0.0f);
    const float aL = (SL - uL) * dL, aR = (SR - uR) * dR;   // rho (S - u) of each side
    const float iden = 1.0f / (aR - aL);
    const float SM = (aR * uR - aL * uL - ptR + ptL) * iden;
    const float pts = (aR * ptL - aL * ptR + aR * aL * (uR - uL)) * iden;

    // the sampled side s (L when SM >= 0) and its star state
    const bool lside = SM >= 0.0f;
    const float sig = lside ? -1.0f : 1.0f;   // S*_s = SM + sig |bn| / sqrt(rho*_s)
    const float d = lside ? dL : dR, u = lside ? uL : uR, v = lside ? vL : vR, w = lside ? wL : wR;
    const float by = lside ? byL : byR, bz = lside ? bzL : bzR, pt = lside ? ptL : ptR;
    const float E = fmaf(lside ? pL : pR, igm1, fmaf(0.5f * d, fmaf(u, u, fmaf(v, v, w * w)), 0.5f * (lside ? b2L : b2R)));
    const float S = lside ? SL : SR, a = lside ? aL : aR;
    const float isM = 1.0f / (S - SM);
    const float ds = fmaxf(a * isM, tiny);
    const float rs = rsqrtf(ds);
    const float Ss = fmaf(sig * fabsf(bn), rs, SM);
    float vys, vzs, bys, bzs;
    {
        const float denK = a * (S - SM) - bn2;
        const float ik = 1.0f / denK;
        const float fac = bn * (SM - u) * ik;
        const float t = (a * (S - u) - bn2) * ik;
        const bool degen = fabsf(denK) < tiny;
        vys = degen ? v : v - by * fac;
        vzs = degen ? w : w - bz * fac;
        bys = degen ? by : by * t;
        bzs = degen ? bz : bz * t;
    }
    const float vdotb = u * bn + v * by + w * bz;
    float vdotbs = SM * bn + vys * bys + vzs * bzs;
    float Es = ((S - u) * E - pt * u + pts * SM + bn * (vdotb - vdotbs)) * isM;
    // double-star regions: SL* < 0 <= SM or SM < 0 <= SR*
    if (lside ? Ss < 0.0f : Ss >= 0.0f) {
        const float od = lside ? dR : dL, ou = lside ? uR : uL, ov = lside ? vR : vL, ow = lside ? wR : wL;
        const float oby = lside ? byR : byL, obz = lside ? bzR : bzL, oS = lside ? SR : SL, oa = lside ? aR : aL;
        const float odsr = fmaxf(oa / (oS - SM), tiny);
        float ovy, ovz, oby_s, obz_s;
        {
            const float denK = oa * (oS - SM) - bn2;
            const float ik = 1.0f / denK;
            const float fac = bn * (SM - ou) * ik;
            const float t = (oa * (oS - ou) - bn2) * ik;
            const bool degen = fabsf(denK) < tiny;
            ovy = degen ? ov : ov - oby * fac;
            ovz = degen ? ow : ow - obz * fac;
            oby_s = degen ? oby : oby * t;
            obz_s = degen ? obz : obz * t;
        }
        const float sq = ds * rs, osq = sqrtf(odsr);
        // sgn(bn) times +1 when s = L, -1 when s = R (the averages are antisymmetric in L, R)
        const float sg = (bn >= 0.0f ? 1.0f : -1.0f) * (lside ? 1.0f : -1.0f);
        const float invsum = 1.0f / (sq + osq);
        const float vyss = (sq * vys + osq * ovy + (oby_s - bys) * sg) * invsum;
        const float vzss = (sq * vzs + osq * ovz + (obz_s - bzs) * sg) * invsum;
        const float sqq = sq * osq;
        const float byss = (sq * oby_s + osq * bys + sqq * (ovy - vys) * sg) * invsum;
        const float bzss = (sq * obz_s + osq * bzs + sqq * (ovz - vzs) * sg) * invsum;
        const float vdotbss = SM * bn + vyss * byss + vzss * bzss;
        Es = Es - sq * (vdotbs - vdotbss) * sg;
        vys = vyss; vzs = vzss; bys = byss; bzs = bzss; vdotbs = vdotbss;
    }
    // the physical flux of the sampled state (rho*_s, SM, v, B, E, pT*)
    const float m = ds * SM;
    Q9<float> f;
    f.v[0] = m;
    f.v[1] = fmaf(m, SM, pts - bn2);
    f.v[2] = fmaf(m, vys, -bn * bys);
    f.v[3] = fmaf(m, vzs, -bn * bzs);
    f.v[4] = fmaf(Es + pts, SM, -bn * vdotbs);
    f.v[5] = fbn;
    f.v[6] = fmaf(bys, SM, -bn * vys);
    f.v[7] = fmaf(bzs, SM, -bn * vzs);
    f.v[8] = fpsi;
    return f;
}
#endif

template <class R> GMT_HD Q9<R> hlld_x(const Q9<R>& L, const Q9<R>& Rr, R gamma, R bn, R fbn, R fpsi) {
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000) && defined(GMT_PACKED_F32)
    if constexpr (std::is_same<R, float>::value) return hlld_x_f32(L, Rr, gamma, bn, fbn, fpsi);
#endif
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
    R sqdLs = sqrt_r(dLs), sqdRs = sqrt_r(dRs);
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

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000) && defined(GMT_PACKED_F32)
// Packed FP32 HLL: the two sides of the face as one f32x2 pair (fast speeds, fluxes, conserved
// states); same expressions as hll_x.  (A packed HLLD measured no faster: its fan branches use one
// side at a time.)
__device__ __forceinline__ F2 pair2(float a, float b) { return {make_float2(a, b)}; }
__device__ __forceinline__ F2 rcp2(F2 a) { return pair2(1.0f / a.v.x, 1.0f / a.v.y); }
__device__ __forceinline__ F2 sqrt2(F2 a) { return pair2(sqrtf(a.v.x), sqrtf(a.v.y)); }
__device__ __forceinline__ F2 max2(F2 a, F2 b) { return pair2(fmaxf(a.v.x, b.v.x), fmaxf(a.v.y, b.v.y)); }

// fast speeds of the two sides with the common normal field bn
__device__ __forceinline__ F2 fast_speed2(const F2* q, F2 gamma, F2 bn) {
    const F2 ir = rcp2(q[0]);
    const F2 c2 = mul2(mul2(gamma, q[4]), ir);
    const F2 b2 = mul2(fma2(q[5], q[5], fma2(q[6], q[6], mul2(q[7], q[7]))), ir);
    const F2 d2 = mul2(splat2(0.5f), add2(b2, c2));
    const F2 disc = max2(fma2(d2, d2, mul2(mul2(mul2(c2, bn), bn), mul2(ir, splat2(-1.0f)))), splat2(0.0f));
    return sqrt2(add2(d2, sqrt2(disc)));
}

__device__ __forceinline__ void prim2cons2(const F2* q, F2 igm1, F2* c) {
    const F2 half = splat2(0.5f);
    const F2 rho = q[0], vx = q[1], vy = q[2], vz = q[3];
    const F2 ekin = mul2(mul2(half, rho), fma2(vx, vx, fma2(vy, vy, mul2(vz, vz))));
    const F2 emag = mul2(half, fma2(q[5], q[5], fma2(q[6], q[6], mul2(q[7], q[7]))));
    c[0] = rho; c[1] = mul2(rho, vx); c[2] = mul2(rho, vy); c[3] = mul2(rho, vz);
    c[4] = fma2(q[4], igm1, add2(ekin, emag));
    c[5] = q[5]; c[6] = q[6]; c[7] = q[7]; c[8] = q[8];
}

__device__ __forceinline__ Q9<float> hll_x_packed(const Q9<float>& L, const Q9<float>& Rr, float gamma, float bn,
                                                 float fbn, float fpsi) {
    F2 q[9];
#pragma unroll
    for (int v = 0; v < 9; ++v) q[v] = pair2(L.v[v], Rr.v[v]);
    const F2 igm1 = splat2(1.0f / (gamma - 1.0f));
    const F2 cf = fast_speed2(q, splat2(gamma), splat2(bn));
    const float SL = fminf(fminf(L.v[1] - cf.v.x, Rr.v[1] - cf.v.y), 0.0f);
    const float SR = fmaxf(fmaxf(L.v[1] + cf.v.x, Rr.v[1] + cf.v.y), 0.0f);
    F2 fl[9], u[9];
    phys_flux_x2(q, igm1, fl);
    prim2cons2(q, igm1, u);
    const float ihd = 1.0f / (SR - SL);
    // f = (SR fL - SL fR + SL SR (uR - uL)) / (SR - SL): as a pair (SR fL, -SL fR) + ...
    const F2 w = pair2(SR * ihd, -SL * ihd);
    const F2 wu = pair2(-SL * SR * ihd, SL * SR * ihd);
    Q9<float> f;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        if (i == 5 || i == 8) continue;
        const F2 t = fma2(u[i], wu, mul2(fl[i], w));
        f.v[i] = t.v.x + t.v.y;
    }
    f.v[5] = fbn; f.v[8] = fpsi;
    return f;
}

#endif

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
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000) && defined(GMT_PACKED_F32)
        if constexpr (std::is_same<R, float>::value) f = hll_x_packed(L, Rr, K.gamma, bns, fbn, fpsi);
        else
#endif
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
