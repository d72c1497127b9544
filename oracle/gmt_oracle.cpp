// gmt_oracle.cpp -- CPU oracle for the GLM-MHD / CT-MHD time step.
//
// TEST INFRASTRUCTURE ONLY (see gmt_oracle.h).  A plain restatement of the
// reference algorithm, written for readability and for bit-stable FP64:
// compile with -ffp-contract=off and without fast-math so every expression is
// evaluated in the source order given here, which follows the reference's
// Julia expressions left to right.
//
// Reference map (paths relative to the GLMMHDTurb project root):
//   cons2prim / prim2cons ........ glmmhd_turb.jl:68-86
//   fast_speed ................... glmmhd_turb.jl:89-95
//   phys_flux_x / rotations ...... glmmhd_turb.jl:98-138
//   moncen / prim_slope .......... glmmhd_turb.jl:145-155
//   hancock (unsplit) ............ glmmhd_turb.jl:165-172
//   glm_pair ..................... glmmhd_turb.jl:175-179
//   llf_x / hlld_x / riemann ..... glmmhd_turb.jl:182-292
//   minmod / lean LLF bound ...... glmmhd_turb.jl:300-333
//   hll_x / riemann_hll .......... glmmhd_turb.jl:335-354
//   recon / flux / update ........ glmmhd_turb.jl:378-480 (+ iflo 618, tiled update 841-861)
//   PPM (ppm_mono, ppm_edges, spj) glmmhd_turb.jl:917-926, stage 2 952-975
//   ctot / compute_dt ............ glmmhd_turb.jl:1963-1978
//   diagnostics .................. glmmhd_turb.jl:1996-2018
//   Orszag-Tang IC ............... glmmhd_turb.jl:2021-2036
//   march (1-D Hancock, HLL) ..... march_bridge/cu/spike_mhd.cu:65-223, 257-299
//   CT ........................... ct_mhd.jl:15-194, march_bridge/cu/spike_ctm.cu:95-298
//   OU forcing (replaced) ........ glmmhd_turb.jl:2094-2113 (projection), 457-475 (kick)
#include "gmt_oracle.h"

#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <class R> using V9 = std::array<R, 9>;
template <class R> using V8 = std::array<R, 8>;

static int g_threads = 0;
static int nthreads() {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

// Branch counters: how often each guarded branch of the reference fired since the last reset
// (ORC_CNT_* in gmt_oracle.h).  A fixture that claims to exercise a branch asserts its count > 0.
// Counting is off unless a caller switches it on, so the timed baseline pays one branch per site.
static std::atomic<int> g_count_on{0};
static std::atomic<long long> g_cnt[ORC_CNT_N];
static inline void count(int i) {
    if (g_count_on.load(std::memory_order_relaxed)) g_cnt[i].fetch_add(1, std::memory_order_relaxed);
}

// IEEE maxNum/minNum, the same semantics as CUDA fmax/fmin and Julia's @fastmath max/min
template <class R> static inline R rmax(R a, R b) { return std::fmax(a, b); }
template <class R> static inline R rmin(R a, R b) { return std::fmin(a, b); }
template <class R> static inline R osqrt(R a) { return std::sqrt(a); }
template <class R> static inline R oabs(R a) { return std::fabs(a); }
template <class R> static inline void set_tangent(R&, const double*) {}

// Forward-mode tangents: a value and up to ORC_JVP_MAXDIR directional derivatives, for the JVP
// entry point (the ForwardDiff counterpart of the reference's CPU step).  Every operation
// evaluates its value exactly as the double code does; comparisons, max/min and |x| act on the
// value, so the tangents follow the branch the value takes (at a kink, the derivative of the
// branch taken).
constexpr int NT = ORC_JVP_MAXDIR;
struct Tan {
    double v;
    double d[NT];
    Tan() : v(0) { for (int i = 0; i < NT; ++i) d[i] = 0; }
    Tan(double x) : v(x) { for (int i = 0; i < NT; ++i) d[i] = 0; }
};
static inline Tan operator+(const Tan& a, const Tan& b) {
    Tan r(a.v + b.v);
    for (int i = 0; i < NT; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
static inline Tan operator-(const Tan& a, const Tan& b) {
    Tan r(a.v - b.v);
    for (int i = 0; i < NT; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
static inline Tan operator-(const Tan& a) {
    Tan r(-a.v);
    for (int i = 0; i < NT; ++i) r.d[i] = -a.d[i];
    return r;
}
static inline Tan operator*(const Tan& a, const Tan& b) {
    Tan r(a.v * b.v);
    for (int i = 0; i < NT; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
static inline Tan operator/(const Tan& a, const Tan& b) {
    Tan r(a.v / b.v);
    for (int i = 0; i < NT; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
    return r;
}
static inline bool operator<(const Tan& a, const Tan& b) { return a.v < b.v; }
static inline bool operator<=(const Tan& a, const Tan& b) { return a.v <= b.v; }
static inline bool operator>(const Tan& a, const Tan& b) { return a.v > b.v; }
static inline bool operator>=(const Tan& a, const Tan& b) { return a.v >= b.v; }
static inline Tan rmax(const Tan& a, const Tan& b) { return a.v >= b.v ? a : b; }
static inline Tan rmin(const Tan& a, const Tan& b) { return a.v <= b.v ? a : b; }
static inline Tan osqrt(const Tan& a) {
    Tan r(std::sqrt(a.v));
    const double s = r.v > 0 ? 0.5 / r.v : 0.0;
    for (int i = 0; i < NT; ++i) r.d[i] = a.d[i] * s;
    return r;
}
static inline Tan oabs(const Tan& a) { return a.v >= 0 ? a : -a; }
static inline void set_tangent(Tan& x, const double* t) { for (int i = 0; i < NT; ++i) x.d[i] = t[i]; }

// ------------------------------------------------------------------------------------------
// Parameters converted to the working precision once per call.
// ------------------------------------------------------------------------------------------
template <class R> struct Phys {
    R gamma, smallr, smallc, pfl, smallp, llf_dmin, llf_pmin, turb_min_rho;
    int recon, riemann, iflo, emf, halfslope;
    explicit Phys(const orc_params* p) {
        gamma = (R)p->gamma; smallr = (R)p->smallr; smallc = (R)p->smallc;
        // pfloor(p) = smallr*smallc^2/gamma (glmmhd_turb.jl:55), evaluated in R
        pfl = smallr * (smallc * smallc) / gamma;
        smallp = (R)p->smallp;
        llf_dmin = (R)p->llf_dmin; llf_pmin = (R)p->llf_pmin; turb_min_rho = (R)p->turb_min_rho;
        recon = p->recon; riemann = p->riemann; iflo = p->iflo; emf = p->emf;
        halfslope = p->ct_halfslope;
    }
};

// ------------------------------------------------------------------------------------------
// Device-physics restatement (glmmhd_turb.jl:68-354)
// ------------------------------------------------------------------------------------------
template <class R> static inline V9<R> cons2prim(const V9<R>& c, R gamma, R smallr, R pfl) {
    R rho = rmax(c[0], smallr);
    R ir = R(1) / rho;
    R vx = c[1] * ir, vy = c[2] * ir, vz = c[3] * ir;
    R bx = c[5], by = c[6], bz = c[7];
    R ekin = R(0.5) * (c[1] * c[1] + c[2] * c[2] + c[3] * c[3]) * ir;
    R emag = R(0.5) * (bx * bx + by * by + bz * bz);
    R p = rmax((gamma - R(1)) * (c[4] - ekin - emag), pfl);
    return {rho, vx, vy, vz, p, bx, by, bz, c[8]};
}

template <class R> static inline V9<R> prim2cons(const V9<R>& q, R gamma) {
    R rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4];
    R bx = q[5], by = q[6], bz = q[7];
    R ekin = R(0.5) * rho * (vx * vx + vy * vy + vz * vz);
    R emag = R(0.5) * (bx * bx + by * by + bz * bz);
    R E = p / (gamma - R(1)) + ekin + emag;
    return {rho, rho * vx, rho * vy, rho * vz, E, bx, by, bz, q[8]};
}

template <class R> static inline R fast_speed(const V9<R>& q, R gamma, R bn) {
    R rho = q[0];
    R c2 = gamma * q[4] / rho;
    R b2 = (q[5] * q[5] + q[6] * q[6] + q[7] * q[7]) / rho;
    R d2 = R(0.5) * (b2 + c2);
    return osqrt(d2 + osqrt(rmax(d2 * d2 - c2 * bn * bn / rho, R(0))));
}

template <class R> static inline V9<R> phys_flux_x(const V9<R>& q, R gamma) {
    R rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4];
    R bx = q[5], by = q[6], bz = q[7];
    R b2 = bx * bx + by * by + bz * bz;
    R ptot = p + R(0.5) * b2;
    R ekin = R(0.5) * rho * (vx * vx + vy * vy + vz * vz);
    R E = p / (gamma - R(1)) + ekin + R(0.5) * b2;
    R vdotb = vx * bx + vy * by + vz * bz;
    return {rho * vx,
            rho * vx * vx + ptot - bx * bx,
            rho * vx * vy - bx * by,
            rho * vx * vz - bx * bz,
            (E + ptot) * vx - bx * vdotb,
            R(0),
            vx * by - vy * bx,
            vx * bz - vz * bx,
            R(0)};
}

// cyclic rotation so direction d (0,1,2) becomes the x normal (glmmhd_turb.jl:118-138)
template <class R> static inline V9<R> rot_to(const V9<R>& q, int d) {
    if (d == 0) return q;
    if (d == 1) return {q[0], q[2], q[3], q[1], q[4], q[6], q[7], q[5], q[8]};
    return {q[0], q[3], q[1], q[2], q[4], q[7], q[5], q[6], q[8]};
}
template <class R> static inline V9<R> rot_from(const V9<R>& f, int d) {
    if (d == 0) return f;
    if (d == 1) return {f[0], f[3], f[1], f[2], f[4], f[7], f[5], f[6], f[8]};
    return {f[0], f[2], f[3], f[1], f[4], f[6], f[7], f[5], f[8]};
}

template <class R> static inline R moncen(R dl, R dr) {
    R dc = R(0.5) * (dl + dr);
    R sgn = dc >= R(0) ? R(1) : R(-1);
    R val = sgn * rmin(R(2) * rmin(oabs(dl), oabs(dr)), oabs(dc));
    return dl * dr <= R(0) ? R(0) : val;
}
template <class R> static inline R minmod(R a, R b) {
    return a * b <= R(0) ? R(0) : (oabs(a) < oabs(b) ? a : b);
}
template <class R> static inline V9<R> slope(const V9<R>& L, const V9<R>& M, const V9<R>& Rr, bool mm) {
    V9<R> s;
    for (int i = 0; i < 9; ++i)
        s[i] = mm ? R(0.5) * minmod(M[i] - L[i], Rr[i] - M[i]) : R(0.5) * moncen(M[i] - L[i], Rr[i] - M[i]);
    return s;
}
template <class R> static inline V9<R> padd(const V9<R>& q, const V9<R>& s, R a) {
    V9<R> r;
    for (int i = 0; i < 9; ++i) r[i] = q[i] + a * s[i];
    return r;
}
template <class R> static inline V9<R> dir_flux(const V9<R>& q, int d, R gamma) {
    return rot_from(phys_flux_x(rot_to(q, d), gamma), d);
}

// unsplit MUSCL-Hancock predictor (glmmhd_turb.jl:165-172)
template <class R>
static inline V9<R> hancock(const V9<R>& m0, const V9<R>& sx, const V9<R>& sy, const V9<R>& sz, R dtdx, R gamma) {
    V9<R> u0 = prim2cons(m0, gamma);
    R h = R(0.5) * dtdx;
    V9<R> fxp = dir_flux(padd(m0, sx, R(1)), 0, gamma), fxm = dir_flux(padd(m0, sx, R(-1)), 0, gamma);
    V9<R> fyp = dir_flux(padd(m0, sy, R(1)), 1, gamma), fym = dir_flux(padd(m0, sy, R(-1)), 1, gamma);
    V9<R> fzp = dir_flux(padd(m0, sz, R(1)), 2, gamma), fzm = dir_flux(padd(m0, sz, R(-1)), 2, gamma);
    V9<R> r;
    for (int i = 0; i < 9; ++i)
        r[i] = u0[i] - h * ((fxp[i] - fxm[i]) + (fyp[i] - fym[i]) + (fzp[i] - fzm[i]));
    return r;
}

template <class R> static inline void glm_pair(R bnL, R bnR, R psiL, R psiR, R ch, R& bns, R& psis) {
    bns = R(0.5) * (bnL + bnR) - R(0.5) * (psiR - psiL) / ch;
    psis = R(0.5) * (psiL + psiR) - R(0.5) * ch * (bnR - bnL);
}

template <class R> static inline V9<R> llf_x(const V9<R>& L, const V9<R>& Rr, R gamma, R ch, R fbn, R fpsi, bool bound) {
    V9<R> fL = phys_flux_x(L, gamma), fR = phys_flux_x(Rr, gamma);
    V9<R> uL = prim2cons(L, gamma), uR = prim2cons(Rr, gamma);
    R sL, sR;
    if (bound) {  // fast_speed_bound (glmmhd_turb.jl:307-310)
        R irL = R(1) / L[0], irR = R(1) / Rr[0];
        sL = oabs(L[1]) + osqrt((gamma * L[4] + L[5] * L[5] + L[6] * L[6] + L[7] * L[7]) * irL);
        sR = oabs(Rr[1]) + osqrt((gamma * Rr[4] + Rr[5] * Rr[5] + Rr[6] * Rr[6] + Rr[7] * Rr[7]) * irR);
    } else {
        sL = oabs(L[1]) + fast_speed(L, gamma, L[5]);
        sR = oabs(Rr[1]) + fast_speed(Rr, gamma, Rr[5]);
    }
    R smax = rmax(rmax(sL, sR), ch);
    V9<R> f;
    for (int i = 0; i < 9; ++i) f[i] = R(0.5) * (fL[i] + fR[i]) - R(0.5) * smax * (uR[i] - uL[i]);
    f[5] = fbn; f[8] = fpsi;
    return f;
}

template <class R> static inline V9<R> hll_x(const V9<R>& L, const V9<R>& Rr, R gamma, R bn, R fbn, R fpsi) {
    R cfL = fast_speed(L, gamma, bn), cfR = fast_speed(Rr, gamma, bn);
    R SL = rmin(rmin(L[1] - cfL, Rr[1] - cfR), R(0));
    R SR = rmax(rmax(L[1] + cfL, Rr[1] + cfR), R(0));
    V9<R> fL = phys_flux_x(L, gamma), fR = phys_flux_x(Rr, gamma);
    V9<R> uL = prim2cons(L, gamma), uR = prim2cons(Rr, gamma);
    R ihd = R(1) / (SR - SL);
    V9<R> f;
    for (int i = 0; i < 9; ++i) f[i] = (SR * fL[i] - SL * fR[i] + SL * SR * (uR[i] - uL[i])) * ihd;
    f[5] = fbn; f[8] = fpsi;
    return f;
}

// Miyoshi & Kusano (2005) HLLD in the x-normal frame (glmmhd_turb.jl:193-272)
template <class R>
static inline V9<R> hlld_x(const V9<R>& L, const V9<R>& Rr, R gamma, R bn, R fbn, R fpsi) {
    const R tiny = R(1e-12);
    R dL = L[0], uL = L[1], vL = L[2], wL = L[3], pL = L[4], byL = L[6], bzL = L[7];
    R dR = Rr[0], uR = Rr[1], vR = Rr[2], wR = Rr[3], pR = Rr[4], byR = Rr[6], bzR = Rr[7];
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
    V9<R> UL = {dL, dL * uL, dL * vL, dL * wL, EL, bn, byL, bzL, R(0)};
    V9<R> UR = {dR, dR * uR, dR * vR, dR * wR, ER, bn, byR, bzR, R(0)};
    V9<R> FL = phys_flux_x(V9<R>{dL, uL, vL, wL, pL, bn, byL, bzL, R(0)}, gamma);
    V9<R> FR = phys_flux_x(V9<R>{dR, uR, vR, wR, pR, bn, byR, bzR, R(0)}, gamma);
    R den = (SR - uR) * dR - (SL - uL) * dL;
    R SM = ((SR - uR) * dR * uR - (SL - uL) * dL * uL - ptR + ptL) / den;
    R pts = ((SR - uR) * dR * ptL - (SL - uL) * dL * ptR + dL * dR * (SR - uR) * (SL - uL) * (uR - uL)) / den;
    R dLs = rmax(dL * (SL - uL) / (SL - SM), tiny);
    R dRs = rmax(dR * (SR - uR) / (SR - SM), tiny);
    R sqdLs = osqrt(dLs), sqdRs = osqrt(dRs);
    R SLs = SM - oabs(bn) / sqdLs;
    R SRs = SM + oabs(bn) / sqdRs;
    auto star = [&](R d, R u, R v, R w, R by, R bz, R S, R& vy, R& vz, R& byS, R& bzS, bool& degen) {
        R denK = d * (S - u) * (S - SM) - bn * bn;
        degen = oabs(denK) < tiny;   // degenerate star state (glmmhd_turb.jl:225-238)
        if (degen) {
            vy = v; vz = w; byS = by; bzS = bz;
        } else {
            R fac = bn * (SM - u) / denK;
            vy = v - by * fac;
            vz = w - bz * fac;
            byS = by * (d * (S - u) * (S - u) - bn * bn) / denK;
            bzS = bz * (d * (S - u) * (S - u) - bn * bn) / denK;
        }
    };
    R vyLs, vzLs, byLs, bzLs, vyRs, vzRs, byRs, bzRs;
    bool degL, degR;
    star(dL, uL, vL, wL, byL, bzL, SL, vyLs, vzLs, byLs, bzLs, degL);
    star(dR, uR, vR, wR, byR, bzR, SR, vyRs, vzRs, byRs, bzRs, degR);
    R vdotbL = uL * bn + vL * byL + wL * bzL;
    R vdotbLs = SM * bn + vyLs * byLs + vzLs * bzLs;
    R ELs = ((SL - uL) * EL - ptL * uL + pts * SM + bn * (vdotbL - vdotbLs)) / (SL - SM);
    R vdotbR = uR * bn + vR * byR + wR * bzR;
    R vdotbRs = SM * bn + vyRs * byRs + vzRs * bzRs;
    R ERs = ((SR - uR) * ER - ptR * uR + pts * SM + bn * (vdotbR - vdotbRs)) / (SR - SM);
    V9<R> ULs = {dLs, dLs * SM, dLs * vyLs, dLs * vzLs, ELs, bn, byLs, bzLs, R(0)};
    V9<R> URs = {dRs, dRs * SM, dRs * vyRs, dRs * vzRs, ERs, bn, byRs, bzRs, R(0)};
    R sgn = bn >= R(0) ? R(1) : R(-1);
    R invsum = R(1) / (sqdLs + sqdRs);
    R vyss = (sqdLs * vyLs + sqdRs * vyRs + (byRs - byLs) * sgn) * invsum;
    R vzss = (sqdLs * vzLs + sqdRs * vzRs + (bzRs - bzLs) * sgn) * invsum;
    R byss = (sqdLs * byRs + sqdRs * byLs + sqdLs * sqdRs * (vyRs - vyLs) * sgn) * invsum;
    R bzss = (sqdLs * bzRs + sqdRs * bzLs + sqdLs * sqdRs * (vzRs - vzLs) * sgn) * invsum;
    R vdotbss = SM * bn + vyss * byss + vzss * bzss;
    R ELss = ELs - sqdLs * (vdotbLs - vdotbss) * sgn;
    R ERss = ERs + sqdRs * (vdotbRs - vdotbss) * sgn;
    V9<R> ULss = {dLs, dLs * SM, dLs * vyss, dLs * vzss, ELss, bn, byss, bzss, R(0)};
    V9<R> URss = {dRs, dRs * SM, dRs * vyss, dRs * vzss, ERss, bn, byss, bzss, R(0)};
    V9<R> f;
    // sampling (glmmhd_turb.jl:262-270); a degenerate star counts when the region uses it
    if (SLs >= R(0)) {
        for (int i = 0; i < 9; ++i) f[i] = FL[i] + SL * (ULs[i] - UL[i]);
        count(ORC_CNT_HLLD_L);
        if (degL) count(ORC_CNT_HLLD_DEGEN);
    } else if (SM >= R(0)) {
        for (int i = 0; i < 9; ++i) f[i] = FL[i] + SLs * ULss[i] - (SLs - SL) * ULs[i] - SL * UL[i];
        count(ORC_CNT_HLLD_LS);
        if (degL || degR) count(ORC_CNT_HLLD_DEGEN);
    } else if (SRs >= R(0)) {
        for (int i = 0; i < 9; ++i) f[i] = FR[i] + SRs * URss[i] - (SRs - SR) * URs[i] - SR * UR[i];
        count(ORC_CNT_HLLD_RS);
        if (degL || degR) count(ORC_CNT_HLLD_DEGEN);
    } else {
        for (int i = 0; i < 9; ++i) f[i] = FR[i] + SR * (URs[i] - UR[i]);
        count(ORC_CNT_HLLD_R);
        if (degR) count(ORC_CNT_HLLD_DEGEN);
    }
    f[5] = fbn; f[8] = fpsi;
    return f;
}

// Riemann dispatch: rotate, floor, clean, solve, rotate back (glmmhd_turb.jl:275-292, 313-354)
template <class R>
static inline V9<R> riemann(const V9<R>& Lq, const V9<R>& Rq, int d, const Phys<R>& P, R ch) {
    V9<R> L = rot_to(Lq, d), Rr = rot_to(Rq, d);
    L[0] = rmax(L[0], P.smallr); L[4] = rmax(L[4], P.pfl);
    Rr[0] = rmax(Rr[0], P.smallr); Rr[4] = rmax(Rr[4], P.pfl);
    R bns, psis;
    glm_pair(L[5], Rr[5], L[8], Rr[8], ch, bns, psis);
    R fbn = psis, fpsi = ch * ch * bns;
    L[5] = bns; Rr[5] = bns;
    V9<R> f;
    if (P.riemann == ORC_RIEMANN_HLL) {
        f = hll_x(L, Rr, P.gamma, bns, fbn, fpsi);
    } else if (P.riemann == ORC_RIEMANN_LLF_BOUND) {
        f = llf_x(L, Rr, P.gamma, ch, fbn, fpsi, true);
    } else {
        bool sw = (P.llf_dmin > R(0) && rmin(L[0], Rr[0]) < P.llf_dmin) ||
                  (P.llf_pmin > R(0) && rmin(L[4], Rr[4]) < P.llf_pmin);   // glmmhd_turb.jl:287-289
        if (sw && P.riemann == ORC_RIEMANN_HLLD) count(ORC_CNT_LLF_SWITCH);
        bool uself = sw || P.riemann == ORC_RIEMANN_LLF;
        f = uself ? llf_x(L, Rr, P.gamma, ch, fbn, fpsi, false) : hlld_x(L, Rr, P.gamma, bns, fbn, fpsi);
    }
    return rot_from(f, d);
}

// PPM edges (glmmhd_turb.jl:917-926)
template <class R> static inline void ppm_mono(R ql, R q0, R qr, R& lo, R& hi) {
    R dq = qr - ql;
    R diff = (q0 - R(0.5) * (ql + qr)) * dq;
    if ((qr - q0) * (q0 - ql) <= R(0)) { lo = q0; hi = q0; }
    else if (diff > dq * dq / R(6)) { lo = R(3) * q0 - R(2) * qr; hi = qr; }
    else if (diff < -(dq * dq / R(6))) { lo = ql; hi = R(3) * q0 - R(2) * ql; }
    else { lo = ql; hi = qr; }
}
template <class R> static inline void ppm_edges(R qm, R q0, R qp, R& lo, R& hi) {
    R sl = R(0.25) * (qp - qm);
    R curve = (qm - R(2) * q0 + qp) / R(12);
    ppm_mono(q0 - sl + curve, q0, q0 + sl + curve, lo, hi);
}
template <class R> static inline bool spj(R a, R b, R c) {
    R hi = rmax(a, rmax(b, c));
    R lo = rmax(rmin(a, rmin(b, c)), R(1e-20));
    return hi / lo > R(2);
}

// ------------------------------------------------------------------------------------------
// Forcing: 61 +/- pairs of integer modes with 1 <= |k|^2 <= 9, evaluated as an exact mode sum
// ------------------------------------------------------------------------------------------
struct ModeTable {
    int k[ORC_NMODES][3];
    int n;
    ModeTable() {
        n = 0;
        for (int kx = 0; kx <= 3; ++kx)
            for (int ky = -3; ky <= 3; ++ky)
                for (int kz = -3; kz <= 3; ++kz) {
                    int k2 = kx * kx + ky * ky + kz * kz;
                    if (k2 < 1 || k2 > 9) continue;
                    bool half = kx > 0 || (kx == 0 && ky > 0) || (kx == 0 && ky == 0 && kz > 0);
                    if (!half) continue;
                    k[n][0] = kx; k[n][1] = ky; k[n][2] = kz; ++n;
                }
    }
};
static const ModeTable& modes_table() { static ModeTable t; return t; }

// cos/sin(2 pi m (i+1/2)/n) for m = 0..3 (cell centres), layout [m][cos|sin][i]
static std::vector<double> trig(int n) {
    std::vector<double> t(8 * (size_t)n);
    const double twopi = 6.283185307179586476925286766559;
    for (int m = 0; m < 4; ++m)
        for (int i = 0; i < n; ++i) {
            double th = twopi * (double)m * ((double)i + 0.5) / (double)n;
            t[(size_t)(2 * m) * n + i] = std::cos(th);
            t[(size_t)(2 * m + 1) * n + i] = std::sin(th);
        }
    return t;
}

// Mode-sum acceleration at one cell: a_c = ramp * sum_{k in H} 2 Re(ahat_{k,c} e^{i 2pi k.x/L}),
// separable order: for each kx, B = sum_{modes of that kx} ahat * e^{i(ky y + kz z)}; then
// a += 2 (Re B cos(kx x) - Im B sin(kx x)).  The GPU kernel evaluates the same order.
template <class R>
struct Forcer {
    const double* modes;
    std::vector<R> tx, ty, tz;
    int nx, ny, nz;
    R md[ORC_NMODES][3][2];
    Forcer(const orc_params* p, const double* m) : modes(m), nx(p->nx), ny(p->ny), nz(p->nz) {
        auto cv = [](const std::vector<double>& v) { return std::vector<R>(v.begin(), v.end()); };
        tx = cv(trig(nx)); ty = cv(trig(ny)); tz = cv(trig(nz));
        for (int q = 0; q < ORC_NMODES; ++q)
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 2; ++r) md[q][c][r] = (R)m[(q * 3 + c) * 2 + r];
    }
    // the modes scale with the forcing amplitude: tangent of a relative amplitude change
    void seed_amplitude(const double* rel) {
        for (int q = 0; q < ORC_NMODES; ++q)
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 2; ++r) {
                    double t[ORC_JVP_MAXDIR];
                    for (int i = 0; i < ORC_JVP_MAXDIR; ++i) t[i] = modes[(q * 3 + c) * 2 + r] * rel[i];
                    set_tangent(md[q][c][r], t);
                }
    }
    void accel(int i, int j, int k, R ramp, R a[3]) const {
        const ModeTable& T = modes_table();
        R S[3] = {R(0), R(0), R(0)};
        int q = 0;
        for (int kx = 0; kx <= 3; ++kx) {
            R Br[3] = {R(0), R(0), R(0)}, Bi[3] = {R(0), R(0), R(0)};
            while (q < T.n && T.k[q][0] == kx) {
                int ky = T.k[q][1], kz = T.k[q][2];
                int ay = ky < 0 ? -ky : ky, az = kz < 0 ? -kz : kz;
                R eyr = ty[(size_t)(2 * ay) * ny + j], eyi = ty[(size_t)(2 * ay + 1) * ny + j];
                R ezr = tz[(size_t)(2 * az) * nz + k], ezi = tz[(size_t)(2 * az + 1) * nz + k];
                if (ky < 0) eyi = -eyi;
                if (kz < 0) ezi = -ezi;
                R er = eyr * ezr - eyi * ezi;
                R ei = eyr * ezi + eyi * ezr;
                for (int c = 0; c < 3; ++c) {
                    R ar = md[q][c][0], ai = md[q][c][1];
                    Br[c] = Br[c] + (ar * er - ai * ei);
                    Bi[c] = Bi[c] + (ar * ei + ai * er);
                }
                ++q;
            }
            R cx = tx[(size_t)(2 * kx) * nx + i], sx = tx[(size_t)(2 * kx + 1) * nx + i];
            for (int c = 0; c < 3; ++c) S[c] = S[c] + R(2) * (Br[c] * cx - Bi[c] * sx);
        }
        for (int c = 0; c < 3; ++c) a[c] = ramp * S[c];
    }
};

// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11), written from the published description.
static inline void philox(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// ------------------------------------------------------------------------------------------
// Grid helpers
// ------------------------------------------------------------------------------------------
struct Grid {
    int nx, ny, nz;
    size_t n;
    explicit Grid(const orc_params* p) : nx(p->nx), ny(p->ny), nz(p->nz), n((size_t)p->nx * p->ny * p->nz) {}
    inline size_t idx(int i, int j, int k) const { return (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k); }
    static inline int wr(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }
};

template <class R> static inline V9<R> load9(const R* u, const Grid& g, int i, int j, int k) {
    size_t c = g.idx(Grid::wr(i, g.nx), Grid::wr(j, g.ny), Grid::wr(k, g.nz));
    V9<R> q;
    for (int v = 0; v < 9; ++v) q[v] = u[(size_t)v * g.n + c];
    return q;
}

// Update epilogue shared by every scheme: void floor, psi damping, forcing kick
// (glmmhd_turb.jl:447-475 with the tiled kernel's sc2 = smallc^2 grouping, :849-858)
template <class R>
static inline V9<R> finish_update(V9<R> r1, const Phys<R>& P, R glm_fac, bool turb, const R acc[3], R dt) {
    if (r1[0] < P.smallr) {   // void floor (glmmhd_turb.jl:450-453)
        R emag = R(0.5) * (r1[5] * r1[5] + r1[6] * r1[6] + r1[7] * r1[7]);
        r1 = {P.smallr, R(0), R(0), R(0), P.pfl / (P.gamma - R(1)) + emag, r1[5], r1[6], r1[7], r1[8]};
        count(ORC_CNT_VOID_FLOOR);
    }
    V9<R> r = r1;
    r[8] = r1[8] * glm_fac;
    if (turb && r[0] >= P.turb_min_rho) {
        R rhom = rmax(r[0], P.smallr);
        R sc2 = P.smallc * P.smallc;
        R rho = r[0];
        R e = r[4];
        R fl = rho * sc2;
        e = rmax(e - R(0.5) * r[1] * r[1] / rhom, fl);
        e = rmax(e - R(0.5) * r[2] * r[2] / rhom, fl);
        e = rmax(e - R(0.5) * r[3] * r[3] / rhom, fl);
        R m2 = r[1] + rhom * acc[0] * dt;
        R m3 = r[2] + rhom * acc[1] * dt;
        R m4 = r[3] + rhom * acc[2] * dt;
        e = rmax(e + R(0.5) * m2 * m2 / rhom, fl);
        e = rmax(e + R(0.5) * m3 * m3 / rhom, fl);
        e = rmax(e + R(0.5) * m4 * m4 / rhom, fl);
        r = {r[0], m2, m3, m4, e, r[5], r[6], r[7], r[8]};
    }
    return r;
}

// ------------------------------------------------------------------------------------------
// Unsplit step.  Reconstruction of one cell -> its 6 interface states (+x,-x,+y,-y,+z,-z).
// ------------------------------------------------------------------------------------------
template <class R> struct Faces { V9<R> f[6]; };

template <class R>
static inline Faces<R> recon_cell(const R* u, const Grid& g, int i, int j, int k, const Phys<R>& P, R dtdx) {
    auto c2p = [&](int a, int b, int c) { return cons2prim(load9(u, g, a, b, c), P.gamma, P.smallr, P.pfl); };
    V9<R> m0 = c2p(i, j, k);
    V9<R> mxl = c2p(i - 1, j, k), mxr = c2p(i + 1, j, k);
    V9<R> myl = c2p(i, j - 1, k), myr = c2p(i, j + 1, k);
    V9<R> mzl = c2p(i, j, k - 1), mzr = c2p(i, j, k + 1);
    bool mm = P.recon == ORC_RECON_MINMOD;
    V9<R> sx = slope(mxl, m0, mxr, mm), sy = slope(myl, m0, myr, mm), sz = slope(mzl, m0, mzr, mm);
    V9<R> mh = cons2prim(hancock(m0, sx, sy, sz, dtdx, P.gamma), P.gamma, P.smallr, P.pfl);
    if (mh[0] <= P.smallr || mh[4] <= P.pfl) {   // predictor revert (glmmhd_turb.jl:393-395)
        mh = m0;
        count(ORC_CNT_HANCOCK_REVERT);
    }
    Faces<R> F;
    const V9<R>* s[3] = {&sx, &sy, &sz};
    if (P.recon == ORC_RECON_PPM) {
        // integrator_plm_ppm! stage 2 (glmmhd_turb.jl:952-975)
        bool up = !(spj(mxl[4], m0[4], mxr[4]) || spj(myl[4], m0[4], myr[4]) || spj(mzl[4], m0[4], mzr[4]));
        if (!up) count(ORC_CNT_PPM_FALLBACK);
        const V9<R>* nb[3][2] = {{&mxl, &mxr}, {&myl, &myr}, {&mzl, &mzr}};
        for (int d = 0; d < 3; ++d) {
            if (up) {
                V9<R> lo, hi;
                for (int v = 0; v < 9; ++v) ppm_edges((*nb[d][0])[v], m0[v], (*nb[d][1])[v], lo[v], hi[v]);
                for (int v = 0; v < 9; ++v) {
                    F.f[2 * d][v] = mh[v] + hi[v] - m0[v];
                    F.f[2 * d + 1][v] = mh[v] + lo[v] - m0[v];
                }
            } else {
                F.f[2 * d] = padd(mh, *s[d], R(1));
                F.f[2 * d + 1] = padd(mh, *s[d], R(-1));
            }
        }
    } else {
        for (int d = 0; d < 3; ++d) {
            F.f[2 * d] = padd(mh, *s[d], R(1));
            F.f[2 * d + 1] = padd(mh, *s[d], R(-1));
        }
    }
    if (P.iflo)
        for (int f = 0; f < 6; ++f)
            if (F.f[f][0] < P.smallr || F.f[f][4] < P.pfl) {   // iflo revert (glmmhd_turb.jl:618)
                F.f[f] = m0;
                count(ORC_CNT_IFLO_REVERT);
            }
    return F;
}

// Plane-streaming driver: each thread owns a z-slab, keeps a ring of 3 reconstructed planes and
// computes every face flux exactly once (the step_multi! semantics of glmmhd_turb.jl:1981-1992
// without its N^3 scratch arrays).
template <class R>
static void step_unsplit(const orc_params* p, const orc_step_args* a, const R* uold, R* unew,
                         const double* amp_rel = nullptr) {
    Grid g(p);
    Phys<R> P(p);
    const R dx = (R)p->boxlen / (R)p->nx;
    const R dt = (R)a->dt, dtdx = dt / dx, ch = (R)a->ch, glm_fac = (R)a->glm_fac, ramp = (R)a->ramp;
    const bool turb = a->do_turb && a->modes;
    Forcer<R>* fo = turb ? new Forcer<R>(p, a->modes) : nullptr;
    if (fo && amp_rel) fo->seed_amplitude(amp_rel);
    const int nxy = g.nx * g.ny;
    int nt = std::max(1, std::min(nthreads(), g.nz));
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        int tid = omp_get_thread_num(), nth = omp_get_num_threads();
#else
        int tid = 0, nth = 1;
#endif
        int za = (int)((long)g.nz * tid / nth), zb = (int)((long)g.nz * (tid + 1) / nth);
        if (zb > za) {
            std::vector<Faces<R>> ring[3];
            for (auto& r : ring) r.resize(nxy);
            std::vector<V9<R>> Fx(nxy), Fy(nxy), Fzlo(nxy), Fzhi(nxy);
            auto rec_plane = [&](int k) {
                std::vector<Faces<R>>& r = ring[((k % 3) + 3) % 3];
                for (int j = 0; j < g.ny; ++j)
                    for (int i = 0; i < g.nx; ++i) r[i + g.nx * j] = recon_cell(uold, g, i, j, Grid::wr(k, g.nz), P, dtdx);
            };
            auto ringp = [&](int k) -> std::vector<Faces<R>>& { return ring[((k % 3) + 3) % 3]; };
            rec_plane(za - 1);
            rec_plane(za);
            {
                auto& rm = ringp(za - 1);
                auto& r0 = ringp(za);
                for (int c = 0; c < nxy; ++c) Fzlo[c] = riemann(rm[c].f[4], r0[c].f[5], 2, P, ch);
            }
            for (int k = za; k < zb; ++k) {
                rec_plane(k + 1);
                auto& r0 = ringp(k);
                auto& rp = ringp(k + 1);
                for (int j = 0; j < g.ny; ++j)
                    for (int i = 0; i < g.nx; ++i) {
                        int c = i + g.nx * j;
                        int cxp = Grid::wr(i + 1, g.nx) + g.nx * j;
                        int cyp = i + g.nx * Grid::wr(j + 1, g.ny);
                        Fx[c] = riemann(r0[c].f[0], r0[cxp].f[1], 0, P, ch);
                        Fy[c] = riemann(r0[c].f[2], r0[cyp].f[3], 1, P, ch);
                        Fzhi[c] = riemann(r0[c].f[4], rp[c].f[5], 2, P, ch);
                    }
                for (int j = 0; j < g.ny; ++j)
                    for (int i = 0; i < g.nx; ++i) {
                        int c = i + g.nx * j;
                        int cxm = Grid::wr(i - 1, g.nx) + g.nx * j;
                        int cym = i + g.nx * Grid::wr(j - 1, g.ny);
                        size_t gc = g.idx(i, j, k);
                        V9<R> r1;
                        for (int v = 0; v < 9; ++v) {
                            R u0 = uold[(size_t)v * g.n + gc];
                            r1[v] = u0 + dtdx * ((Fx[cxm][v] - Fx[c][v]) + (Fy[cym][v] - Fy[c][v]) +
                                                 (Fzlo[c][v] - Fzhi[c][v]));
                        }
                        R acc[3] = {R(0), R(0), R(0)};
                        if (turb) fo->accel(i, j, k, ramp, acc);
                        V9<R> r = finish_update(r1, P, glm_fac, turb, acc, dt);
                        for (int v = 0; v < 9; ++v) unew[(size_t)v * g.n + gc] = r[v];
                    }
                std::swap(Fzlo, Fzhi);
            }
        }
    }
    delete fo;
}

// ------------------------------------------------------------------------------------------
// Transverse-free 1-D Hancock march scheme (spike_mhd.cu:65-223, 257-299) with an update base
// taken from the state itself (not from a 16-bit tile).  Face fluxes at the lower face of each
// cell per direction are computed once and shared by the two neighbours (bit-identical to the
// spike's per-cell recomputation).
// ------------------------------------------------------------------------------------------
template <class R> static inline V9<R> prim_from_cons_floor(const V9<R>& c, R gamma, R smallr, R smallp) {
    return cons2prim(c, gamma, smallr, smallp);
}
template <class R>
static inline V9<R> hanc1d(const V9<R>& c0, const V9<R>& s, int d, R dtdx, R gamma, R smallr, R smallp) {
    // s is the FULL limited slope here (spike convention); faces at c0 -/+ s/2
    V9<R> FL = dir_flux(padd(c0, s, R(-0.5)), d, gamma), FR = dir_flux(padd(c0, s, R(0.5)), d, gamma);
    V9<R> U = prim2cons(c0, gamma);
    R h = R(0.5) * dtdx;
    for (int v = 0; v < 9; ++v) U[v] = U[v] - h * (FR[v] - FL[v]);
    V9<R> q = prim_from_cons_floor(U, gamma, smallr, smallp);
    if (q[0] <= smallr || q[4] <= smallp) count(ORC_CNT_PRED1D_FLOOR);   // floored predictor
    return q;
}
// spike moncen(a,b,c) = sgn*min(|dc|, 2|dl|, 2|dr|), dc = (c-a)/2  (full slope)
template <class R> static inline R full_mc(R a, R b, R c) {
    R dl = b - a, dr = c - b, dc = R(0.5) * (c - a);
    if (dl * dr <= R(0)) return R(0);
    R sg = dl > R(0) ? R(1) : R(-1);
    return sg * rmin(std::fabs(dc), rmin(R(2) * std::fabs(dl), R(2) * std::fabs(dr)));
}
template <class R> static inline V9<R> full_slope(const V9<R>& a, const V9<R>& b, const V9<R>& c) {
    V9<R> s;
    for (int v = 0; v < 9; ++v) s[v] = full_mc(a[v], b[v], c[v]);
    return s;
}
// one lower-face flux in direction d from 4 cells along d (m2, m1 | c0, p1)
template <class R>
static inline V9<R> march_face(const V9<R>& m2, const V9<R>& m1, const V9<R>& c0, const V9<R>& p1, int d,
                               const Phys<R>& P, R dtdx, R ch, bool ppm) {
    V9<R> sL = full_slope(m2, m1, c0), sR = full_slope(m1, c0, p1);
    V9<R> mhL = hanc1d(m1, sL, d, dtdx, P.gamma, P.smallr, P.smallp);
    V9<R> mhR = hanc1d(c0, sR, d, dtdx, P.gamma, P.smallr, P.smallp);
    V9<R> L, Rr;
    if (ppm) {  // parabolic edge (Julia ppm_edges form) + predictor shift e + mh - c
        // only the neighbours m2..p1 are available: +face of m1 uses (m2,m1,c0), -face of c0 uses (m1,c0,p1)
        for (int v = 0; v < 9; ++v) {
            R lo, hi;
            ppm_edges(m2[v], m1[v], c0[v], lo, hi);
            L[v] = hi + mhL[v] - m1[v];
            ppm_edges(m1[v], c0[v], p1[v], lo, hi);
            Rr[v] = lo + mhR[v] - c0[v];
        }
    } else {
        L = padd(mhL, sL, R(0.5));
        Rr = padd(mhR, sR, R(-0.5));
    }
    if (L[0] < P.smallr || L[4] < P.smallp || Rr[0] < P.smallr || Rr[4] < P.smallp) count(ORC_CNT_FACE_FLOOR);
    L[0] = rmax(L[0], P.smallr); L[4] = rmax(L[4], P.smallp);
    Rr[0] = rmax(Rr[0], P.smallr); Rr[4] = rmax(Rr[4], P.smallp);
    // hllMHD (spike_mhd.cu:199-223) == riemann_hll with the floors already applied
    V9<R> Lr = rot_to(L, d), Rrr = rot_to(Rr, d);
    R bns, psis;
    glm_pair(Lr[5], Rrr[5], Lr[8], Rrr[8], ch, bns, psis);
    Lr[5] = bns; Rrr[5] = bns;
    V9<R> f = hll_x(Lr, Rrr, P.gamma, bns, psis, ch * ch * bns);
    return rot_from(f, d);
}

// Passive species (spike_mhd.cu:55-61, 128-139, 155-158, 218-221, 241-244, 278-296): the fraction
// X = rho*X / max(rho, smallr) gets the full MonCen slope, the predictor X - dt/(2dx) u_n dX and the
// faces X_h +- s/2 (or the PPM edge + predictor shift), and rides the face mass flux (consistent
// multi-fluid advection): F_X = F_rho X_L if F_rho >= 0, else F_rho X_R.
template <class R>
static inline R species_face(R xm2, R xm1, R xc0, R xp1, R un_m1, R un_c0, R h, R frho, bool ppm) {
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
static void step_march1d(const orc_params* p, const orc_step_args* a, const R* uold, R* unew) {
    Grid g(p);
    Phys<R> P(p);
    const R dx = (R)p->boxlen / (R)p->nx;
    const R dt = (R)a->dt, dtdx = dt / dx, ch = (R)a->ch, glm_fac = (R)a->glm_fac;
    const bool ppm = p->recon == ORC_RECON_PPM;
    std::vector<V9<R>> prim(g.n);
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i)
                prim[g.idx(i, j, k)] = cons2prim(load9(uold, g, i, j, k), P.gamma, P.smallr, P.smallp);
    std::vector<V9<R>> F[3];
    for (auto& f : F) f.resize(g.n);
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i)
                for (int d = 0; d < 3; ++d) {
                    int o[3] = {d == 0, d == 1, d == 2};
                    auto P_ = [&](int s) {
                        return prim[g.idx(Grid::wr(i + s * o[0], g.nx), Grid::wr(j + s * o[1], g.ny),
                                          Grid::wr(k + s * o[2], g.nz))];
                    };
                    F[d][g.idx(i, j, k)] = march_face(P_(-2), P_(-1), P_(0), P_(1), d, P, dtdx, ch, ppm);
                }
    // species fractions and their lower-face fluxes
    const int nsp = p->nsp;
    std::vector<R> X((size_t)nsp * g.n), FS((size_t)3 * nsp * g.n);
    for (int s = 0; s < nsp; ++s)
        for (size_t c = 0; c < g.n; ++c) X[(size_t)s * g.n + c] = uold[(size_t)(9 + s) * g.n + c] / prim[c][0];
    const R h = R(0.5) * dtdx;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i)
                for (int d = 0; d < 3; ++d) {
                    int o[3] = {d == 0, d == 1, d == 2};
                    auto I_ = [&](int s) {
                        return g.idx(Grid::wr(i + s * o[0], g.nx), Grid::wr(j + s * o[1], g.ny), Grid::wr(k + s * o[2], g.nz));
                    };
                    size_t c = g.idx(i, j, k);
                    for (int s = 0; s < nsp; ++s) {
                        const R* x = X.data() + (size_t)s * g.n;
                        FS[((size_t)d * nsp + s) * g.n + c] =
                            species_face(x[I_(-2)], x[I_(-1)], x[I_(0)], x[I_(1)], prim[I_(-1)][1 + d], prim[I_(0)][1 + d], h,
                                         F[d][c][0], ppm);
                    }
                }
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                size_t c = g.idx(i, j, k);
                size_t cp[3] = {g.idx(Grid::wr(i + 1, g.nx), j, k), g.idx(i, Grid::wr(j + 1, g.ny), k),
                                g.idx(i, j, Grid::wr(k + 1, g.nz))};
                for (int v = 0; v < 9; ++v) {
                    R div = R(0);
                    for (int d = 0; d < 3; ++d) div = div + (F[d][cp[d]][v] - F[d][c][v]);
                    R u = uold[(size_t)v * g.n + c] - dtdx * div;
                    if (v == 8) u = u * glm_fac;
                    unew[(size_t)v * g.n + c] = u;
                }
                for (int s = 0; s < nsp; ++s) {
                    R div = R(0);
                    for (int d = 0; d < 3; ++d) {
                        const R* f = FS.data() + ((size_t)d * nsp + s) * g.n;
                        div = div + (f[cp[d]] - f[c]);
                    }
                    unew[(size_t)(9 + s) * g.n + c] = uold[(size_t)(9 + s) * g.n + c] - dtdx * div;
                }
            }
}

// ------------------------------------------------------------------------------------------
// Constrained transport (ct_mhd.jl, spike_ctm.cu).  q = [rho, mx, my, mz, E, bxf, byf, bzf],
// bxf[i,j,k] = Bx on the lower-x face (i-1/2, j, k).  Cell prims use Bcc = face average.
// Per direction, the lower-face flux uses the transverse-free 1-D Hancock predictor on the
// 4-cell stencil (i-2 .. i+1), the face normal B, and HLL or HLLD (no GLM).  Edge EMFs are the
// Balsara-Spicer average (ct_mhd.jl:139-154) or the upwind contact-mode EMF of Gardiner & Stone
// (2005, J. Comput. Phys. 205, 509), the latter selected by ORC_EMF_CONTACT.
// ------------------------------------------------------------------------------------------
template <class R>
static inline V9<R> ct_face_flux(const V9<R>& m2, const V9<R>& m1, const V9<R>& c0, const V9<R>& p1, R bn, int d,
                                 const Phys<R>& P, R dtdx) {
    // slopes: spike_ctm full slope (faces at +-s/2); ct_mhd.jl's pslope adds another factor 1/2
    V9<R> sL = full_slope(m2, m1, c0), sR = full_slope(m1, c0, p1);
    if (P.halfslope)
        for (int v = 0; v < 9; ++v) { sL[v] = R(0.5) * sL[v]; sR[v] = R(0.5) * sR[v]; }
    V9<R> mhL = hanc1d(m1, sL, d, dtdx, P.gamma, P.smallr, P.smallp);
    V9<R> mhR = hanc1d(c0, sR, d, dtdx, P.gamma, P.smallr, P.smallp);
    V9<R> L, Rr;
    if (P.recon == ORC_RECON_PPM) {
        for (int v = 0; v < 9; ++v) {
            R lo, hi;
            ppm_edges(m2[v], m1[v], c0[v], lo, hi);
            L[v] = hi + mhL[v] - m1[v];
            ppm_edges(m1[v], c0[v], p1[v], lo, hi);
            Rr[v] = lo + mhR[v] - c0[v];
        }
    } else {
        L = padd(mhL, sL, R(0.5));
        Rr = padd(mhR, sR, R(-0.5));
    }
    if (L[0] < P.smallr || L[4] < P.smallp || Rr[0] < P.smallr || Rr[4] < P.smallp) count(ORC_CNT_FACE_FLOOR);
    L[0] = rmax(L[0], P.smallr); L[4] = rmax(L[4], P.smallp);
    Rr[0] = rmax(Rr[0], P.smallr); Rr[4] = rmax(Rr[4], P.smallp);
    L[5 + d] = bn; Rr[5 + d] = bn;
    L[8] = R(0); Rr[8] = R(0);
    V9<R> Lr = rot_to(L, d), Rrr = rot_to(Rr, d);
    V9<R> f = P.riemann == ORC_RIEMANN_HLLD ? hlld_x(Lr, Rrr, P.gamma, bn, R(0), R(0))
                                            : hll_x(Lr, Rrr, P.gamma, bn, R(0), R(0));
    return rot_from(f, d);
}

template <class R> struct CTWork {
    std::vector<V9<R>> prim;   // cell prims with Bcc (psi slot unused = 0)
    std::vector<V9<R>> F[3];   // lower-face fluxes
    std::vector<R> ecc[3];     // cell-centre EMF components (contact EMF only)
    std::vector<R> ed[3];      // edge EMFs ex, ey, ez
};

template <class R>
static void step_ct(const orc_params* p, const orc_step_args* a, const R* qold, R* qnew) {
    Grid g(p);
    Phys<R> P(p);
    const R dx = (R)p->boxlen / (R)p->nx;
    const R dt = (R)a->dt, dtdx = dt / dx, ramp = (R)a->ramp;
    const bool turb = a->do_turb && a->modes;
    Forcer<R>* fo = turb ? new Forcer<R>(p, a->modes) : nullptr;
    const size_t n = g.n;
    const R* bf[3] = {qold + 5 * n, qold + 6 * n, qold + 7 * n};
    CTWork<R> W;
    W.prim.resize(n);
    for (auto& f : W.F) f.resize(n);
    for (auto& e : W.ed) e.resize(n);
    const int nt = nthreads();
    // bcc + cell prims (ct_mhd.jl:85-97, cellprim :25-33)
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                size_t c = g.idx(i, j, k);
                R bx = R(0.5) * (bf[0][c] + bf[0][g.idx(Grid::wr(i + 1, g.nx), j, k)]);
                R by = R(0.5) * (bf[1][c] + bf[1][g.idx(i, Grid::wr(j + 1, g.ny), k)]);
                R bz = R(0.5) * (bf[2][c] + bf[2][g.idx(i, j, Grid::wr(k + 1, g.nz))]);
                V9<R> cu = {qold[c], qold[n + c], qold[2 * n + c], qold[3 * n + c], qold[4 * n + c], bx, by, bz, R(0)};
                W.prim[c] = cons2prim(cu, P.gamma, P.smallr, P.smallp);
            }
    // lower-face fluxes per direction (ct_mhd.jl:99-121)
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i)
                for (int d = 0; d < 3; ++d) {
                    int o[3] = {d == 0, d == 1, d == 2};
                    auto Pc = [&](int s) {
                        return W.prim[g.idx(Grid::wr(i + s * o[0], g.nx), Grid::wr(j + s * o[1], g.ny),
                                            Grid::wr(k + s * o[2], g.nz))];
                    };
                    size_t c = g.idx(i, j, k);
                    W.F[d][c] = ct_face_flux(Pc(-2), Pc(-1), Pc(0), Pc(1), bf[d][c], d, P, dtdx);
                }
    // edge EMFs.  ez at (i-1/2,j-1/2,k); ex at (i,j-1/2,k-1/2); ey at (i-1/2,j,k-1/2).
    // Face EMF values: E_z on an x face = -Fx[By], on a y face = +Fy[Bx]; E_x on a y face = -Fy[Bz],
    // on a z face = +Fz[By]; E_y on a z face = -Fz[Bx], on an x face = +Fx[Bz].
    if (P.emf == ORC_EMF_CONTACT) {
        for (auto& e : W.ecc) e.resize(n);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (size_t c = 0; c < n; ++c) {
            const V9<R>& q = W.prim[c];
            // E = -v x B
            W.ecc[0][c] = q[2] * q[7] - q[3] * q[6];   // Ex = vy Bz - vz By  ... sign: E = -(v x B)
            W.ecc[1][c] = q[3] * q[5] - q[1] * q[7];
            W.ecc[2][c] = q[1] * q[6] - q[2] * q[5];
            for (int v = 0; v < 3; ++v) W.ecc[v][c] = -W.ecc[v][c];
        }
    }
    // generic corner EMF for the edge along axis e, spanned by the two other axes a (first) and
    // b (second) in cyclic order: e=z -> (a,b)=(x,y); e=x -> (y,z); e=y -> (z,x).
    // Face EMF on an a-face (normal a): Ea = sa * F_a[B_b]; on a b-face: Eb = sb * F_b[B_a],
    // with sa = -1, sb = +1 for the cyclic (a,b,e) order.
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                for (int e = 0; e < 3; ++e) {
                    int A = (e + 1) % 3, B = (e + 2) % 3;
                    int ia[3] = {0, 0, 0}, ib[3] = {0, 0, 0};
                    ia[A] = 1; ib[B] = 1;
                    auto at = [&](int sa, int sb) {
                        return g.idx(Grid::wr(i - sa * ia[0] - sb * ib[0], g.nx),
                                     Grid::wr(j - sa * ia[1] - sb * ib[1], g.ny),
                                     Grid::wr(k - sa * ia[2] - sb * ib[2], g.nz));
                    };
                    // cell (i,j,k) = (a0,b0); edge sits at (a0-1/2, b0-1/2)
                    size_t c00 = at(0, 0), c10 = at(1, 0), c01 = at(0, 1), c11 = at(1, 1);
                    // a-face (a0-1/2, b0) is stored at cell c00 in F[A]; (a0-1/2, b0-1) at c01
                    R EaN = -W.F[A][c00][5 + B];   // a-face at b0
                    R EaS = -W.F[A][c01][5 + B];   // a-face at b0-1
                    R EbE = W.F[B][c00][5 + A];    // b-face at a0
                    R EbW = W.F[B][c10][5 + A];    // b-face at a0-1
                    R E = R(0.25) * (EbE + EbW + EaN + EaS);
                    if (P.emf == ORC_EMF_CONTACT) {
                        const std::vector<R>& Ec = W.ecc[e];
                        auto up = [](R flux, R minus, R plus) {
                            return flux > R(0) ? minus : (flux < R(0) ? plus : R(0.5) * (minus + plus));
                        };
                        // d/db at b0-1/4 along the a-face row b0: cells (a0-1,b0), (a0,b0)
                        R dN = up(W.F[A][c00][0], Ec[c10] - EbW, Ec[c00] - EbE);
                        // d/db at b0-3/4 along row b0-1: cells (a0-1,b0-1), (a0,b0-1)
                        R dS = up(W.F[A][c01][0], EbW - Ec[c11], EbE - Ec[c01]);
                        // d/da at a0-1/4 along the b-face column a0: cells (a0,b0-1), (a0,b0)
                        R dE = up(W.F[B][c00][0], Ec[c01] - EaS, Ec[c00] - EaN);
                        // d/da at a0-3/4 along column a0-1: cells (a0-1,b0-1), (a0-1,b0)
                        R dW = up(W.F[B][c10][0], EaS - Ec[c11], EaN - Ec[c10]);
                        E = E + R(0.25) * (dS - dN) + R(0.25) * (dW - dE);
                    }
                    W.ed[e][c00] = E;
                }
            }
    // hydro update (ct_mhd.jl:124-137) + face-B curl (ct_mhd.jl:156-172) + floor/kick epilogue
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                size_t c = g.idx(i, j, k);
                int ip = Grid::wr(i + 1, g.nx), jp = Grid::wr(j + 1, g.ny), kp = Grid::wr(k + 1, g.nz);
                size_t cxp = g.idx(ip, j, k), cyp = g.idx(i, jp, k), czp = g.idx(i, j, kp);
                const std::vector<R>& ex = W.ed[0];
                const std::vector<R>& ey = W.ed[1];
                const std::vector<R>& ez = W.ed[2];
                R bxn = bf[0][c] - dtdx * ((ez[cyp] - ez[c]) - (ey[czp] - ey[c]));
                R byn = bf[1][c] - dtdx * ((ex[czp] - ex[c]) - (ez[cxp] - ez[c]));
                R bzn = bf[2][c] - dtdx * ((ey[cxp] - ey[c]) - (ex[cyp] - ex[c]));
                qnew[5 * n + c] = bxn; qnew[6 * n + c] = byn; qnew[7 * n + c] = bzn;
                V9<R> r1;
                for (int v = 0; v < 5; ++v)
                    r1[v] = qold[(size_t)v * n + c] + dtdx * ((W.F[0][c][v] - W.F[0][cxp][v]) +
                                                              (W.F[1][c][v] - W.F[1][cyp][v]) +
                                                              (W.F[2][c][v] - W.F[2][czp][v]));
                // epilogue sees the OLD cell-centred field (the new face field is not averaged here)
                r1[5] = W.prim[c][5]; r1[6] = W.prim[c][6]; r1[7] = W.prim[c][7]; r1[8] = R(0);
                R acc[3] = {R(0), R(0), R(0)};
                if (turb) fo->accel(i, j, k, ramp, acc);
                V9<R> r = finish_update(r1, P, R(1), turb, acc, dt);
                for (int v = 0; v < 5; ++v) qnew[(size_t)v * n + c] = r[v];
            }
    delete fo;
}

// ------------------------------------------------------------------------------------------
// CFL and diagnostics
// ------------------------------------------------------------------------------------------
template <class R> static void cfl(const orc_params* p, const R* u, double* out) {
    Grid g(p);
    Phys<R> P(p);
    double m0 = 0.0, m1 = 0.0;
#pragma omp parallel for num_threads(nthreads()) reduction(max : m0, m1) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                V9<R> q = cons2prim(load9(u, g, i, j, k), P.gamma, P.smallr, P.pfl);
                R sx = std::fabs(q[1]) + fast_speed(q, P.gamma, q[5]);
                R sy = std::fabs(q[2]) + fast_speed(q, P.gamma, q[6]);
                R sz = std::fabs(q[3]) + fast_speed(q, P.gamma, q[7]);
                R ct = sx + sy + sz;
                R sm = rmax(rmax(sx, sy), sz);
                m0 = std::max(m0, (double)ct);
                m1 = std::max(m1, (double)sm);
            }
    out[0] = m0; out[1] = m1;
}

template <class R> static void diag(const orc_params* p, const R* u, orc_diag* d) {
    Grid g(p);
    const double dx = p->boxlen / p->nx;
    double mass = 0, ke2 = 0, et = 0, dbm = 0, rmin_ = 1e300, db2 = 0, ps2 = 0;
    int fin = 1;
    const size_t n = g.n;
#pragma omp parallel for num_threads(nthreads()) reduction(+ : mass, ke2, et, db2, ps2) reduction(max : dbm) \
    reduction(min : rmin_) reduction(&& : fin) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                size_t c = g.idx(i, j, k);
                double rho = u[c], mx = u[n + c], my = u[2 * n + c], mz = u[3 * n + c];
                mass += rho;
                ke2 += (mx * mx + my * my + mz * mz) / std::max(rho, p->smallr);
                et += (double)u[4 * n + c];
                rmin_ = std::min(rmin_, rho);
                ps2 += (double)u[8 * n + c] * (double)u[8 * n + c];
                double bxp = u[5 * n + g.idx(Grid::wr(i + 1, g.nx), j, k)], bxm = u[5 * n + g.idx(Grid::wr(i - 1, g.nx), j, k)];
                double byp = u[6 * n + g.idx(i, Grid::wr(j + 1, g.ny), k)], bym = u[6 * n + g.idx(i, Grid::wr(j - 1, g.ny), k)];
                double bzp = u[7 * n + g.idx(i, j, Grid::wr(k + 1, g.nz))], bzm = u[7 * n + g.idx(i, j, Grid::wr(k - 1, g.nz))];
                double db = std::fabs((bxp - bxm) + (byp - bym) + (bzp - bzm)) / (2.0 * dx);
                dbm = std::max(dbm, db);
                db2 += db * db;
                for (int v = 0; v < 9; ++v)
                    if (!std::isfinite((double)u[(size_t)v * n + c])) fin = 0;
            }
    d->mass = mass; d->ke2 = ke2; d->vrms = std::sqrt(ke2 / mass); d->divbmax = dbm; d->rhomin = rmin_;
    d->etot = et; d->divb_l2 = std::sqrt(db2 / (double)n); d->psi_l2 = std::sqrt(ps2 / (double)n); d->finite = fin;
}

}  // namespace

// ==========================================================================================
// C ABI
// ==========================================================================================
extern "C" {

int orc_set_threads(int n) { g_threads = n; return nthreads(); }
void orc_count_reset(int on) {
    g_count_on.store(0);
    for (auto& c : g_cnt) c.store(0);
    g_count_on.store(on ? 1 : 0);
}
void orc_count_get(int64_t* out, int n) {
    for (int i = 0; i < n && i < ORC_CNT_N; ++i) out[i] = (int64_t)g_cnt[i].load();
}
int orc_num_modes(void) { return modes_table().n; }
void orc_mode_k(int32_t* k3) {
    const ModeTable& t = modes_table();
    for (int q = 0; q < t.n; ++q)
        for (int c = 0; c < 3; ++c) k3[3 * q + c] = t.k[q][c];
}
void orc_trig_table(int n, double* out) {
    std::vector<double> t = trig(n);
    std::memcpy(out, t.data(), t.size() * sizeof(double));
}
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { philox(ctr, key, out); }

// sigma0 such that the stationary rms of |a(x)| equals amp (sqrt(P(k)) = 1/|k| weighting as
// glmmhd_turb.jl:2085): <|a|^2> = sum_H 2 E|ahat_k|^2, E|ahat_k|^2 = 4 (sigma0/|k|)^2 beta^2/(1-alpha^2)
double orc_forcing_sigma0(double amp, double alpha, double beta) {
    const ModeTable& t = modes_table();
    double s = 0.0;
    for (int q = 0; q < t.n; ++q) s += 1.0 / (double)(t.k[q][0] * t.k[q][0] + t.k[q][1] * t.k[q][1] + t.k[q][2] * t.k[q][2]);
    return amp * std::sqrt((1.0 - alpha * alpha) / (8.0 * beta * beta * s));
}

// One OU step of every mode: ahat <- alpha*ahat + beta*sigma_k*P_k(xi), P_k = solenoidal projector
// (comp_frac = 0 in glmmhd_turb.jl:2104-2108).  xi: 6 standard normals per mode from
// Philox4x32-10(counter = {counter, mode, 0|1, 0}, key = {seed, 0x9E3779B9}) + Box-Muller.
void orc_ou_update(double* modes, uint32_t seed, uint32_t counter, double alpha, double beta, double sigma0) {
    const ModeTable& t = modes_table();
    const double twopi = 6.283185307179586476925286766559;
    for (int q = 0; q < t.n; ++q) {
        uint32_t r[8];
        uint32_t key[2] = {seed, 0x9E3779B9u};
        uint32_t c0[4] = {counter, (uint32_t)q, 0u, 0u}, c1[4] = {counter, (uint32_t)q, 1u, 0u};
        philox(c0, key, r);
        philox(c1, key, r + 4);
        double z[6];
        for (int b = 0; b < 3; ++b) {
            double u1 = ((double)r[2 * b] + 0.5) * 2.3283064365386962890625e-10;
            double u2 = ((double)r[2 * b + 1] + 0.5) * 2.3283064365386962890625e-10;
            double rr = std::sqrt(-2.0 * std::log(u1));
            double th = twopi * u2;
            z[2 * b] = rr * std::cos(th);
            z[2 * b + 1] = rr * std::sin(th);
        }
        double kx = t.k[q][0], ky = t.k[q][1], kz = t.k[q][2];
        double kk = std::sqrt(kx * kx + ky * ky + kz * kz);
        double ux = kx / kk, uy = ky / kk, uz = kz / kk;
        double sig = sigma0 / kk;
        // xi_c = z[2c] + i z[2c+1]
        double kr = ux * z[0] + uy * z[2] + uz * z[4];
        double ki = ux * z[1] + uy * z[3] + uz * z[5];
        double u[3] = {ux, uy, uz};
        for (int c = 0; c < 3; ++c) {
            double pr = z[2 * c] - u[c] * kr;
            double pi = z[2 * c + 1] - u[c] * ki;
            double* m = modes + (q * 3 + c) * 2;
            m[0] = alpha * m[0] + beta * sig * pr;
            m[1] = alpha * m[1] + beta * sig * pi;
        }
    }
}

void orc_accel_f64(const orc_params* p, const double* modes, double ramp, double* a3) {
    Forcer<double> f(p, modes);
    Grid g(p);
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                double a[3];
                f.accel(i, j, k, ramp, a);
                for (int c = 0; c < 3; ++c) a3[(size_t)c * g.n + g.idx(i, j, k)] = a[c];
            }
}

int orc_step_unsplit_f64(const orc_params* p, const orc_step_args* a, const double* uold, double* unew) {
    step_unsplit<double>(p, a, uold, unew); return 0;
}
int orc_jvp_unsplit_f64(const orc_params* p, const orc_step_args* a, const double* uold, int32_t ndir,
                        const double* duold, const double* amp_rel, double* unew, double* dunew) {
    if (ndir < 1 || ndir > ORC_JVP_MAXDIR) return 1;
    const size_t n = (size_t)p->nx * p->ny * p->nz * 9;
    std::vector<Tan> in(n), out(n);
    for (size_t i = 0; i < n; ++i) {
        in[i] = Tan(uold[i]);
        for (int k = 0; k < ndir; ++k) in[i].d[k] = duold ? duold[(size_t)k * n + i] : 0.0;
    }
    double rel[ORC_JVP_MAXDIR] = {0};
    bool any = false;
    for (int k = 0; k < ndir && amp_rel; ++k) { rel[k] = amp_rel[k]; any = any || rel[k] != 0.0; }
    step_unsplit<Tan>(p, a, in.data(), out.data(), any ? rel : nullptr);
    for (size_t i = 0; i < n; ++i) {
        if (unew) unew[i] = out[i].v;
        for (int k = 0; k < ndir; ++k) dunew[(size_t)k * n + i] = out[i].d[k];
    }
    return 0;
}
int orc_step_unsplit_f32(const orc_params* p, const orc_step_args* a, const float* uold, float* unew) {
    step_unsplit<float>(p, a, uold, unew); return 0;
}
int orc_step_march1d_f64(const orc_params* p, const orc_step_args* a, const double* uold, double* unew) {
    step_march1d<double>(p, a, uold, unew); return 0;
}
int orc_step_march1d_f32(const orc_params* p, const orc_step_args* a, const float* uold, float* unew) {
    step_march1d<float>(p, a, uold, unew); return 0;
}
int orc_ct_step_f64(const orc_params* p, const orc_step_args* a, const double* qold, double* qnew) {
    step_ct<double>(p, a, qold, qnew); return 0;
}
int orc_ct_step_f32(const orc_params* p, const orc_step_args* a, const float* qold, float* qnew) {
    step_ct<float>(p, a, qold, qnew); return 0;
}
void orc_cfl_f64(const orc_params* p, const double* u, double* out) { cfl<double>(p, u, out); }
void orc_cfl_f32(const orc_params* p, const float* u, double* out) { cfl<float>(p, u, out); }

void orc_ct_cfl_f64(const orc_params* p, const double* q, double* out) {
    Grid g(p);
    const size_t n = g.n;
    std::vector<double> u(9 * n);
    for (size_t c = 0; c < 5 * n; ++c) u[c] = q[c];
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                size_t c = g.idx(i, j, k);
                u[5 * n + c] = 0.5 * (q[5 * n + c] + q[5 * n + g.idx(Grid::wr(i + 1, g.nx), j, k)]);
                u[6 * n + c] = 0.5 * (q[6 * n + c] + q[6 * n + g.idx(i, Grid::wr(j + 1, g.ny), k)]);
                u[7 * n + c] = 0.5 * (q[7 * n + c] + q[7 * n + g.idx(i, j, Grid::wr(k + 1, g.nz))]);
                u[8 * n + c] = 0.0;
            }
    cfl<double>(p, u.data(), out);
}

void orc_diag_f64(const orc_params* p, const double* u, orc_diag* d) { diag<double>(p, u, d); }
void orc_diag_f32(const orc_params* p, const float* u, orc_diag* d) { diag<float>(p, u, d); }

// face div B max (ct_mhd.jl:190-194): (upper - lower)/dx per dim
double orc_ct_divb_max_f64(const orc_params* p, const double* q) {
    Grid g(p);
    const size_t n = g.n;
    const double dx = p->boxlen / p->nx;
    const double* bx = q + 5 * n; const double* by = q + 6 * n; const double* bz = q + 7 * n;
    double m = 0.0;
#pragma omp parallel for num_threads(nthreads()) reduction(max : m) schedule(static)
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                size_t c = g.idx(i, j, k);
                double d = (bx[g.idx(Grid::wr(i + 1, g.nx), j, k)] - bx[c] + by[g.idx(i, Grid::wr(j + 1, g.ny), k)] -
                            by[c] + bz[g.idx(i, j, Grid::wr(k + 1, g.nz))] - bz[c]) / dx;
                m = std::max(m, std::fabs(d));
            }
    return m;
}

// Orszag-Tang (glmmhd_turb.jl:2021-2036), 0-based centres x = (i+1/2)/N
void orc_ic_ot_f64(const orc_params* p, double* u) {
    Grid g(p);
    const double pi = 3.14159265358979323846, twopi = 2.0 * pi, gamma = p->gamma;
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                double x = (i + 0.5) / g.nx, y = (j + 0.5) / g.ny;
                double rho = 25.0 / (36.0 * pi), pr = 5.0 / (12.0 * pi);
                double vx = -std::sin(twopi * y), vy = std::sin(twopi * x), vz = 0.0;
                double sb = 1.0 / std::sqrt(4.0 * pi);
                double bx = -sb * std::sin(twopi * y), by = sb * std::sin(2.0 * twopi * x), bz = 0.0;
                double ekin = 0.5 * rho * (vx * vx + vy * vy + vz * vz), emag = 0.5 * (bx * bx + by * by + bz * bz);
                size_t c = g.idx(i, j, k);
                double v9[9] = {rho, rho * vx, rho * vy, rho * vz, pr / (gamma - 1.0) + ekin + emag, bx, by, bz, 0.0};
                for (int v = 0; v < 9; ++v) u[(size_t)v * g.n + c] = v9[v];
            }
}

void orc_ic_uniform_f64(const orc_params* p, double rho0, double p0, double bx0, double by0, double bz0, double* u) {
    Grid g(p);
    double e = p0 / (p->gamma - 1.0) + 0.5 * (bx0 * bx0 + by0 * by0 + bz0 * bz0);
    double v9[9] = {rho0, 0, 0, 0, e, bx0, by0, bz0, 0};
    for (int v = 0; v < 9; ++v)
        for (size_t c = 0; c < g.n; ++c) u[(size_t)v * g.n + c] = v9[v];
}

// Orszag-Tang with face B from the corner vector potential Az (discrete div B = 0)
void orc_ct_ic_ot_f64(const orc_params* p, double* q) {
    Grid g(p);
    const size_t n = g.n;
    const double pi = 3.14159265358979323846, twopi = 2.0 * pi, gamma = p->gamma;
    const double sb = 1.0 / std::sqrt(4.0 * pi);
    auto Az = [&](double x, double y) { return sb * (std::cos(twopi * y) / twopi + std::cos(2.0 * twopi * x) / (2.0 * twopi)); };
    const double dx = 1.0 / g.nx, dy = 1.0 / g.ny;
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                size_t c = g.idx(i, j, k);
                double xl = i * dx, yl = j * dy;
                double bxf = (Az(xl, yl + dy) - Az(xl, yl)) / dy;
                double byf = -(Az(xl + dx, yl) - Az(xl, yl)) / dx;
                q[5 * n + c] = bxf; q[6 * n + c] = byf; q[7 * n + c] = 0.0;
            }
    for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
                size_t c = g.idx(i, j, k);
                double x = (i + 0.5) * dx, y = (j + 0.5) * dy;
                double rho = 25.0 / (36.0 * pi), pr = 5.0 / (12.0 * pi);
                double vx = -std::sin(twopi * y), vy = std::sin(twopi * x);
                double bx = 0.5 * (q[5 * n + c] + q[5 * n + g.idx(Grid::wr(i + 1, g.nx), j, k)]);
                double by = 0.5 * (q[6 * n + c] + q[6 * n + g.idx(i, Grid::wr(j + 1, g.ny), k)]);
                double ekin = 0.5 * rho * (vx * vx + vy * vy), emag = 0.5 * (bx * bx + by * by);
                q[c] = rho; q[n + c] = rho * vx; q[2 * n + c] = rho * vy; q[3 * n + c] = 0.0;
                q[4 * n + c] = pr / (gamma - 1.0) + ekin + emag;
            }
}

}  // extern "C"
