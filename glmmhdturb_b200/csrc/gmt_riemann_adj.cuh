// gmt_riemann_adj.cuh -- hand-written reverse sweeps of the step's physics functions: cons2prim and
// prim2cons, the ideal-MHD flux, the fast speed, HLL and the Miyoshi-Kusano HLLD (gmt_phys.cuh;
// glmmhd_turb.jl:68-115, 193-272, 335-354), and of riemann_glm (GLM pair and state floors) in the
// x-normal frame.
//
// Each function re-evaluates the forward expressions it needs and then propagates the adjoint of
// its outputs back to its inputs.  The branch conventions are those of the dual numbers and of
// the oracle's tangent step: max(a, b) passes the derivative of a when a >= b, min(a, b) of a when
// a <= b, |a| takes the sign of a >= 0, sqrt has derivative 0 at 0, and the degenerate star state
// (|denK| < 1e-12) and the fan region follow the branch the values take.  The exact-speed LLF
// paths are not covered here (riemann_x_adj returns false and the caller uses dual numbers).
#pragma once
#include "gmt_phys.cuh"

namespace gmt {

template <class R> GMT_HD R sel_ge(R a, R b) { return a >= b ? R(1) : R(0); }   // d max(a, b) / da
template <class R> GMT_HD R sel_le(R a, R b) { return a <= b ? R(1) : R(0); }   // d min(a, b) / da

// qb[0,4,5,6,7], bnb += adjoint of fast_speed(q, gamma, bn) for output adjoint cb
template <class R> GMT_HD void fast_speed_adj(const Q9<R>& q, R gamma, R bn, R cb, Q9<R>& qb, R& bnb) {
    const R rho = q.v[0];
    const R c2 = gamma * q.v[4] / rho;
    const R bsq = q.v[5] * q.v[5] + q.v[6] * q.v[6] + q.v[7] * q.v[7];
    const R b2 = bsq / rho;
    const R d2 = R(0.5) * (b2 + c2);
    const R disc = d2 * d2 - c2 * bn * bn / rho;
    const R dm = rmax(disc, R(0));
    const R sd = sqrt_r(dm);
    const R cf = sqrt_r(d2 + sd);
    const R t_b = cf > R(0) ? cb * (R(0.5) / cf) : R(0);
    R d2_b = t_b;
    const R dm_b = sd > R(0) ? t_b * (R(0.5) / sd) : R(0);
    const R disc_b = dm_b * sel_ge(disc, R(0));
    d2_b += disc_b * R(2) * d2;
    R c2_b = -disc_b * (bn * bn / rho);
    bnb += -disc_b * c2 * R(2) * bn / rho;
    R rho_b = disc_b * (c2 * bn * bn / (rho * rho));
    const R b2_b = R(0.5) * d2_b;
    c2_b += R(0.5) * d2_b;
    const R bsq_b = b2_b / rho;
    rho_b += -b2_b * b2 / rho;
    qb.v[5] += bsq_b * R(2) * q.v[5];
    qb.v[6] += bsq_b * R(2) * q.v[6];
    qb.v[7] += bsq_b * R(2) * q.v[7];
    qb.v[4] += c2_b * gamma / rho;
    rho_b += -c2_b * c2 / rho;
    qb.v[0] += rho_b;
}

// qb += adjoint of phys_flux_x(q, gamma) (F[Bx] = F[psi] = 0) for output adjoint fb
template <class R> GMT_HD void phys_flux_x_adj(const Q9<R>& q, R gamma, const Q9<R>& fb, Q9<R>& qb) {
    const R rho = q.v[0], vx = q.v[1], vy = q.v[2], vz = q.v[3], p = q.v[4];
    const R bx = q.v[5], by = q.v[6], bz = q.v[7];
    const R b2 = bx * bx + by * by + bz * bz;
    const R ptot = p + R(0.5) * b2;
    const R vsq = vx * vx + vy * vy + vz * vz;
    const R E = p / (gamma - R(1)) + R(0.5) * rho * vsq + R(0.5) * b2;
    const R vdotb = vx * bx + vy * by + vz * bz;
    const R f0 = fb.v[0], f1 = fb.v[1], f2 = fb.v[2], f3 = fb.v[3], f4 = fb.v[4], f6 = fb.v[6], f7 = fb.v[7];
    R rho_b = f0 * vx + f1 * vx * vx + f2 * vx * vy + f3 * vx * vz;
    R vx_b = f0 * rho + f1 * R(2) * rho * vx + f2 * rho * vy + f3 * rho * vz + f4 * (E + ptot) + f6 * by + f7 * bz;
    R vy_b = f2 * rho * vx - f6 * bx;
    R vz_b = f3 * rho * vx - f7 * bx;
    const R ptot_b = f1 + f4 * vx;
    const R E_b = f4 * vx;
    const R vdotb_b = -f4 * bx;
    R bx_b = -R(2) * f1 * bx - f2 * by - f3 * bz - f4 * vdotb - f6 * vy - f7 * vz;
    R by_b = -f2 * bx + f6 * vx;
    R bz_b = -f3 * bx + f7 * vx;
    vx_b += vdotb_b * bx; vy_b += vdotb_b * by; vz_b += vdotb_b * bz;
    bx_b += vdotb_b * vx; by_b += vdotb_b * vy; bz_b += vdotb_b * vz;
    R p_b = E_b / (gamma - R(1)) + ptot_b;
    rho_b += E_b * R(0.5) * vsq;
    vx_b += E_b * rho * vx; vy_b += E_b * rho * vy; vz_b += E_b * rho * vz;
    const R b2_b = R(0.5) * E_b + R(0.5) * ptot_b;
    bx_b += b2_b * R(2) * bx; by_b += b2_b * R(2) * by; bz_b += b2_b * R(2) * bz;
    qb.v[0] += rho_b; qb.v[1] += vx_b; qb.v[2] += vy_b; qb.v[3] += vz_b; qb.v[4] += p_b;
    qb.v[5] += bx_b; qb.v[6] += by_b; qb.v[7] += bz_b;
}

// cb += adjoint of cons2prim(c, gamma, smallr, pf) for output adjoint qb
template <class R>
GMT_HD void cons2prim_adj(const Q9<R>& c, R gamma, R smallr, R pf, const Q9<R>& qb, Q9<R>& cb) {
    const R rho = rmax(c.v[0], smallr);
    const R ir = R(1) / rho;
    const R msq = c.v[1] * c.v[1] + c.v[2] * c.v[2] + c.v[3] * c.v[3];
    const R ekin = R(0.5) * msq * ir;
    const R emag = R(0.5) * (c.v[5] * c.v[5] + c.v[6] * c.v[6] + c.v[7] * c.v[7]);
    const R pr = (gamma - R(1)) * (c.v[4] - ekin - emag);
    const R pr_b = qb.v[4] * sel_ge(pr, pf);
    const R g1 = pr_b * (gamma - R(1));
    const R ekin_b = -g1, emag_b = -g1;
    cb.v[4] += g1;
    cb.v[5] += qb.v[5] + emag_b * c.v[5];
    cb.v[6] += qb.v[6] + emag_b * c.v[6];
    cb.v[7] += qb.v[7] + emag_b * c.v[7];
    cb.v[8] += qb.v[8];
    cb.v[1] += qb.v[1] * ir + ekin_b * c.v[1] * ir;
    cb.v[2] += qb.v[2] * ir + ekin_b * c.v[2] * ir;
    cb.v[3] += qb.v[3] * ir + ekin_b * c.v[3] * ir;
    const R ir_b = qb.v[1] * c.v[1] + qb.v[2] * c.v[2] + qb.v[3] * c.v[3] + ekin_b * R(0.5) * msq;
    const R rho_b = qb.v[0] - ir_b * ir * ir;
    cb.v[0] += rho_b * sel_ge(c.v[0], smallr);
}

// qb += adjoint of prim2cons(q, gamma) for output adjoint ub (the psi slot passes through)
template <class R> GMT_HD void prim2cons_adj(const Q9<R>& q, R gamma, const Q9<R>& ub, Q9<R>& qb) {
    const R rho = q.v[0], vx = q.v[1], vy = q.v[2], vz = q.v[3];
    const R vsq = vx * vx + vy * vy + vz * vz;
    const R E_b = ub.v[4];
    qb.v[0] += ub.v[0] + ub.v[1] * vx + ub.v[2] * vy + ub.v[3] * vz + E_b * R(0.5) * vsq;
    qb.v[1] += ub.v[1] * rho + E_b * rho * vx;
    qb.v[2] += ub.v[2] * rho + E_b * rho * vy;
    qb.v[3] += ub.v[3] * rho + E_b * rho * vz;
    qb.v[4] += E_b / (gamma - R(1));
    qb.v[5] += ub.v[5] + E_b * q.v[5];
    qb.v[6] += ub.v[6] + E_b * q.v[6];
    qb.v[7] += ub.v[7] + E_b * q.v[7];
    qb.v[8] += ub.v[8];
}

// HLL (hll_x): Lb, Rb, bnb += adjoint for flux adjoint fb; f[5], f[8] are the GLM fluxes set by the
// caller, so fb[5], fb[8] do not enter
template <class R>
GMT_HD void hll_x_adj(const Q9<R>& L, const Q9<R>& Rr, R gamma, R bn, const Q9<R>& fb, Q9<R>& Lb, Q9<R>& Rb, R& bnb) {
    const R cfL = fast_speed(L, gamma, bn), cfR = fast_speed(Rr, gamma, bn);
    const R aL = L.v[1] - cfL, aR = Rr.v[1] - cfR;
    const R m = rmin(aL, aR);
    const R SL = rmin(m, R(0));
    const R bL = L.v[1] + cfL, bR = Rr.v[1] + cfR;
    const R M = rmax(bL, bR);
    const R SR = rmax(M, R(0));
    const Q9<R> fL = phys_flux_x(L, gamma), fR = phys_flux_x(Rr, gamma);
    const Q9<R> uL = prim2cons(L, gamma), uR = prim2cons(Rr, gamma);
    const R ihd = R(1) / (SR - SL);
    Q9<R> fLb, fRb, uLb, uRb;
    R SL_b = R(0), SR_b = R(0), ihd_b = R(0);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const R g = (i == 5 || i == 8) ? R(0) : fb.v[i];
        const R num = SR * fL.v[i] - SL * fR.v[i] + SL * SR * (uR.v[i] - uL.v[i]);
        ihd_b += g * num;
        const R nb = g * ihd;
        SR_b += nb * fL.v[i] + nb * SL * (uR.v[i] - uL.v[i]);
        SL_b += -nb * fR.v[i] + nb * SR * (uR.v[i] - uL.v[i]);
        fLb.v[i] = nb * SR;
        fRb.v[i] = -nb * SL;
        uRb.v[i] = nb * SL * SR;
        uLb.v[i] = -nb * SL * SR;
    }
    // ihd = 1 / (SR - SL)
    const R dd_b = -ihd_b * ihd * ihd;
    SR_b += dd_b;
    SL_b -= dd_b;
    phys_flux_x_adj(L, gamma, fLb, Lb);
    phys_flux_x_adj(Rr, gamma, fRb, Rb);
    prim2cons_adj(L, gamma, uLb, Lb);
    prim2cons_adj(Rr, gamma, uRb, Rb);
    // SL = min(min(aL, aR), 0), SR = max(max(bL, bR), 0)
    const R m_b = SL_b * sel_le(m, R(0));
    const R aL_b = m_b * sel_le(aL, aR), aR_b = m_b - aL_b;
    const R M_b = SR_b * sel_ge(M, R(0));
    const R bL_b = M_b * sel_ge(bL, bR), bR_b = M_b - bL_b;
    Lb.v[1] += aL_b + bL_b;
    Rb.v[1] += aR_b + bR_b;
    fast_speed_adj(L, gamma, bn, -aL_b + bL_b, Lb, bnb);
    fast_speed_adj(Rr, gamma, bn, -aR_b + bR_b, Rb, bnb);
}

// HLLD star state (hlld_star) and its reverse
template <class R>
GMT_HD void hlld_star_adj(R d, R u, R v, R w, R by, R bz, R S, R SM, R bn, R vy_b, R vz_b, R byS_b, R bzS_b, R& d_b,
                          R& u_b, R& v_b, R& w_b, R& by_b, R& bz_b, R& S_b, R& SM_b, R& bn_b) {
    const R a = S - u, b = S - SM;
    const R denK = d * a * b - bn * bn;
    if (rabs(denK) < R(1e-12)) {
        v_b += vy_b; w_b += vz_b; by_b += byS_b; bz_b += bzS_b;
        return;
    }
    const R fac = bn * (SM - u) / denK;
    const R num = d * a * a - bn * bn;
    const R byS = by * num / denK, bzS = bz * num / denK;
    v_b += vy_b;
    w_b += vz_b;
    by_b += -vy_b * fac + byS_b * num / denK;
    bz_b += -vz_b * fac + bzS_b * num / denK;
    const R fac_b = -vy_b * by - vz_b * bz;
    const R num_b = (byS_b * by + bzS_b * bz) / denK;
    R denK_b = -(byS_b * byS + bzS_b * bzS) / denK - fac_b * fac / denK;
    bn_b += fac_b * (SM - u) / denK;
    SM_b += fac_b * bn / denK;
    u_b += -fac_b * bn / denK;
    d_b += num_b * a * a + denK_b * a * b;
    const R a_b = num_b * R(2) * d * a + denK_b * d * b;
    const R b_b = denK_b * d * a;
    bn_b += -num_b * R(2) * bn - denK_b * R(2) * bn;
    S_b += a_b + b_b;
    u_b += -a_b;
    SM_b += -b_b;
}

// one side of the HLLD fan: the side's primitive state and its star quantities
template <class R> struct HSide {
    R d, u, v, w, p, by, bz, E, pt, S;
    R vys, vzs, bys, bzs, vdotb, vdotbs, Es;
};
template <class R> struct HSideB {
    R d, u, v, w, p, by, bz, E, pt, S, vys, vzs, bys, bzs, vdotbs, Es;
};

template <class R> GMT_HD void hside_zero(HSideB<R>& b) {
    b.d = b.u = b.v = b.w = b.p = b.by = b.bz = b.E = b.pt = b.S = R(0);
    b.vys = b.vzs = b.bys = b.bzs = b.vdotbs = b.Es = R(0);
}

template <class R> GMT_HD void hside_star(HSide<R>& s, R SM, R pts, R bn) {
    hlld_star(s.d, s.u, s.v, s.w, s.by, s.bz, s.S, SM, bn, s.vys, s.vzs, s.bys, s.bzs);
    s.vdotb = s.u * bn + s.v * s.by + s.w * s.bz;
    s.vdotbs = SM * bn + s.vys * s.bys + s.vzs * s.bzs;
    s.Es = ((s.S - s.u) * s.E - s.pt * s.u + pts * SM + bn * (s.vdotb - s.vdotbs)) / (s.S - SM);
}

// reverse of hside_star: from b.vys..b.bzs, b.vdotbs, b.Es to the side inputs, SM, pts, bn
template <class R> GMT_HD void hside_star_adj(const HSide<R>& s, R SM, R pts, R bn, HSideB<R>& b, R& SM_b, R& pts_b,
                                              R& bn_b) {
    const R den = s.S - SM;
    const R num_b = b.Es / den;
    const R den_b = -b.Es * s.Es / den;
    b.S += den_b + num_b * s.E;
    SM_b += -den_b + num_b * pts;
    b.u += -num_b * s.E - num_b * s.pt;
    b.E += num_b * (s.S - s.u);
    b.pt += -num_b * s.u;
    pts_b += num_b * SM;
    bn_b += num_b * (s.vdotb - s.vdotbs);
    const R vdotb_b = num_b * bn;
    const R vdotbs_b = b.vdotbs - num_b * bn;
    SM_b += vdotbs_b * bn;
    bn_b += vdotbs_b * SM;
    b.vys += vdotbs_b * s.bys; b.bys += vdotbs_b * s.vys;
    b.vzs += vdotbs_b * s.bzs; b.bzs += vdotbs_b * s.vzs;
    b.u += vdotb_b * bn; bn_b += vdotb_b * s.u;
    b.v += vdotb_b * s.by; b.by += vdotb_b * s.v;
    b.w += vdotb_b * s.bz; b.bz += vdotb_b * s.w;
    hlld_star_adj(s.d, s.u, s.v, s.w, s.by, s.bz, s.S, SM, bn, b.vys, b.vzs, b.bys, b.bzs, b.d, b.u, b.v, b.w, b.by,
                  b.bz, b.S, SM_b, bn_b);
}

// adjoint of U = {d, d u, d v, d w, E, bn, by, bz, 0} (the side's conserved state) for ub
template <class R> GMT_HD void hside_u_adj(const HSide<R>& s, const R* ub, HSideB<R>& b, R& bn_b) {
    b.d += ub[0] + ub[1] * s.u + ub[2] * s.v + ub[3] * s.w;
    b.u += ub[1] * s.d; b.v += ub[2] * s.d; b.w += ub[3] * s.d;
    b.E += ub[4]; bn_b += ub[5]; b.by += ub[6]; b.bz += ub[7];
}

// outer region of the HLLD fan on side s: F = F_s + S_s (U*_s - U_s)
template <class R>
GMT_HD void hlld_outer_adj(HSide<R>& s, HSideB<R>& b, R ds, R SM, R pts, R bn, const R* g, Q9<R>& Fb, R& ds_b,
                           R& SM_b, R& pts_b, R& bn_b) {
    hside_star(s, SM, pts, bn);
    const R Us[9] = {ds, ds * SM, ds * s.vys, ds * s.vzs, s.Es, bn, s.bys, s.bzs, R(0)};
    const R U[9] = {s.d, s.d * s.u, s.d * s.v, s.d * s.w, s.E, bn, s.by, s.bz, R(0)};
    R Usb[9], Ub[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        b.S += g[i] * (Us[i] - U[i]);
        Usb[i] = g[i] * s.S;
        Ub[i] = -g[i] * s.S;
        Fb.v[i] = g[i];
    }
    ds_b += Usb[0] + Usb[1] * SM + Usb[2] * s.vys + Usb[3] * s.vzs;
    SM_b += Usb[1] * ds;
    b.vys += Usb[2] * ds;
    b.vzs += Usb[3] * ds;
    b.Es += Usb[4];
    bn_b += Usb[5];
    b.bys += Usb[6];
    b.bzs += Usb[7];
    hside_u_adj(s, Ub, b, bn_b);
    hside_star_adj(s, SM, pts, bn, b, SM_b, pts_b, bn_b);
}

// inner region: F = F_s + S*s Uss - (S*s - S_s) Us - S_s U on the sampled side s (LO: the left
// side, SM >= 0; else the right side); both star states are already evaluated
template <bool LO, class R>
GMT_HD void hlld_inner_adj(const HSide<R>& sl, const HSide<R>& sr, HSideB<R>& bl, HSideB<R>& br, R ds, R sqdLs,
                           R sqdRs, R Ssx, R SM, R pts, R bn, const R* g, Q9<R>& Fb, R& ds_b, R& sqdLs_b, R& sqdRs_b,
                           R& Ssx_b, R& SM_b, R& bn_b) {
    const HSide<R>& s = LO ? sl : sr;
    HSideB<R>& b = LO ? bl : br;
    const R sgn = bn >= R(0) ? R(1) : R(-1);
    const R ssum = sqdLs + sqdRs;
    const R invsum = R(1) / ssum;
    const R nvy = sqdLs * sl.vys + sqdRs * sr.vys + (sr.bys - sl.bys) * sgn;
    const R nvz = sqdLs * sl.vzs + sqdRs * sr.vzs + (sr.bzs - sl.bzs) * sgn;
    const R nby = sqdLs * sr.bys + sqdRs * sl.bys + sqdLs * sqdRs * (sr.vys - sl.vys) * sgn;
    const R nbz = sqdLs * sr.bzs + sqdRs * sl.bzs + sqdLs * sqdRs * (sr.vzs - sl.vzs) * sgn;
    const R vyss = nvy * invsum, vzss = nvz * invsum, byss = nby * invsum, bzss = nbz * invsum;
    const R vdotbss = SM * bn + vyss * byss + vzss * bzss;
    const R sq = LO ? sqdLs : sqdRs;
    const R sign_e = LO ? R(-1) : R(1);   // ELss = ELs - sq(.)sgn, ERss = ERs + sq(.)sgn
    const R Ess = s.Es + sign_e * (sq * (s.vdotbs - vdotbss) * sgn);
    const R Uss[9] = {ds, ds * SM, ds * vyss, ds * vzss, Ess, bn, byss, bzss, R(0)};
    const R Us[9] = {ds, ds * SM, ds * s.vys, ds * s.vzs, s.Es, bn, s.bys, s.bzs, R(0)};
    const R U[9] = {s.d, s.d * s.u, s.d * s.v, s.d * s.w, s.E, bn, s.by, s.bz, R(0)};
    R Ussb[9], Usb[9], Ub[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        Ssx_b += g[i] * (Uss[i] - Us[i]);
        b.S += g[i] * (Us[i] - U[i]);
        Ussb[i] = g[i] * Ssx;
        Usb[i] = -g[i] * (Ssx - s.S);
        Ub[i] = -g[i] * s.S;
        Fb.v[i] = g[i];
    }
    // Uss
    ds_b += Ussb[0] + Ussb[1] * SM + Ussb[2] * vyss + Ussb[3] * vzss;
    SM_b += Ussb[1] * ds;
    R vyss_b = Ussb[2] * ds, vzss_b = Ussb[3] * ds;
    const R Ess_b = Ussb[4];
    bn_b += Ussb[5];
    R byss_b = Ussb[6], bzss_b = Ussb[7];
    // Ess = Es + sign_e * sq * (vdotbs - vdotbss) * sgn
    b.Es += Ess_b;
    (LO ? sqdLs_b : sqdRs_b) += Ess_b * sign_e * (s.vdotbs - vdotbss) * sgn;
    b.vdotbs += Ess_b * sign_e * sq * sgn;
    const R vdotbss_b = -Ess_b * sign_e * sq * sgn;
    // vdotbss = SM bn + vyss byss + vzss bzss
    SM_b += vdotbss_b * bn;
    bn_b += vdotbss_b * SM;
    vyss_b += vdotbss_b * byss; byss_b += vdotbss_b * vyss;
    vzss_b += vdotbss_b * bzss; bzss_b += vdotbss_b * vzss;
    // Us (the sampled side's star state) and U
    ds_b += Usb[0] + Usb[1] * SM + Usb[2] * s.vys + Usb[3] * s.vzs;
    SM_b += Usb[1] * ds;
    b.vys += Usb[2] * ds;
    b.vzs += Usb[3] * ds;
    b.Es += Usb[4];
    bn_b += Usb[5];
    b.bys += Usb[6];
    b.bzs += Usb[7];
    hside_u_adj(s, Ub, b, bn_b);
    // the double-star averages
    const R invsum_b = vyss_b * nvy + vzss_b * nvz + byss_b * nby + bzss_b * nbz;
    const R tvy = vyss_b * invsum, tvz = vzss_b * invsum, tby = byss_b * invsum, tbz = bzss_b * invsum;
    sqdLs_b += tvy * sl.vys + tvz * sl.vzs + tby * sr.bys + tbz * sr.bzs + tby * sqdRs * (sr.vys - sl.vys) * sgn +
               tbz * sqdRs * (sr.vzs - sl.vzs) * sgn;
    sqdRs_b += tvy * sr.vys + tvz * sr.vzs + tby * sl.bys + tbz * sl.bzs + tby * sqdLs * (sr.vys - sl.vys) * sgn +
               tbz * sqdLs * (sr.vzs - sl.vzs) * sgn;
    bl.vys += tvy * sqdLs - tby * sqdLs * sqdRs * sgn;
    br.vys += tvy * sqdRs + tby * sqdLs * sqdRs * sgn;
    bl.vzs += tvz * sqdLs - tbz * sqdLs * sqdRs * sgn;
    br.vzs += tvz * sqdRs + tbz * sqdLs * sqdRs * sgn;
    bl.bys += -tvy * sgn + tby * sqdRs;
    br.bys += tvy * sgn + tby * sqdLs;
    bl.bzs += -tvz * sgn + tbz * sqdRs;
    br.bzs += tvz * sgn + tbz * sqdLs;
    const R ssum_b = -invsum_b * invsum * invsum;
    sqdLs_b += ssum_b;
    sqdRs_b += ssum_b;
}

// HLLD (hlld_x): Lb, Rb, bnb += adjoint for flux adjoint fb (fb[5], fb[8] do not enter)
template <class R>
GMT_HD void hlld_x_adj(const Q9<R>& L, const Q9<R>& Rr, R gamma, R bn, const Q9<R>& fb, Q9<R>& Lb, Q9<R>& Rb, R& bnb) {
    const R tiny = R(1e-12);
    HSide<R> sl, sr;
    sl.d = L.v[0]; sl.u = L.v[1]; sl.v = L.v[2]; sl.w = L.v[3]; sl.p = L.v[4]; sl.by = L.v[6]; sl.bz = L.v[7];
    sr.d = Rr.v[0]; sr.u = Rr.v[1]; sr.v = Rr.v[2]; sr.w = Rr.v[3]; sr.p = Rr.v[4]; sr.by = Rr.v[6]; sr.bz = Rr.v[7];
    const R b2L = bn * bn + sl.by * sl.by + sl.bz * sl.bz;
    const R b2R = bn * bn + sr.by * sr.by + sr.bz * sr.bz;
    sl.pt = sl.p + R(0.5) * b2L;
    sr.pt = sr.p + R(0.5) * b2R;
    sl.E = sl.p / (gamma - R(1)) + R(0.5) * sl.d * (sl.u * sl.u + sl.v * sl.v + sl.w * sl.w) + R(0.5) * b2L;
    sr.E = sr.p / (gamma - R(1)) + R(0.5) * sr.d * (sr.u * sr.u + sr.v * sr.v + sr.w * sr.w) + R(0.5) * b2R;
    const R cfL = fast_speed(L, gamma, bn), cfR = fast_speed(Rr, gamma, bn);
    const R umin = rmin(sl.u, sr.u), umax = rmax(sl.u, sr.u), cmax = rmax(cfL, cfR);
    const R xL = umin - cmax, xR = umax + cmax;
    sl.S = rmin(xL, R(0));
    sr.S = rmax(xR, R(0));
    const R aL = sl.S - sl.u, aR = sr.S - sr.u;
    const R den = aR * sr.d - aL * sl.d;
    const R SM = (aR * sr.d * sr.u - aL * sl.d * sl.u - sr.pt + sl.pt) / den;
    const R du = sr.u - sl.u;
    const R pts = (aR * sr.d * sl.pt - aL * sl.d * sr.pt + sl.d * sr.d * aR * aL * du) / den;
    const R qL = sl.d * aL / (sl.S - SM), qR = sr.d * aR / (sr.S - SM);
    const R dLs = rmax(qL, tiny), dRs = rmax(qR, tiny);
    const R sqdLs = sqrt_r(dLs), sqdRs = sqrt_r(dRs);
    const R abn = rabs(bn);
    const R SLs = SM - abn / sqdLs;
    const R SRs = SM + abn / sqdRs;

    R g[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) g[i] = (i == 5 || i == 8) ? R(0) : fb.v[i];
    HSideB<R> bl, br;
    hside_zero(bl);
    hside_zero(br);
    R SM_b = R(0), pts_b = R(0), bn_b = R(0), SLs_b = R(0), SRs_b = R(0), dLs_b = R(0), dRs_b = R(0);
    R sqdLs_b = R(0), sqdRs_b = R(0);
    Q9<R> FLb, FRb;
#pragma unroll
    for (int i = 0; i < 9; ++i) { FLb.v[i] = R(0); FRb.v[i] = R(0); }
    if (SLs >= R(0)) {
        hlld_outer_adj(sl, bl, dLs, SM, pts, bn, g, FLb, dLs_b, SM_b, pts_b, bn_b);
    } else if (SRs < R(0)) {
        hlld_outer_adj(sr, br, dRs, SM, pts, bn, g, FRb, dRs_b, SM_b, pts_b, bn_b);
    } else {
        hside_star(sl, SM, pts, bn);
        hside_star(sr, SM, pts, bn);
        if (SM >= R(0))
            hlld_inner_adj<true>(sl, sr, bl, br, dLs, sqdLs, sqdRs, SLs, SM, pts, bn, g, FLb, dLs_b, sqdLs_b, sqdRs_b,
                                 SLs_b, SM_b, bn_b);
        else
            hlld_inner_adj<false>(sl, sr, bl, br, dRs, sqdLs, sqdRs, SRs, SM, pts, bn, g, FRb, dRs_b, sqdLs_b, sqdRs_b,
                                  SRs_b, SM_b, bn_b);
        hside_star_adj(sl, SM, pts, bn, bl, SM_b, pts_b, bn_b);
        hside_star_adj(sr, SM, pts, bn, br, SM_b, pts_b, bn_b);
    }
    // SLs = SM - |bn| / sqdLs, SRs = SM + |bn| / sqdRs
    SM_b += SLs_b + SRs_b;
    const R abn_b = -SLs_b / sqdLs + SRs_b / sqdRs;
    sqdLs_b += SLs_b * abn / (sqdLs * sqdLs);
    sqdRs_b += -SRs_b * abn / (sqdRs * sqdRs);
    bn_b += abn_b * (bn >= R(0) ? R(1) : R(-1));
    // sqrt and the tiny floors
    dLs_b += sqdLs > R(0) ? sqdLs_b * (R(0.5) / sqdLs) : R(0);
    dRs_b += sqdRs > R(0) ? sqdRs_b * (R(0.5) / sqdRs) : R(0);
    const R qL_b = dLs_b * sel_ge(qL, tiny), qR_b = dRs_b * sel_ge(qR, tiny);
    {
        const R dl = sl.S - SM, num_b = qL_b / dl, dl_b = -qL_b * qL / dl;
        bl.d += num_b * aL;
        R aL_b = num_b * sl.d;
        bl.S += dl_b;
        SM_b -= dl_b;
        const R dr = sr.S - SM, numr_b = qR_b / dr, dr_b = -qR_b * qR / dr;
        br.d += numr_b * aR;
        R aR_b = numr_b * sr.d;
        br.S += dr_b;
        SM_b -= dr_b;
        // pts = (aR dR ptL - aL dL ptR + dL dR aR aL du) / den ; SM = (aR dR uR - aL dL uL - ptR + ptL) / den
        const R ptsn_b = pts_b / den;
        R den_b = -pts_b * pts / den;
        const R smn_b = SM_b / den;
        den_b += -SM_b * SM / den;
        aR_b += ptsn_b * sr.d * sl.pt + ptsn_b * sl.d * sr.d * aL * du + smn_b * sr.d * sr.u + den_b * sr.d;
        aL_b += -ptsn_b * sl.d * sr.pt + ptsn_b * sl.d * sr.d * aR * du - smn_b * sl.d * sl.u - den_b * sl.d;
        br.d += ptsn_b * aR * sl.pt + ptsn_b * sl.d * aR * aL * du + smn_b * aR * sr.u + den_b * aR;
        bl.d += -ptsn_b * aL * sr.pt + ptsn_b * sr.d * aR * aL * du - smn_b * aL * sl.u - den_b * aL;
        bl.pt += ptsn_b * aR * sr.d + smn_b;
        br.pt += -ptsn_b * aL * sl.d - smn_b;
        const R du_b = ptsn_b * sl.d * sr.d * aR * aL;
        br.u += du_b + smn_b * aR * sr.d - aR_b;
        bl.u += -du_b - smn_b * aL * sl.d - aL_b;
        bl.S += aL_b;
        br.S += aR_b;
    }
    // S_L = min(min(uL, uR) - max(cfL, cfR), 0), S_R = max(max(uL, uR) + max(cfL, cfR), 0)
    const R xL_b = bl.S * sel_le(xL, R(0)), xR_b = br.S * sel_ge(xR, R(0));
    const R umin_b = xL_b, umax_b = xR_b, cmax_b = -xL_b + xR_b;
    const R ul_min = sel_le(sl.u, sr.u), ul_max = sel_ge(sl.u, sr.u), cl_max = sel_ge(cfL, cfR);
    bl.u += umin_b * ul_min + umax_b * ul_max;
    br.u += umin_b * (R(1) - ul_min) + umax_b * (R(1) - ul_max);
    fast_speed_adj(L, gamma, bn, cmax_b * cl_max, Lb, bn_b);
    fast_speed_adj(Rr, gamma, bn, cmax_b * (R(1) - cl_max), Rb, bn_b);
    // the outer-side fluxes F_s = phys_flux_x({d, u, v, w, p, bn, by, bz, 0})
    {
        Q9<R> qLf, qRf, qLb, qRb;
#pragma unroll
        for (int i = 0; i < 9; ++i) { qLb.v[i] = R(0); qRb.v[i] = R(0); }
        qLf.v[0] = sl.d; qLf.v[1] = sl.u; qLf.v[2] = sl.v; qLf.v[3] = sl.w; qLf.v[4] = sl.p;
        qLf.v[5] = bn; qLf.v[6] = sl.by; qLf.v[7] = sl.bz; qLf.v[8] = R(0);
        qRf.v[0] = sr.d; qRf.v[1] = sr.u; qRf.v[2] = sr.v; qRf.v[3] = sr.w; qRf.v[4] = sr.p;
        qRf.v[5] = bn; qRf.v[6] = sr.by; qRf.v[7] = sr.bz; qRf.v[8] = R(0);
        phys_flux_x_adj(qLf, gamma, FLb, qLb);
        phys_flux_x_adj(qRf, gamma, FRb, qRb);
        bl.d += qLb.v[0]; bl.u += qLb.v[1]; bl.v += qLb.v[2]; bl.w += qLb.v[3]; bl.p += qLb.v[4];
        bn_b += qLb.v[5] + qRb.v[5];
        bl.by += qLb.v[6]; bl.bz += qLb.v[7];
        br.d += qRb.v[0]; br.u += qRb.v[1]; br.v += qRb.v[2]; br.w += qRb.v[3]; br.p += qRb.v[4];
        br.by += qRb.v[6]; br.bz += qRb.v[7];
    }
    // E_s = p/(gamma-1) + d|v|^2/2 + b2/2, pt_s = p + b2/2, b2_s = bn^2 + by^2 + bz^2
    {
        HSide<R>* ss[2] = {&sl, &sr};
        HSideB<R>* bb[2] = {&bl, &br};
        Q9<R>* out[2] = {&Lb, &Rb};
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const HSide<R>& s = *ss[k];
            HSideB<R>& b = *bb[k];
            const R b2_b = R(0.5) * b.E + R(0.5) * b.pt;
            b.p += b.E / (gamma - R(1)) + b.pt;
            b.d += b.E * R(0.5) * (s.u * s.u + s.v * s.v + s.w * s.w);
            b.u += b.E * s.d * s.u;
            b.v += b.E * s.d * s.v;
            b.w += b.E * s.d * s.w;
            bn_b += b2_b * R(2) * bn;
            b.by += b2_b * R(2) * s.by;
            b.bz += b2_b * R(2) * s.bz;
            Q9<R>& o = *out[k];
            o.v[0] += b.d; o.v[1] += b.u; o.v[2] += b.v; o.v[3] += b.w; o.v[4] += b.p;
            o.v[6] += b.by; o.v[7] += b.bz;
        }
    }
    bnb += bn_b;
}

// Reverse of riemann_glm<0, RIEM> (floors, GLM pair, solver; glmmhd_turb.jl:275-292): Lqb, Rqb =
// J^T fb.  Returns false for the exact-speed LLF paths, which the caller differentiates otherwise.
template <int RIEM, class R>
GMT_HD bool riemann_x_adj(const Q9<R>& Lq, const Q9<R>& Rq, const Q9<R>& fb, const Consts<R>& K, R ch, bool use_llf,
                          Q9<R>& Lqb, Q9<R>& Rqb) {
    if (RIEM != RIEM_HLLD && RIEM != RIEM_HLL) return false;
    Q9<R> L = Lq, Rr = Rq;
    L.v[0] = rmax(L.v[0], K.smallr); L.v[4] = rmax(L.v[4], K.pfl);
    Rr.v[0] = rmax(Rr.v[0], K.smallr); Rr.v[4] = rmax(Rr.v[4], K.pfl);
    if (RIEM == RIEM_HLLD) {
        const bool uself = (K.llf_dmin > R(0) && rmin(L.v[0], Rr.v[0]) < K.llf_dmin) ||
                           (K.llf_pmin > R(0) && rmin(L.v[4], Rr.v[4]) < K.llf_pmin) || use_llf;
        if (uself) return false;
    }
    R bns, psis;
    glm_pair(L.v[5], Rr.v[5], L.v[8], Rr.v[8], ch, bns, psis);
    L.v[5] = bns;
    Rr.v[5] = bns;
    Q9<R> Lb, Rb;
#pragma unroll
    for (int i = 0; i < 9; ++i) { Lb.v[i] = R(0); Rb.v[i] = R(0); }
    R bnb = R(0);
    if (RIEM == RIEM_HLLD) hlld_x_adj(L, Rr, K.gamma, bns, fb, Lb, Rb, bnb);
    else hll_x_adj(L, Rr, K.gamma, bns, fb, Lb, Rb, bnb);
    // f[5] = psis, f[8] = ch^2 bns; the solver's L[5] = R[5] = bns
    const R bns_b = bnb + Lb.v[5] + Rb.v[5] + fb.v[8] * ch * ch;
    const R psis_b = fb.v[5];
    Lb.v[5] = R(0.5) * bns_b + R(0.5) * ch * psis_b;
    Rb.v[5] = R(0.5) * bns_b - R(0.5) * ch * psis_b;
    Lb.v[8] += R(0.5) * bns_b / ch + R(0.5) * psis_b;
    Rb.v[8] += -R(0.5) * bns_b / ch + R(0.5) * psis_b;
    Lqb = Lb;
    Rqb = Rb;
    Lqb.v[0] = Lb.v[0] * sel_ge(Lq.v[0], K.smallr);
    Lqb.v[4] = Lb.v[4] * sel_ge(Lq.v[4], K.pfl);
    Rqb.v[0] = Rb.v[0] * sel_ge(Rq.v[0], K.smallr);
    Rqb.v[4] = Rb.v[4] * sel_ge(Rq.v[4], K.pfl);
    return true;
}


// Reverse sweep of the update epilogue finish_update (void floor, psi damping, forcing kick;
// glmmhd_turb.jl:450-475): given the output adjoint ob, the adjoint rb of the pre-epilogue state
// r and ab of the three accelerations.  A max(a, b) passes its adjoint to a when a >= b, as the
// dual-number evaluation of the forward does.
template <class R>
GMT_HD void finish_update_adj(const Q9<R>& rin, const Consts<R>& K, R glm_fac, bool turb, R ax, R ay, R az, R dt,
                              const Q9<R>& ob, Q9<R>& rb, R ab[3]) {
    Q9<R> r = rin;
    const bool voidf = r.v[0] < K.smallr;
    if (voidf) {
        r.v[0] = K.smallr; r.v[1] = R(0); r.v[2] = R(0); r.v[3] = R(0);
        r.v[4] = K.pfl / (K.gamma - R(1)) + R(0.5) * (r.v[5] * r.v[5] + r.v[6] * r.v[6] + r.v[7] * r.v[7]);
    }
    Q9<R> b = ob;   // adjoint of the state after the void floor (psi handled below)
    ab[0] = ab[1] = ab[2] = R(0);
    if (turb && r.v[0] >= K.turb_min_rho) {
        const R rho = r.v[0], rhom = rmax(rho, K.smallr), irm = R(1) / rhom;
        const R fl = rho * (K.smallc * K.smallc);
        const R acc[3] = {ax, ay, az};
        // forward values and branch flags of the six floored energy updates
        R e = r.v[4], m[3];
        bool t[6];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const R x = e - R(0.5) * r.v[1 + i] * r.v[1 + i] / rhom;
            t[i] = x >= fl;
            e = t[i] ? x : fl;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) m[i] = r.v[1 + i] + rhom * acc[i] * dt;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const R x = e + R(0.5) * m[i] * m[i] / rhom;
            t[3 + i] = x >= fl;
            e = t[3 + i] ? x : fl;
        }
        // reverse
        R eb = ob.v[4], flb = R(0), rhomb = R(0);
        R mb[3] = {ob.v[1], ob.v[2], ob.v[3]};
        R vb[3] = {R(0), R(0), R(0)};
#pragma unroll
        for (int i = 2; i >= 0; --i) {
            if (t[3 + i]) {
                mb[i] += eb * m[i] * irm;
                rhomb -= eb * R(0.5) * m[i] * m[i] * irm * irm;
            } else {
                flb += eb;
                eb = R(0);
            }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            vb[i] += mb[i];
            rhomb += mb[i] * acc[i] * dt;
            ab[i] = mb[i] * rhom * dt;
        }
#pragma unroll
        for (int i = 2; i >= 0; --i) {
            if (t[i]) {
                vb[i] -= eb * r.v[1 + i] * irm;
                rhomb += eb * R(0.5) * r.v[1 + i] * r.v[1 + i] * irm * irm;
            } else {
                flb += eb;
                eb = R(0);
            }
        }
        b.v[1] = vb[0]; b.v[2] = vb[1]; b.v[3] = vb[2];
        b.v[4] = eb;
        b.v[0] = ob.v[0] + flb * (K.smallc * K.smallc) + (rho >= K.smallr ? rhomb : R(0));
    }
    rb = b;
    rb.v[8] = ob.v[8] * glm_fac;
    if (voidf) {
        // rho, momentum and E were overwritten: only B reaches E through the magnetic energy
        rb.v[5] += b.v[4] * r.v[5];
        rb.v[6] += b.v[4] * r.v[6];
        rb.v[7] += b.v[4] * r.v[7];
        rb.v[0] = rb.v[1] = rb.v[2] = rb.v[3] = rb.v[4] = R(0);
    }
}

}  // namespace gmt
