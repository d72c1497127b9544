// Host-only check of the hand-written reverse sweeps of the adjoint (gmt_riemann_adj.cuh) against
// forward-mode dual-number VJPs of the same forward functions, on randomised FP64 states (the
// HLLD faces are counted per fan region and degenerate star state, and the test requires each to
// occur), the state floors and the epilogue's void floor and energy floors.  Built by
// tests/test_adjoint_host.py with nvcc; no GPU is used.  Prints one line per function:
// "<name> <samples> <max relative error>", and "hlld_regions <outer L> <inner L> <inner R>
// <outer R> <degenerate>".
#include <cmath>
#include <cstdio>
#include <random>

#include "../../glmmhdturb_b200/csrc/gmt_adjoint.cuh"

using namespace gmt;
using R = double;

static std::mt19937_64 rng(12345);
static R uni(R a, R b) { return std::uniform_real_distribution<R>(a, b)(rng); }

// a random primitive state; `wild` widens the velocity and field ranges (supersonic faces, outer
// HLLD regions), `weak` makes the transverse and normal fields vanish (degenerate star state)
static Q9<R> rand_prim(bool wild, bool weak) {
    Q9<R> q;
    q.v[0] = uni(0.2, 3.0);
    const R vs = wild ? 6.0 : 1.5, bs = weak ? 0.0 : (wild ? 3.0 : 1.0);
    for (int i = 1; i < 4; ++i) q.v[i] = uni(-vs, vs);
    q.v[4] = uni(0.05, 3.0);
    for (int i = 5; i < 8; ++i) q.v[i] = uni(-bs, bs);
    q.v[8] = uni(-0.1, 0.1);
    return q;
}

static R rel(const R* a, const R* b, int n) {
    R e = 0, s = 1e-300;
    for (int i = 0; i < n; ++i) {
        e = std::fmax(e, std::fabs(a[i] - b[i]));
        s = std::fmax(s, std::fmax(std::fabs(a[i]), std::fabs(b[i])));
    }
    return e / s;
}

static Consts<R> consts() {
    Consts<R> K;
    K.gamma = 5.0 / 3.0; K.smallr = 1e-6; K.smallc = 1e-6; K.pfl = K.smallr * K.smallc * K.smallc / K.gamma;
    K.smallp = 1e-6; K.llf_dmin = 0; K.llf_pmin = 0; K.turb_min_rho = 0;
    return K;
}

// dual VJP of riemann_glm<0, RIEM>: 18 inputs in three chunks of 6
template <int RIEM> static void riemann_dual(const Q9<R>& L, const Q9<R>& Rr, const Q9<R>& fb, const Consts<R>& K, R ch,
                                             Q9<R>& Lb, Q9<R>& Rb) {
    constexpr int N = 6;
    using DD = Dual<R, N>;
    const Consts<DD> KD = dual_consts<R, N>(K);
    for (int c0 = 0; c0 < 18; c0 += N) {
        Q9<DD> Ld, Rd;
        for (int v = 0; v < 9; ++v) {
            Ld.v[v] = DD(L.v[v]);
            Rd.v[v] = DD(Rr.v[v]);
            for (int j = 0; j < N; ++j) {
                Ld.v[v].d[j] = (c0 + j == v) ? 1.0 : 0.0;
                Rd.v[v].d[j] = (c0 + j == 9 + v) ? 1.0 : 0.0;
            }
        }
        Q9<DD> F = riemann_glm<0, RIEM>(Ld, Rd, KD, DD(ch), false);
        for (int j = 0; j < N; ++j) {
            R acc = 0;
            for (int v = 0; v < 9; ++v) acc += fb.v[v] * F.v[v].d[j];
            const int i = c0 + j;
            if (i < 9) Lb.v[i] = acc; else Rb.v[i - 9] = acc;
        }
    }
}

// fan region of an HLLD face (hlld_x's sampling): 0 outer left, 1 inner left, 2 inner right,
// 3 outer right; counts[4] = faces with a degenerate star state on either side
static long region_counts[5];
static void hlld_region(Q9<R> L, Q9<R> Rr, const Consts<R>& K, R ch) {
    L.v[0] = std::fmax(L.v[0], K.smallr); L.v[4] = std::fmax(L.v[4], K.pfl);
    Rr.v[0] = std::fmax(Rr.v[0], K.smallr); Rr.v[4] = std::fmax(Rr.v[4], K.pfl);
    R bn, psis;
    glm_pair(L.v[5], Rr.v[5], L.v[8], Rr.v[8], ch, bn, psis);
    const R g = K.gamma, dL = L.v[0], uL = L.v[1], dR = Rr.v[0], uR = Rr.v[1];
    const R ptL = L.v[4] + 0.5 * (bn * bn + L.v[6] * L.v[6] + L.v[7] * L.v[7]);
    const R ptR = Rr.v[4] + 0.5 * (bn * bn + Rr.v[6] * Rr.v[6] + Rr.v[7] * Rr.v[7]);
    const R cf = std::fmax(fast_speed(L, g, bn), fast_speed(Rr, g, bn));
    const R SL = std::fmin(std::fmin(uL, uR) - cf, 0.0), SR = std::fmax(std::fmax(uL, uR) + cf, 0.0);
    const R den = (SR - uR) * dR - (SL - uL) * dL;
    const R SM = ((SR - uR) * dR * uR - (SL - uL) * dL * uL - ptR + ptL) / den;
    const R dLs = std::fmax(dL * (SL - uL) / (SL - SM), 1e-12), dRs = std::fmax(dR * (SR - uR) / (SR - SM), 1e-12);
    const R SLs = SM - std::fabs(bn) / std::sqrt(dLs), SRs = SM + std::fabs(bn) / std::sqrt(dRs);
    region_counts[SLs >= 0 ? 0 : (SRs < 0 ? 3 : (SM >= 0 ? 1 : 2))]++;
    const R kL = dL * (SL - uL) * (SL - SM) - bn * bn, kR = dR * (SR - uR) * (SR - SM) - bn * bn;
    if (std::fabs(kL) < 1e-12 || std::fabs(kR) < 1e-12) region_counts[4]++;
}

template <int RIEM> static R check_riemann(int ns) {
    const Consts<R> K = consts();
    R worst = 0;
    for (int s = 0; s < ns; ++s) {
        const bool wild = s % 3 == 1, weak = s % 7 == 3;
        Q9<R> L = rand_prim(wild, weak), Rr = rand_prim(wild, weak), fb;
        if (s % 11 == 5) { Rr = L; Rr.v[1] += 1e-3; }   // nearly equal states
        if (s % 17 == 8) {
            // equal states at rest with no transverse field and Alfven speed above the sound speed:
            // the fast and Alfven waves coincide and both star states are degenerate
            L.v[1] = 0; L.v[6] = L.v[7] = 0;
            L.v[5] = std::sqrt(2.0 * K.gamma * L.v[4]) * (s % 2 ? 1 : -1);
            Rr = L;
        }
        for (int v = 0; v < 9; ++v) fb.v[v] = uni(-1, 1);
        const R ch = uni(0.5, 5.0);
        if (RIEM == RIEM_HLLD) hlld_region(L, Rr, K, ch);
        Q9<R> Lh, Rh, Ld, Rd;
        if (!riemann_x_adj<RIEM>(L, Rr, fb, K, ch, false, Lh, Rh)) return 1.0;
        riemann_dual<RIEM>(L, Rr, fb, K, ch, Ld, Rd);
        R a[18], b[18];
        for (int v = 0; v < 9; ++v) { a[v] = Lh.v[v]; a[9 + v] = Rh.v[v]; b[v] = Ld.v[v]; b[9 + v] = Rd.v[v]; }
        worst = std::fmax(worst, rel(a, b, 18));
    }
    return worst;
}

static R check_cons2prim(int ns) {
    const Consts<R> K = consts();
    using DD = Dual<R, 9>;
    R worst = 0;
    for (int s = 0; s < ns; ++s) {
        Q9<R> q = rand_prim(s % 2, false), qb;
        if (s % 5 == 2) q.v[4] = 1e-9;   // pressure floor active
        const Q9<R> c = prim2cons(q, K.gamma);
        for (int v = 0; v < 9; ++v) qb.v[v] = uni(-1, 1);
        Q9<R> cb_h;
        for (int v = 0; v < 9; ++v) cb_h.v[v] = 0;
        cons2prim_adj(c, K.gamma, K.smallr, K.pfl, qb, cb_h);
        Q9<DD> cd;
        for (int v = 0; v < 9; ++v) { cd.v[v] = DD(c.v[v]); for (int j = 0; j < 9; ++j) cd.v[v].d[j] = j == v; }
        const Q9<DD> qd = cons2prim(cd, DD(K.gamma), DD(K.smallr), DD(K.pfl));
        R a[9], b[9];
        for (int j = 0; j < 9; ++j) {
            R acc = 0;
            for (int v = 0; v < 9; ++v) acc += qb.v[v] * qd.v[v].d[j];
            a[j] = cb_h.v[j]; b[j] = acc;
        }
        worst = std::fmax(worst, rel(a, b, 9));
    }
    return worst;
}

static R check_prim2cons_flux(int ns, bool flux) {
    const Consts<R> K = consts();
    using DD = Dual<R, 9>;
    R worst = 0;
    for (int s = 0; s < ns; ++s) {
        Q9<R> q = rand_prim(s % 2, false), ob, qb_h;
        for (int v = 0; v < 9; ++v) { ob.v[v] = uni(-1, 1); qb_h.v[v] = 0; }
        if (flux) phys_flux_x_adj(q, K.gamma, ob, qb_h);
        else prim2cons_adj(q, K.gamma, ob, qb_h);
        Q9<DD> qd;
        for (int v = 0; v < 9; ++v) { qd.v[v] = DD(q.v[v]); for (int j = 0; j < 9; ++j) qd.v[v].d[j] = j == v; }
        const Q9<DD> od = flux ? phys_flux_x(qd, DD(K.gamma)) : prim2cons(qd, DD(K.gamma));
        R a[9], b[9];
        for (int j = 0; j < 9; ++j) {
            R acc = 0;
            for (int v = 0; v < 9; ++v) acc += ob.v[v] * od.v[v].d[j];
            a[j] = qb_h.v[j]; b[j] = acc;
        }
        worst = std::fmax(worst, rel(a, b, 9));
    }
    return worst;
}

static R check_epilogue(int ns) {
    Consts<R> K = consts();
    K.turb_min_rho = 0.3;
    K.smallc = 0.8;   // an energy floor rho*smallc^2 that the kick's KE removal can reach
    R worst = 0;
    for (int s = 0; s < ns; ++s) {
        Q9<R> q = rand_prim(s % 2, false);
        Q9<R> r = prim2cons(q, K.gamma);
        if (s % 9 == 4) r.v[0] = 0.5 * K.smallr;   // void floor
        if (s % 6 == 1) r.v[4] = 0.3 * r.v[0];      // low energy: the floors bind
        if (s % 13 == 7) r.v[0] = 0.2;              // below turb_min_rho: no kick
        const R a3[3] = {uni(-3, 3), uni(-3, 3), uni(-3, 3)};
        const R glm = uni(0.5, 1.0), dt = uni(0.01, 0.2);
        Q9<R> ob, rb_h, rb_d;
        for (int v = 0; v < 9; ++v) ob.v[v] = uni(-1, 1);
        R ab_h[3], ab_d[3];
        finish_update_adj(r, K, glm, true, a3[0], a3[1], a3[2], dt, ob, rb_h, ab_h);
        finish_update_adj_dual(r, K, glm, true, a3, dt, ob, rb_d, ab_d);
        R a[12], b[12];
        for (int v = 0; v < 9; ++v) { a[v] = rb_h.v[v]; b[v] = rb_d.v[v]; }
        for (int i = 0; i < 3; ++i) { a[9 + i] = ab_h[i]; b[9 + i] = ab_d[i]; }
        worst = std::fmax(worst, rel(a, b, 12));
    }
    return worst;
}

int main() {
    const int ns = 20000;
    std::printf("hlld %d %.3e\n", ns, check_riemann<RIEM_HLLD>(ns));
    std::printf("hlld_regions %ld %ld %ld %ld %ld\n", region_counts[0], region_counts[1], region_counts[2],
                region_counts[3], region_counts[4]);
    std::printf("hll %d %.3e\n", ns, check_riemann<RIEM_HLL>(ns));
    std::printf("cons2prim %d %.3e\n", ns, check_cons2prim(ns));
    std::printf("prim2cons %d %.3e\n", ns, check_prim2cons_flux(ns, false));
    std::printf("phys_flux_x %d %.3e\n", ns, check_prim2cons_flux(ns, true));
    std::printf("epilogue %d %.3e\n", ns, check_epilogue(ns));
    return 0;
}
