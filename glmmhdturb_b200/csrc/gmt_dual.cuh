// gmt_dual.cuh -- forward-mode dual numbers for the device physics.
//
// Dual<R, N> carries a value and N tangents.  Every physics function of gmt_phys.cuh is a template
// over the real type, so instantiating it with Dual<R, N> evaluates the same expressions and
// propagates N directional derivatives exactly; the adjoint kernels use this to form Jacobian-
// transpose products of the Riemann solvers and of the Hancock block.  Comparisons and the
// max/min/abs selections act on the value (the subgradient at a kink follows the branch taken).
#pragma once
#include <type_traits>

#include "gmt_phys.cuh"

namespace gmt {

template <class R, int N> struct Dual {
    R v;
    R d[N];
    GMT_HD Dual() {}
    template <class T, class = typename std::enable_if<std::is_arithmetic<T>::value>::type>
    GMT_HD Dual(T x) : v((R)x) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = R(0);
    }
};

template <class R, int N> GMT_HD Dual<R, N> operator+(const Dual<R, N>& a, const Dual<R, N>& b) {
    Dual<R, N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <class R, int N> GMT_HD Dual<R, N> operator-(const Dual<R, N>& a, const Dual<R, N>& b) {
    Dual<R, N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <class R, int N> GMT_HD Dual<R, N> operator-(const Dual<R, N>& a) {
    Dual<R, N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <class R, int N> GMT_HD Dual<R, N> operator*(const Dual<R, N>& a, const Dual<R, N>& b) {
    Dual<R, N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <class R, int N> GMT_HD Dual<R, N> operator/(const Dual<R, N>& a, const Dual<R, N>& b) {
    Dual<R, N> r;
    r.v = a.v / b.v;
    const R ib = R(1) / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <class R, int N> GMT_HD bool operator<(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v < b.v; }
template <class R, int N> GMT_HD bool operator<=(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v <= b.v; }
template <class R, int N> GMT_HD bool operator>(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v > b.v; }
template <class R, int N> GMT_HD bool operator>=(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v >= b.v; }

template <class R, int N> GMT_HD Dual<R, N> rmax(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v >= b.v ? a : b; }
template <class R, int N> GMT_HD Dual<R, N> rmin(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v <= b.v ? a : b; }
template <class R, int N> GMT_HD Dual<R, N> rabs(const Dual<R, N>& a) { return a.v >= R(0) ? a : -a; }
template <class R, int N> GMT_HD Dual<R, N> sqrt_r(const Dual<R, N>& a) {
    Dual<R, N> r;
    r.v = sqrt_r(a.v);
    const R s = r.v > R(0) ? R(0.5) / r.v : R(0);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * s;
    return r;
}

template <class R, int N> GMT_HD Consts<Dual<R, N>> dual_consts(const Consts<R>& K) {
    Consts<Dual<R, N>> D;
    D.gamma = Dual<R, N>(K.gamma);
    D.smallr = Dual<R, N>(K.smallr);
    D.pfl = Dual<R, N>(K.pfl);
    D.smallc = Dual<R, N>(K.smallc);
    D.smallp = Dual<R, N>(K.smallp);
    D.llf_dmin = Dual<R, N>(K.llf_dmin);
    D.llf_pmin = Dual<R, N>(K.llf_pmin);
    D.turb_min_rho = Dual<R, N>(K.turb_min_rho);
    return D;
}

}  // namespace gmt
