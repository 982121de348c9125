// phx_dual.hpp — TEST INFRASTRUCTURE ONLY (part of the oracle): forward-mode dual numbers for the
// analytic FP64 gradient of the frozen-path estimator (phx_frozen.hpp).
//
// Dual<N> carries a value and N tangent components: every arithmetic operation applies the chain
// rule exactly (sum, product and quotient rules, d sqrt x = dx / (2 sqrt x), d x^y = y x^(y-1) dx
// for a constant exponent y, |x|, max and min taking the derivative of the selected operand).
// Comparisons look at the value only, so a code path's branches are the ones its value takes.
// Seeding the parameters θ with unit tangents and evaluating F(θ) once gives N partial derivatives
// of every output in double precision, with no step size and no cancellation — an analytic
// gradient computed by a method independent of the library's hand-written reverse-mode adjoint.
#pragma once

#include <cmath>

#include "phx_oracle.hpp"

namespace orc {

template <int N> struct Dual {
    double v;
    double d[N];
    constexpr Dual() : v(0.0), d{} {}
    constexpr Dual(double x) : v(x), d{} {} // a constant: zero tangent
};

template <int N> inline Dual<N> operator+(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r(a.v + b.v);
    for (int i = 0; i < N; i++)
        r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N> inline Dual<N> operator-(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r(a.v - b.v);
    for (int i = 0; i < N; i++)
        r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N> inline Dual<N> operator-(const Dual<N> &a) {
    Dual<N> r(-a.v);
    for (int i = 0; i < N; i++)
        r.d[i] = -a.d[i];
    return r;
}
template <int N> inline Dual<N> operator*(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r(a.v * b.v);
    for (int i = 0; i < N; i++)
        r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N> inline Dual<N> operator/(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r(a.v / b.v);
    const double inv = 1.0 / b.v;
    for (int i = 0; i < N; i++)
        r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
}
template <int N> inline Dual<N> &operator+=(Dual<N> &a, const Dual<N> &b) { return a = a + b; }
template <int N> inline Dual<N> &operator*=(Dual<N> &a, const Dual<N> &b) { return a = a * b; }
template <int N> inline bool operator<(const Dual<N> &a, const Dual<N> &b) { return a.v < b.v; }
template <int N> inline bool operator>(const Dual<N> &a, const Dual<N> &b) { return a.v > b.v; }
template <int N> inline bool operator<=(const Dual<N> &a, const Dual<N> &b) { return a.v <= b.v; }
template <int N> inline bool operator>=(const Dual<N> &a, const Dual<N> &b) { return a.v >= b.v; }
template <int N> inline bool operator==(const Dual<N> &a, const Dual<N> &b) { return a.v == b.v; }
template <int N> inline bool operator!=(const Dual<N> &a, const Dual<N> &b) { return a.v != b.v; }

template <int N> inline Dual<N> scale_d(const Dual<N> &a, double value, double dfdx) {
    Dual<N> r(value);
    for (int i = 0; i < N; i++)
        r.d[i] = dfdx * a.d[i];
    return r;
}

template <int N> struct M<Dual<N>> {
    using D = Dual<N>;
    static D sqrt(const D &x) {
        const double s = std::sqrt(x.v);
        return scale_d(x, s, s > 0.0 ? 0.5 / s : 0.0);
    }
    static D fabs(const D &x) { return x.v < 0.0 ? -x : x; }
    static D fmax(const D &a, const D &b) { return (a.v < b.v || std::isnan(a.v)) ? b : a; }
    static D fmin(const D &a, const D &b) { return (b.v < a.v || std::isnan(a.v)) ? b : a; }
    // x^y for a constant exponent y (the only form the weights use: Schlick's ^5, sRGB's ^2.2)
    static D pow(const D &x, const D &y) {
        const double p = std::pow(x.v, y.v);
        return scale_d(x, p, x.v != 0.0 ? y.v * std::pow(x.v, y.v - 1.0) : 0.0);
    }
    static D exp(const D &x) {
        const double e = std::exp(x.v);
        return scale_d(x, e, e);
    }
    static D log(const D &x) { return scale_d(x, std::log(x.v), 1.0 / x.v); }
};

template <int N> struct C<Dual<N>> {
    static constexpr Dual<N> EPS = Dual<N>((double)EPS_F);
    static constexpr Dual<N> INF = Dual<N>((double)INF_F);
    static constexpr Dual<N> PI = Dual<N>((double)PI_F);
};

} // namespace orc
