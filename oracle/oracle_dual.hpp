// ORACLE — test infrastructure only. Forward-mode dual numbers with ForwardDiff 1.4's rules
// (third-party dependency of GeometricSolvers.jl, Project.toml:11), as the R1 Jacobian
// `jacobian!!` (src/ad/forwarddiff_static.jl:50-65) and JVP `jvp!!` (src/ad/jvp.jl:96-107)
// use them: a value and K partials; each rule is value op value and the derivative rule times
// the partials.
#pragma once

#include <cmath>

namespace orc {

template <int K> struct Dual {
    static constexpr int nparts = K;
    double v;
    double p[K];
};

template <int K> inline Dual<K> dconst(double c) {
    Dual<K> r;
    r.v = c;
    for (int k = 0; k < K; ++k) r.p[k] = 0.0;
    return r;
}

template <int K> inline Dual<K> operator+(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v + b.v;
    for (int k = 0; k < K; ++k) r.p[k] = a.p[k] + b.p[k];
    return r;
}
template <int K> inline Dual<K> operator+(const Dual<K>& a, double c) {
    Dual<K> r = a;
    r.v = a.v + c;
    return r;
}
template <int K> inline Dual<K> operator+(double c, const Dual<K>& a) {
    Dual<K> r = a;
    r.v = c + a.v;
    return r;
}
template <int K> inline Dual<K> operator-(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v - b.v;
    for (int k = 0; k < K; ++k) r.p[k] = a.p[k] - b.p[k];
    return r;
}
template <int K> inline Dual<K> operator-(const Dual<K>& a, double c) {
    Dual<K> r = a;
    r.v = a.v - c;
    return r;
}
template <int K> inline Dual<K> operator-(double c, const Dual<K>& a) {
    Dual<K> r;
    r.v = c - a.v;
    for (int k = 0; k < K; ++k) r.p[k] = -a.p[k];
    return r;
}
template <int K> inline Dual<K> operator-(const Dual<K>& a) {
    Dual<K> r;
    r.v = -a.v;
    for (int k = 0; k < K; ++k) r.p[k] = -a.p[k];
    return r;
}
// x * y: partials px * vy + py * vx (ForwardDiff `_mul_partials`).
template <int K> inline Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v * b.v;
    for (int k = 0; k < K; ++k) r.p[k] = a.p[k] * b.v + b.p[k] * a.v;
    return r;
}
template <int K> inline Dual<K> operator*(double c, const Dual<K>& a) {
    Dual<K> r;
    r.v = c * a.v;
    for (int k = 0; k < K; ++k) r.p[k] = c * a.p[k];
    return r;
}
template <int K> inline Dual<K> operator*(const Dual<K>& a, double c) {
    Dual<K> r;
    r.v = a.v * c;
    for (int k = 0; k < K; ++k) r.p[k] = a.p[k] * c;
    return r;
}
// x / y: partials px * inv(vy) + py * (-(vx / (vy * vy))) (ForwardDiff `_div_partials`).
template <int K> inline Dual<K> operator/(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v / b.v;
    double ib = 1.0 / b.v;
    double q = -(a.v / (b.v * b.v));
    for (int k = 0; k < K; ++k) r.p[k] = a.p[k] * ib + b.p[k] * q;
    return r;
}
template <int K> inline Dual<K> operator/(const Dual<K>& a, double c) {
    Dual<K> r;
    r.v = a.v / c;
    for (int k = 0; k < K; ++k) r.p[k] = a.p[k] / c;
    return r;
}
template <int K> inline Dual<K> operator/(double c, const Dual<K>& b) {
    Dual<K> r;
    r.v = c / b.v;
    double q = -(c / (b.v * b.v));
    for (int k = 0; k < K; ++k) r.p[k] = q * b.p[k];
    return r;
}
// f(x) with derivative df: Dual(f(v), df(v) * p).
template <int K> inline Dual<K> chain(const Dual<K>& a, double fv, double dfv) {
    Dual<K> r;
    r.v = fv;
    for (int k = 0; k < K; ++k) r.p[k] = dfv * a.p[k];
    return r;
}
template <int K> inline Dual<K> exp(const Dual<K>& a) {
    double e = std::exp(a.v);
    return chain(a, e, e);
}
template <int K> inline Dual<K> sqrt(const Dual<K>& a) {
    double s = std::sqrt(a.v);
    return chain(a, s, 1.0 / (2.0 * s));
}
template <int K> inline Dual<K> atan(const Dual<K>& a) {
    return chain(a, std::atan(a.v), 1.0 / (1.0 + a.v * a.v));
}
template <int K> inline Dual<K> sin(const Dual<K>& a) {
    return chain(a, std::sin(a.v), std::cos(a.v));
}
template <int K> inline Dual<K> cos(const Dual<K>& a) {
    return chain(a, std::cos(a.v), -std::sin(a.v));
}

// Scalar versions usable in the same generic residual code.
inline double value(double x) { return x; }
template <int K> inline double value(const Dual<K>& x) { return x.v; }

// Integer powers: value v^n, derivative n v^(n-1) (ForwardDiff's `^(::Dual, ::Integer)`).
inline double ipow(double v, int n) {
    if (n == 2) return v * v;
    if (n == 3) return v * v * v;
    double r = 1.0;
    for (int i = 0; i < n; ++i) r = r * v;
    return r;
}
template <int K> inline Dual<K> ipow(const Dual<K>& a, int n) {
    return chain(a, ipow(a.v, n), double(n) * ipow(a.v, n - 1));
}

}  // namespace orc
