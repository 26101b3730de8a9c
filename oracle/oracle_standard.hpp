// ORACLE — test infrastructure only. The 23 systems of the reference's standard test set
// (test/helpers/standard_problems.jl:58-424: NonlinearProblemLibrary.jl's problems after Moré,
// Garbow and Hillstrom 1981), each generic over double and Dual<K>, with the operation order of
// the reference's expressions. They pin the solve loop against the golden table
// test/verification/standard_reference.csv.
#pragma once

#include <cmath>

#include "oracle_families.hpp"

namespace orc {

inline double sinpi_(double x);
// cospi(x) with exact argument reduction: exact zeros at half-integers.
inline double cospi_(double x) {
    double r = std::fmod(std::fabs(x), 2.0);
    if (r > 1.0) r = 2.0 - r;  // cos(pi r) = cos(pi (2 - r))
    double sgn = 1.0;
    if (r > 0.5) {
        r = 1.0 - r;
        sgn = -1.0;
    }
    double v = r > 0.25 ? std::sin(M_PI * (0.5 - r)) : std::cos(M_PI * r);
    return sgn * v;
}
inline double sinpi_(double x) {
    double ax = std::fabs(x);
    double r = std::fmod(ax, 2.0);
    double sgn = x < 0 ? -1.0 : 1.0;
    if (r > 1.0) {
        r = r - 1.0;
        sgn = -sgn;
    }
    if (r > 0.5) r = 1.0 - r;
    double v = r > 0.25 ? std::cos(M_PI * (0.5 - r)) : std::sin(M_PI * r);
    return sgn * v;
}
inline double cospi(double x) { return cospi_(x); }
template <int K> inline Dual<K> cospi(const Dual<K>& a) {
    return chain(a, cospi_(a.v), -M_PI * sinpi_(a.v));
}
inline double sign(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : x); }
template <int K> inline Dual<K> sign(const Dual<K>& a) { return dconst<K>(sign(a.v)); }
inline double sin(double x) { return std::sin(x); }
inline double cos(double x) { return std::cos(x); }
inline double atan(double x) { return std::atan(x); }
// ForwardDiff's iszero of a Dual reads the partials too.
inline bool iszero_(double x) { return x == 0.0; }
template <int K> inline bool iszero_(const Dual<K>& a) {
    if (a.v != 0.0) return false;
    for (int k = 0; k < K; ++k)
        if (a.p[k] != 0.0) return false;
    return true;
}

template <int N_, int NUM> struct Standard {
    static constexpr int N = N_, M = N_;
    static constexpr bool lsq = false, analytic_J = false;
    template <class S> void F(const S* x, S* out) const;
    void J(const double*, double*) const {}
};

template <class S> inline S ifelse_(bool c, const S& a, const S& b) { return c ? a : b; }

#define STD_F(NN, NUM)                                                                          \
    template <> template <class S> void Standard<NN, NUM>::F(const S* x, S* out) const

STD_F(10, 1) {
    const int n = 10;
    out[0] = 1.0 - x[0];
    for (int i = 1; i < n; ++i) out[i] = 10.0 * (x[i] - x[i - 1] * x[i - 1]);
}
STD_F(4, 2) {
    out[0] = x[0] + 10.0 * x[1];
    out[1] = std::sqrt(5.0) * (x[2] - x[3]);
    out[2] = ipow(x[1] - 2.0 * x[2], 2);
    out[3] = std::sqrt(10.0) * (x[0] - x[3]) * (x[0] - x[3]);
}
STD_F(2, 3) {
    out[0] = 10000.0 * x[0] * x[1] - 1.0;
    out[1] = exp(-x[0]) + exp(-x[1]) - 1.0001;
}
STD_F(4, 4) {
    S t1 = x[1] - x[0] * x[0];
    S t2 = x[3] - x[2] * x[2];
    out[0] = -200.0 * x[0] * t1 - (1.0 - x[0]);
    out[1] = 200.0 * t1 + 20.2 * (x[1] - 1.0) + 19.8 * (x[3] - 1.0);
    out[2] = -180.0 * x[2] * t2 - (1.0 - x[2]);
    out[3] = 180.0 * t2 + 20.2 * (x[3] - 1.0) + 19.8 * (x[1] - 1.0);
}
STD_F(3, 5) {
    S temp1 = atan(x[1] / x[0]) / (2.0 * M_PI);
    S temp = ifelse_(0.0 < value(x[0]), temp1,
                     ifelse_(value(x[0]) < 0.0, temp1 + 0.5, 0.25 * sign(x[1])));
    out[0] = 10.0 * (x[2] - 10.0 * temp);
    out[1] = 10.0 * (sqrt(x[0] * x[0] + x[1] * x[1]) - 1.0);
    out[2] = x[2];
}
STD_F(2, 6) {
    const int n = 2;
    for (int k = 0; k < n; ++k) out[k] = cst<S>(0.0);
    for (int i = 1; i <= 29; ++i) {
        double ti = double(i) / 29.0;
        S sum1 = cst<S>(0.0);
        double temp = 1.0;
        for (int j = 2; j <= n; ++j) {
            sum1 = sum1 + (double(j) * temp) * x[j - 1];
            temp = ti * temp;
        }
        S sum2 = cst<S>(0.0);
        temp = 1.0;
        for (int j = 1; j <= n; ++j) {
            sum2 = sum2 + temp * x[j - 1];
            temp = ti * temp;
        }
        temp = 1.0 / ti;
        for (int k = 1; k <= n; ++k) {
            out[k - 1] = out[k - 1] + temp * (sum1 - sum2 * sum2 - 1.0) * (double(k) - 2.0 * ti * sum2);
            temp = ti * temp;
        }
    }
    out[0] = out[0] + x[0] * (3.0 - 2.0 * x[1] + 2.0 * ipow(x[0], 2));
    out[1] = out[1] + (x[1] * (1.0 - x[1]) - 1.0);
}
STD_F(2, 7) {
    const int n = 2;
    for (int k = 0; k < n; ++k) out[k] = cst<S>(0.0);
    for (int j = 0; j < n; ++j) {
        S t1 = cst<S>(1.0);
        S t2 = x[j];
        for (int i = 0; i < n; ++i) {
            out[i] = out[i] + t2;
            S t3 = 2.0 * x[j] * t2 - t1;
            t1 = t2;
            t2 = t3;
        }
    }
    for (int i = 1; i <= n; ++i)
        out[i - 1] = out[i - 1] / double(n) + ((i % 2 == 0) ? 1.0 / double(i * i - 1) : 0.0);
}
STD_F(10, 8) {
    const int n = 10;
    S sum = x[0];
    for (int i = 1; i < n; ++i) sum = sum + x[i];
    for (int i = 0; i < n - 1; ++i) out[i] = x[i] + sum - double(n + 1);
    S prod = x[0];
    for (int i = 1; i < n; ++i) prod = prod * x[i];
    out[n - 1] = prod - 1.0;
}
template <class S> inline S bvf_kernel(const S& xk, int k, double h) {
    return 2.0 * xk + 0.5 * (h * h) * ipow(xk + double(k) * h + 1.0, 3);
}
STD_F(10, 9) {
    const int n = 10;
    double h = 1.0 / double(n + 1);
    out[0] = bvf_kernel(x[0], 1, h) - x[1];
    for (int k = 2; k <= n - 1; ++k) out[k - 1] = bvf_kernel(x[k - 1], k, h) - x[k - 2] - x[k];
    out[n - 1] = bvf_kernel(x[n - 1], n, h) - x[n - 2];
}
STD_F(10, 10) {
    const int n = 10;
    double h = 1.0 / double(n + 1);
    for (int k = 1; k <= n; ++k) {
        double tk = double(k) / double(n + 1);
        S sum1 = cst<S>(0.0);
        for (int j = 1; j <= k; ++j) {
            double tj = double(j) * h;
            sum1 = sum1 + tj * ipow(x[j - 1] + tj + 1.0, 3);
        }
        S sum2 = cst<S>(0.0);
        for (int j = k; j <= n; ++j) {
            double tj = double(j) * h;
            sum2 = sum2 + (1.0 - tj) * ipow(x[j - 1] + tj + 1.0, 3);
        }
        out[k - 1] = x[k - 1] + h * ((1.0 - tk) * sum1 + tk * sum2) / 2.0;
    }
}
STD_F(10, 11) {
    const int n = 10;
    S csum = cos(x[0]);
    for (int i = 1; i < n; ++i) csum = csum + cos(x[i]);
    for (int k = 1; k <= n; ++k) {
        S sx = sin(x[k - 1]), cx = cos(x[k - 1]);
        out[k - 1] = double(n) - csum + double(k) * (1.0 - cx) - sx;
    }
}
STD_F(10, 12) {
    const int n = 10;
    S sum1 = cst<S>(0.0);
    for (int j = 1; j <= n; ++j) sum1 = sum1 + double(j) * (x[j - 1] - 1.0);
    for (int k = 1; k <= n; ++k)
        out[k - 1] = x[k - 1] - 1.0 + double(k) * sum1 * (1.0 + 2.0 * sum1 * sum1);
}
template <class S> inline S tridiag_kernel(const S& xk) { return (3.0 - 2.0 * xk) * xk + 1.0; }
STD_F(10, 13) {
    const int n = 10;
    out[0] = tridiag_kernel(x[0]) - 2.0 * x[1];
    for (int k = 2; k <= n - 1; ++k)
        out[k - 1] = tridiag_kernel(x[k - 1]) - x[k - 2] - 2.0 * x[k];
    out[n - 1] = tridiag_kernel(x[n - 1]) - x[n - 2];
}
STD_F(10, 14) {
    const int n = 10;
    for (int k = 1; k <= n; ++k) {
        int k1 = k - 5 > 1 ? k - 5 : 1;
        int k2 = k + 1 < n ? k + 1 : n;
        S temp = cst<S>(0.0);
        for (int j = k1; j <= k2; ++j)
            if (j != k) temp = temp + x[j - 1] * (1.0 + x[j - 1]);
        out[k - 1] = x[k - 1] * (2.0 + 5.0 * x[k - 1] * x[k - 1]) + 1.0 - temp;
    }
}
STD_F(4, 15) {
    out[0] = (x[0] * x[0] + x[1] * x[2]) - 0.0001;
    out[1] = (x[0] * x[1] + x[1] * x[3]) - 1.0;
    out[2] = (x[2] * x[0] + x[3] * x[2]) - 0.0;
    out[3] = (x[2] * x[1] + x[3] * x[3]) - 0.0001;
}
STD_F(9, 16) {
    out[0] = (x[0] * x[0] + x[1] * x[3] + x[2] * x[6]) - 0.0001;
    out[1] = (x[0] * x[1] + x[1] * x[4] + x[2] * x[7]) - 1.0;
    out[2] = x[0] * x[2] + x[1] * x[5] + x[2] * x[8];
    out[3] = x[3] * x[0] + x[4] * x[3] + x[5] * x[6];
    out[4] = (x[3] * x[1] + x[4] * x[4] + x[5] * x[7]) - 0.0001;
    out[5] = x[3] * x[2] + x[4] * x[5] + x[5] * x[8];
    out[6] = x[6] * x[0] + x[7] * x[3] + x[8] * x[6];
    out[7] = x[6] * x[1] + x[7] * x[4] + x[8] * x[7];
    out[8] = (x[6] * x[2] + x[7] * x[5] + x[8] * x[8]) - 0.0001;
}
STD_F(2, 17) {
    out[0] = x[0] + x[1] - 3.0;
    out[1] = ipow(x[0], 2) + ipow(x[1], 2) - 9.0;
}
STD_F(2, 18) {
    if (iszero_(x[0])) out[0] = cst<S>(0.0);
    else out[0] = ipow(x[1], 2) * (1.0 - exp(-x[0] * x[0])) / x[0];
    if (iszero_(x[1])) out[1] = cst<S>(0.0);
    else out[1] = x[0] * (1.0 - exp(-x[1] * x[1])) / x[1];
}
STD_F(2, 19) {
    S tmp = ipow(x[0], 2) + ipow(x[1], 2);
    out[0] = x[0] * tmp;
    out[1] = x[1] * tmp;
}
STD_F(1, 20) { out[0] = x[0] * ipow(x[0] - 5.0, 2); }
STD_F(2, 21) {
    out[0] = x[0] - ipow(x[1], 3) + 5.0 * ipow(x[1], 2) - 2.0 * x[1] - 13.0;
    out[1] = x[0] + ipow(x[1], 3) + ipow(x[1], 2) - 14.0 * x[1] - 29.0;
}
STD_F(2, 22) {
    out[0] = x[0] * x[0] - x[1] + 1.0;
    out[1] = x[0] - cospi(0.5 * x[1]);
}
STD_F(10, 23) {
    const int n = 10;
    double c = 0.9;
    for (int i = 0; i < n; ++i) out[i] = x[i];
    for (int i = 1; i <= n; ++i) {
        S mui = cst<S>(double(i)) / double(n);
        S s = cst<S>(0.0);
        for (int j = 1; j <= n; ++j) {
            S muj = cst<S>(double(j)) / double(n);
            s = s + (mui * x[j - 1]) / (mui + muj);
        }
        S term = 1.0 - c * s / (2.0 * double(n));
        out[i - 1] = out[i - 1] - 1.0 / term;
    }
}

#undef STD_F

}  // namespace orc
