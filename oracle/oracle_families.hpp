// ORACLE — test infrastructure only. The residual families of the batch configurations and the
// residuals that the reference's own tests pin, each generic over double and Dual<K> so that
// the Jacobian and the JVP come from forward-mode duals as in the reference
// (src/ad/forwarddiff_static.jl:50-65, src/ad/jvp.jl:96-107).
#pragma once

#include <cmath>

#include "../geometricsolvers.jl_b200/csrc/gsb_exp.h"
#include "oracle_dual.hpp"

namespace orc {

// A constant in the number type S.
template <class S> inline S cst(double c);
template <> inline double cst<double>(double c) { return c; }
template <class S> inline S cst(double c) { return dconst<S::nparts>(c); }

// fma(c, x, acc) with a constant c: value and partials each fused (the family's own
// definition of its dot products).
inline double fmac(double c, double x, double acc) { return std::fma(c, x, acc); }
template <int K> inline Dual<K> fmac(double c, const Dual<K>& x, const Dual<K>& acc) {
    Dual<K> r;
    r.v = std::fma(c, x.v, acc.v);
    for (int k = 0; k < K; ++k) r.p[k] = std::fma(c, x.p[k], acc.p[k]);
    return r;
}

inline double exp(double x) { return std::exp(x); }
inline double sqrt(double x) { return std::sqrt(x); }

// The exponential of the exponential-sum family: the batch kernel's own (gsb_exp.h, Tang's
// table-driven method, the same bits on the host as on the device), so that the fit is checked
// bit for bit. The reference evaluates Julia's Base.exp, which neither the C library's exp nor
// this one reproduces in every last bit; every other exp of the oracle is the C library's.
inline double fam_exp(double x) { return gsb_exp::exp(x); }
template <int K> inline Dual<K> fam_exp(const Dual<K>& a) {
    const double e = gsb_exp::exp(a.v);
    return chain(a, e, e);
}

// ─── GSB_FAMILY_CUBIC_AFFINE: F(x) = A x + 0.1 x.^3 - b, p = (A column-major, b) ───────────
// Each row is the fused dot product fma(A_in, x_n, ... fma(A_i2, x_2, A_i1 x_1)), then
// fma(0.1, (x_i x_i) x_i, row) - b_i.
template <int N_> struct CubicAffine {
    static constexpr int N = N_, M = N_;
    static constexpr bool lsq = false, analytic_J = false;
    const double* p;
    template <class S> void F(const S* x, S* out) const {
        const double* A = p;
        const double* b = p + N * N;
        for (int i = 0; i < N; ++i) {
            S t = A[i] * x[0];
            for (int j = 1; j < N; ++j) t = fmac(A[i + j * N], x[j], t);
            S c = x[i] * x[i] * x[i];
            out[i] = fmac(0.1, c, t) - b[i];
        }
    }
    void J(const double*, double*) const {}
};

// ─── GSB_FAMILY_WOOD: Wood's function with the coupling weight w = p[0] ─────────────────────
// Problem 4 of test/helpers/standard_problems.jl (w = 20.2 there), generic over double and Dual.
struct Wood {
    static constexpr int N = 4, M = 4;
    static constexpr bool lsq = false, analytic_J = false;
    const double* p;
    template <class S> void F(const S* x, S* out) const {
        const double w = p[0];
        S t1 = x[1] - x[0] * x[0];
        S t2 = x[3] - x[2] * x[2];
        out[0] = -200.0 * x[0] * t1 - (1.0 - x[0]);
        out[1] = 200.0 * t1 + w * (x[1] - 1.0) + 19.8 * (x[3] - 1.0);
        out[2] = -180.0 * x[2] * t2 - (1.0 - x[2]);
        out[3] = 180.0 * t2 + w * (x[3] - 1.0) + 19.8 * (x[1] - 1.0);
    }
    void J(const double*, double*) const {}
};

// ─── GSB_FAMILY_EXPSUM3_LSQ: r_i = a1 e^{-b1 t_i} + a2 e^{-b2 t_i} + a3 e^{-b3 t_i} - y_i ──────
// x = (a1, b1, a2, b2, a3, b3), p = y (M values), t = the shared abscissae.
template <int M_> struct ExpSum3 {
    static constexpr int N = 6, M = M_;
    static constexpr bool lsq = true, analytic_J = false;
    const double* y;
    const double* t;
    template <class S> void F(const S* x, S* out) const {
        for (int i = 0; i < M; ++i) {
            S e1 = fam_exp(-(x[1] * t[i]));
            S e2 = fam_exp(-(x[3] * t[i]));
            S e3 = fam_exp(-(x[5] * t[i]));
            out[i] = ((x[0] * e1 + x[2] * e2) + x[4] * e3) - y[i];
        }
    }
    void J(const double*, double*) const {}
};

// ─── GSB_FAMILY_IRK3_HENON_HEILES: G(Z) = Z - h (A ⊗ I) f(y + Z) ──────────────────────────────
// Z = (Z_1, Z_2, Z_3) stacked stage increments in R^4, y = (q1, q2, p1, p2), f the
// Hénon–Heiles field (p1, p2, -q1 - 2 q1 q2, -q2 - q1^2 + q2^2). shared = (h, A col-major 3x3).
// The accumulation order is that of the stage residual of test/helpers/stage_problems.jl:
// 205-222: G = Z, then for each stage j, Y = y + Z_j and G_i -= (h A_ij) f(Y) for every i.
struct IrkHenonHeiles {
    static constexpr int N = 12, M = 12;
    static constexpr bool lsq = false, analytic_J = false;
    const double* y;
    const double* shared;
    template <class S> static void field(const S* Y, S* f) {
        f[0] = Y[2];
        f[1] = Y[3];
        f[2] = -Y[0] - 2.0 * (Y[0] * Y[1]);
        f[3] = (-Y[1] - Y[0] * Y[0]) + Y[1] * Y[1];
    }
    template <class S> void F(const S* Z, S* out) const {
        const double h = shared[0];
        const double* A = shared + 1;
        for (int k = 0; k < 12; ++k) out[k] = Z[k];
        for (int j = 0; j < 3; ++j) {
            S Y[4], f[4];
            for (int k = 0; k < 4; ++k) Y[k] = y[k] + Z[4 * j + k];
            field(Y, f);
            for (int i = 0; i < 3; ++i) {
                double a = h * A[i + 3 * j];
                for (int k = 0; k < 4; ++k) out[4 * i + k] = out[4 * i + k] - a * f[k];
            }
        }
    }
    void J(const double*, double*) const {}
};

// ─── test/nonlinear/batched.jl:54-90, the six-outcome residual with its analytic J ─────────
struct Hetero6 {
    static constexpr int N = 2, M = 2;
    static constexpr bool lsq = false, analytic_J = true;
    const double* p;  // p[0] = outcome 1..6
    int code() const { return int(p[0]); }
    void F(const double* x, double* out) const {
        switch (code()) {
        case 1: out[0] = x[0] - 2.0; out[1] = x[1] - 3.0; break;
        case 2: out[0] = 1.0; out[1] = 1.0; break;
        case 3: out[0] = x[0] - 100.0; out[1] = x[1] - 100.0; break;
        case 4: out[0] = 1.0; out[1] = 1.0; break;
        case 5: out[0] = kNaN; out[1] = kNaN; break;
        default: out[0] = x[0] * x[0] + 1.0; out[1] = x[1] * x[1] + 1.0; break;
        }
    }
    template <int K> void F(const Dual<K>*, Dual<K>*) const {}
    void J(const double*, double* J) const {
        double d;
        switch (code()) {
        case 1: d = 1.0; break;
        case 2: d = 1e16; break;
        case 3: d = 2.0; break;
        case 4: d = 0.0; break;
        case 5: d = 1.0; break;
        default: d = -1.0; break;
        }
        J[0] = d; J[1] = 0.0; J[2] = 0.0; J[3] = d;
    }
};

// ─── test/nonlinear/batched.jl:92-104, the coupled 2-D residual with its analytic J ─────────
struct Coupled2 {
    static constexpr int N = 2, M = 2;
    static constexpr bool lsq = false, analytic_J = true;
    const double* p;
    void F(const double* x, double* out) const {
        out[0] = x[0] + (x[1] * x[1]) / 8.0 - p[0];
        out[1] = x[1] + (x[0] * x[0]) / 8.0 - p[1];
    }
    template <int K> void F(const Dual<K>*, Dual<K>*) const {}
    void J(const double* x, double* J) const {
        J[0] = 1.0;
        J[1] = x[0] / 4.0;
        J[2] = x[1] / 4.0;
        J[3] = 1.0;
    }
};

// ─── test/nonlinear/refinement.jl:40-96, u = A x, F = (u1 + 0.1 u1^2 - b1, u2 - 0.2 u2^2 - b2),
// J = Diagonal(1 + 0.2 u1, 1 - 0.4 u2) A; p = (A column-major 2x2, b) ─────────────────────
struct QuadMod2 {
    static constexpr int N = 2, M = 2;
    static constexpr bool lsq = false, analytic_J = true;
    const double* p;
    void u(const double* x, double* uu) const {
        uu[0] = p[0] * x[0] + p[2] * x[1];
        uu[1] = p[1] * x[0] + p[3] * x[1];
    }
    void F(const double* x, double* out) const {
        double uu[2];
        u(x, uu);
        out[0] = (uu[0] + 0.1 * (uu[0] * uu[0])) - p[4];
        out[1] = (uu[1] - 0.2 * (uu[1] * uu[1])) - p[5];
    }
    template <int K> void F(const Dual<K>*, Dual<K>*) const {}
    void J(const double* x, double* J) const {
        double uu[2];
        u(x, uu);
        double d0 = 1.0 + 0.2 * uu[0], d1 = 1.0 - 0.4 * uu[1];
        J[0] = d0 * p[0];
        J[1] = d1 * p[1];
        J[2] = d0 * p[2];
        J[3] = d1 * p[3];
    }
};

// ─── test/nonlinear/refinement.jl:686-725 (Check 1): F = A x .+ c .* x.^3 .- b,
// J = A + Diagonal(3 .* c .* x.^2); p = (A column-major 2x2, c, b) ──────────────────────
struct CubicDiag2 {
    static constexpr int N = 2, M = 2;
    static constexpr bool lsq = false, analytic_J = true;
    const double* p;
    void F(const double* x, double* out) const {
        for (int i = 0; i < 2; ++i) {
            double ax = p[i] * x[0] + p[i + 2] * x[1];
            out[i] = (ax + p[4 + i] * ((x[i] * x[i]) * x[i])) - p[6 + i];
        }
    }
    template <int K> void F(const Dual<K>*, Dual<K>*) const {}
    void J(const double* x, double* J) const {
        J[0] = p[0] + (3.0 * p[4]) * (x[0] * x[0]);
        J[1] = p[1];
        J[2] = p[2];
        J[3] = p[3] + (3.0 * p[5]) * (x[1] * x[1]);
    }
};

}  // namespace orc
