// The per-system Levenberg–Marquardt solve of a least-squares batch: one CUDA thread runs the R1
// loop `solve!!` (src/nonlinear/solver.jl:277-378) with the LevenbergMarquardt step of
// src/nonlinear/newton.jl:1897-1971 on the stacked QR path (src/globalization/
// levenbergmarquardt.jl:349-584, scaling = :none), for a residual of M rows in N unknowns.
//
// Nothing of size M is stored. The Jacobian pass generates the rows [J_i | -F_i] one at a time
// (forward-mode rules of ForwardDiff, written out for the residual family) and folds each one
// at once into the gradient J'F, the squared Frobenius norm of J, and the stacked Givens
// reduction to the triangle R0 and c0 = Q'(-F) (lm_qr_factor!, levenbergmarquardt.jl:359-421):
// the first N rows as a block reduced column by column, then every further row rotated into the
// triangle. A trial (lm_step_damping and lm_qr_solve!, levenbergmarquardt.jl:425-482, 575-584)
// works on the N x N triangle only. The predicted reduction -2 F'(J d) - |J d|^2 (newton.jl:
// 1934-1944) is formed from the same orthogonal factorisation: with u = R0 d it is
// 2 c0'u - |u|^2, and the fallback |F + J d| is sqrt(|u - c0|^2 + |w|^2), w the residual
// components the rotations moved out of the triangle. These equal the reference's expressions in
// exact arithmetic; the rounding differs, as it already does through `exp`.
#pragma once

#include "../../include/gsb.h"
#include "gsb_exp.h"
#include "gsb_newton.cuh"
#include "gsb_numerics.cuh"

namespace gsb {

// r_i = sum_j a_j exp(-b_j t_i) - y_i with x = (a1, b1, a2, b2, a3, b3): the residual of the
// exponential-sum fit. `y` (M observations of this system) and `t` (M abscissae shared by the
// batch) are in shared memory.
template <int M_> struct ExpSum3 {
    static constexpr int N = 6, M = M_, NP = M_;
    static constexpr bool lsq = true;
    const double* y;
    const double* t;

    __device__ __forceinline__ double yv(int i) const { return lds(smem_addr(y) + 8u * i); }
    __device__ __forceinline__ double tv(int i) const { return lds(smem_addr(t) + 8u * i); }

    // F_i(x): ((a1 e1 + a2 e2) + a3 e3) - y_i with e_j = exp(-(b_j t_i)), exp being
    // gsb_exp::exp (Tang's method, the same bits on the host).
    template <bool F> __device__ __forceinline__ double residual(const double (&x)[6], int i) const {
        using A = Arith<F>;
        const double ti = tv(i);
        const double e1 = gsb_exp::exp(-A::mul(x[1], ti));
        const double e2 = gsb_exp::exp(-A::mul(x[3], ti));
        const double e3 = gsb_exp::exp(-A::mul(x[5], ti));
        return A::sub(A::madd(x[4], e3, A::madd(x[2], e2, A::mul(x[0], e1))), yv(i));
    }

    // F_i(x) and the Jacobian row by the dual rules with seeded identity partials: the partial
    // of a_j is e_j; that of b_j is (e_j (-t_i)) a_j (exp rule e * (-(1 t)), then the product
    // rule with the structurally zero partial of a_j). The value part is `residual`.
    template <bool F>
    __device__ __forceinline__ double row(const double (&x)[6], int i, double (&J)[6]) const {
        using A = Arith<F>;
        const double ti = tv(i);
        const double e1 = gsb_exp::exp(-A::mul(x[1], ti));
        const double e2 = gsb_exp::exp(-A::mul(x[3], ti));
        const double e3 = gsb_exp::exp(-A::mul(x[5], ti));
        J[0] = e1;
        J[1] = A::mul(A::mul(e1, -ti), x[0]);
        J[2] = e2;
        J[3] = A::mul(A::mul(e2, -ti), x[2]);
        J[4] = e3;
        J[5] = A::mul(A::mul(e3, -ti), x[4]);
        return A::sub(A::madd(x[4], e3, A::madd(x[2], e2, A::mul(x[0], e1))), yv(i));
    }
};

// Julia's LinearAlgebra.givens(f, g, 1, 2) for real arguments (LAPACK's DLARTG as Julia's
// givensAlgorithm states it): c, s, r with [c s; -s c] [f; g] = [r; 0]. The rescaling loops for
// |f|, |g| outside [2^-485, 2^485] are out of line.
constexpr double kSafmn2 = 1.2486130624093112e-146;  // 2^-485
constexpr double kSafmx2 = 8.0088483185531275e+145;  // 2^485

template <bool F>
static __device__ __noinline__ void givens_rescaled(double f1, double g1, double& cs, double& sn,
                                                    double& r) {
    using A = Arith<F>;
    double scale = jmax(fabs(f1), fabs(g1));
    int count = 0;
    if (scale >= kSafmx2) {
        while (true) {
            ++count;
            f1 = A::mul(f1, kSafmn2);
            g1 = A::mul(g1, kSafmn2);
            scale = jmax(fabs(f1), fabs(g1));
            if (scale < kSafmx2 || count >= 20) break;
        }
        r = __dsqrt_rn(A::madd(g1, g1, A::mul(f1, f1)));
        cs = __ddiv_rn(f1, r);
        sn = __ddiv_rn(g1, r);
        for (int i = 0; i < count; ++i) r = A::mul(r, kSafmx2);
    } else {
        while (true) {
            ++count;
            f1 = A::mul(f1, kSafmx2);
            g1 = A::mul(g1, kSafmx2);
            scale = jmax(fabs(f1), fabs(g1));
            if (scale > kSafmn2) break;
        }
        r = __dsqrt_rn(A::madd(g1, g1, A::mul(f1, f1)));
        cs = __ddiv_rn(f1, r);
        sn = __ddiv_rn(g1, r);
        for (int i = 0; i < count; ++i) r = A::mul(r, kSafmn2);
    }
}

template <bool F>
__device__ __forceinline__ void givens(double f, double g, double& cs, double& sn, double& r) {
    using A = Arith<F>;
    if (g == 0.0) {
        cs = 1.0;
        sn = 0.0;
        r = f;
        return;
    }
    if (f == 0.0) {
        cs = 0.0;
        sn = 1.0;
        r = g;
        return;
    }
    const double scale = jmax(fabs(f), fabs(g));
    if (scale >= kSafmx2 || scale <= kSafmn2) {
        givens_rescaled<F>(f, g, cs, sn, r);
    } else if constexpr (F) {
        // fused arithmetic: one reciprocal square root in place of a square root and two
        // divisions (the rotation agrees with the reference's to rounding)
        const double q = A::madd(g, g, A::mul(f, f));
        const double ri = rsqrt(q);
        r = A::mul(q, ri);
        cs = A::mul(f, ri);
        sn = A::mul(g, ri);
    } else {
        r = __dsqrt_rn(A::madd(g, g, A::mul(f, f)));
        cs = __ddiv_rn(f, r);
        sn = __ddiv_rn(g, r);
    }
    if (fabs(f) > fabs(g) && cs < 0.0) {
        cs = -cs;
        sn = -sn;
        r = -r;
    }
}

// The FP32 rotation of the FP32 stacked factor (the mixed form): one reciprocal square root;
// arguments whose squares leave the FP32 range take the FP64 rotation.
template <bool F>
__device__ __forceinline__ void givens(float f, float g, float& cs, float& sn, float& r) {
    using A = Arith<F>;
    if (g == 0.0f) {
        cs = 1.0f;
        sn = 0.0f;
        r = f;
        return;
    }
    if (f == 0.0f) {
        cs = 0.0f;
        sn = 1.0f;
        r = g;
        return;
    }
    const float scale = fmaxf(fabsf(f), fabsf(g));
    if (!(scale < 1.0e18f && scale > 1.0e-18f)) {
        double c2, s2, r2;
        givens<F>((double)f, (double)g, c2, s2, r2);
        cs = (float)c2;
        sn = (float)s2;
        r = (float)r2;
        return;
    }
    const float q = A::madd(g, g, A::mul(f, f));
    const float ri = rsqrtf(q);
    r = A::mul(q, ri);
    cs = A::mul(f, ri);
    sn = A::mul(g, ri);
    if (fabsf(f) > fabsf(g) && cs < 0.0f) {
        cs = -cs;
        sn = -sn;
        r = -r;
    }
}

// (u, v) <- (c u + s v, -s u + c v)
template <bool F, class T> __device__ __forceinline__ void rotate(T cs, T sn, T& u, T& v) {
    using A = Arith<F>;
    const T nu = A::madd(cs, u, A::mul(sn, v));
    const T nv = A::madd(cs, v, A::mul(-sn, u));
    u = nu;
    v = nv;
}

// Fold the row (w | wr) into the triangle (R, c) from column k0 on: the row loop of
// lm_qr_factor! and of the damping rows. Returns the residual component left in wr.
template <bool F, int N, class T>
__device__ __forceinline__ T fold_row(T (&R)[N * N], T (&c)[N], T (&w)[N], T wr, int k0) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
        if (k < k0) continue;
        const T b = w[k];
        if (b == T(0)) continue;
        T cs, sn, rv;
        givens<F>(R[k + k * N], b, cs, sn, rv);
        R[k + k * N] = rv;
        w[k] = T(0);
#pragma unroll
        for (int l = k + 1; l < N; ++l) rotate<F, T>(cs, sn, R[k + l * N], w[l]);
        rotate<F, T>(cs, sn, c[k], wr);
    }
    return wr;
}

// The stacked factorisation of one Jacobian pass: R0 (upper triangle of R), c0, and the sum of
// squares of the components rotated out.
template <int N> struct StackedQR {
    double R[N * N];
    double c[N];
    double rest2;
};

// The mixed form's factorisation of one Jacobian pass: the FP32 stacked triangle, and in FP64
// the Gram matrix J'J (upper triangle, row by row) and the gradient J'F, from which the
// refinement's residuals and the predicted reduction are formed.
template <int N> struct MixedQR {
    float R[N * N];
    float c[N];
    double G[N * (N + 1) / 2];
    double g[N];
    bool fits;  // every row entry within the FP32 range
};

template <int N> __host__ __device__ constexpr int gram_index(int k, int l) {
    return k * N - k * (k - 1) / 2 + (l - k);  // k <= l
}

template <class Fam, bool F, bool Mixed = false> struct LMSolver {
    static constexpr int N = Fam::N, M = Fam::M;
    using A = Arith<F>;
    const Fam& fam;
    const GsbMethod& m;
    const GsbOptions& o;

    struct State {
        double mu, fnorm, fmax, gradratio, jnorm;
    };

    __device__ LMSolver(const Fam& f, const GsbMethod& mm, const GsbOptions& oo)
        : fam(f), m(mm), o(oo) {}

    // rnorm(F(x)) with its scaled fallback (src/base/reductions.jl:348-364) and maximum(abs,
    // F(x)) (reductions.jl:374), over the residual rows as they are generated.
    __device__ void fnorms(const double (&x)[N], double& fn, double& fmax) const {
        double s = 0.0, mx = 0.0;
#pragma unroll 1
        for (int i = 0; i < M; ++i) {
            const double r = fam.template residual<F>(x, i);
            s = i == 0 ? A::mul(r, r) : A::madd(r, r, s);
            mx = i == 0 ? fabs(r) : jmax(mx, fabs(r));
        }
        fmax = mx;
        if (isfin(s) && s >= double(M) * kFloatmin) {
            fn = __dsqrt_rn(s);
            return;
        }
        if (mx == 0.0 || !isfin(mx)) {
            fn = mx;
            return;
        }
        const int e = jexponent(mx);
        double acc = 0.0;
#pragma unroll 1
        for (int i = 0; i < M; ++i) {
            const double u = ldexp2_slow(fam.template residual<F>(x, i), -e);
            acc = i == 0 ? A::mul(u, u) : A::madd(u, u, acc);
        }
        fn = ldexp2_slow(__dsqrt_rn(acc), e);
    }

    // The Jacobian pass at x: grad_ratio_and_norm (newton.jl:1287-1298) into the state, the
    // finiteness of J, and (QR = true) the stacked factorisation of [J | -F].
    template <bool QR>
    __device__ void jacobian_pass(const double (&x)[N], double fnorm, State& st, StackedQR<N>& q,
                                  bool& finite) const {
        jacobian_pass_impl<QR ? 1 : 0>(x, fnorm, st, &q, nullptr, finite);
    }
    __device__ void jacobian_pass_mixed(const double (&x)[N], double fnorm, State& st,
                                        MixedQR<N>& q, bool& finite) const {
        jacobian_pass_impl<2>(x, fnorm, st, nullptr, &q, finite);
    }

    // Mode 0: the diagnostics only; 1: and the FP64 stacked factor; 2: and the FP32 stacked
    // factor with the FP64 Gram matrix and gradient (the mixed form).
    template <int Mode>
    __device__ void jacobian_pass_impl(const double (&x)[N], double fnorm, State& st,
                                       StackedQR<N>* qp, MixedQR<N>* qmp, bool& finite) const {
        StackedQR<N>& q = *qp;   // bound only where Mode == 1 reads it
        MixedQR<N>& qm = *qmp;   // bound only where Mode == 2 reads it
        constexpr bool QR = Mode == 1;
        double g[N];
        double js = 0.0, jm = 0.0;
        bool fin = true;
        bool fits = true;
        double rest2 = 0.0;
        if constexpr (Mode == 2) {
#pragma unroll
            for (int k = 0; k < N * (N + 1) / 2; ++k) qm.G[k] = 0.0;
        }
        // rows 0..N-1: the block of R0 and c0, reduced column by column
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double J[N];
            const double r = fam.template row<F>(x, i, J);
#pragma unroll
            for (int k = 0; k < N; ++k) {
                g[k] = i == 0 ? A::mul(J[k], r) : A::madd(J[k], r, g[k]);
                js = (i == 0 && k == 0) ? A::mul(J[k], J[k]) : A::madd(J[k], J[k], js);
                jm = (i == 0 && k == 0) ? fabs(J[k]) : jmax(jm, fabs(J[k]));
                fin = fin && isfin(J[k]);
                if constexpr (QR) q.R[i + k * N] = J[k];
                if constexpr (Mode == 2) {
                    qm.R[i + k * N] = (float)J[k];
                    fits = fits && isfinite(qm.R[i + k * N]);
#pragma unroll
                    for (int l = k; l < N; ++l)
                        qm.G[gram_index<N>(k, l)] = A::madd(J[k], J[l], qm.G[gram_index<N>(k, l)]);
                }
            }
            if constexpr (QR) q.c[i] = -r;
            if constexpr (Mode == 2) {
                qm.c[i] = -(float)r;
                fits = fits && isfinite(qm.c[i]);
            }
        }
        if constexpr (Mode == 2) {
#pragma unroll
            for (int j = 0; j < N; ++j)
#pragma unroll
                for (int i = j + 1; i < N; ++i) {
                    const float b = qm.R[i + j * N];
                    if (b == 0.0f) continue;
                    float cs, sn, rv;
                    givens<F>(qm.R[j + j * N], b, cs, sn, rv);
                    qm.R[j + j * N] = rv;
                    qm.R[i + j * N] = 0.0f;
#pragma unroll
                    for (int k = j + 1; k < N; ++k) rotate<F, float>(cs, sn, qm.R[j + k * N], qm.R[i + k * N]);
                    rotate<F, float>(cs, sn, qm.c[j], qm.c[i]);
                }
        }
        if constexpr (QR) {
#pragma unroll
            for (int j = 0; j < N; ++j)
#pragma unroll
                for (int i = j + 1; i < N; ++i) {
                    const double b = q.R[i + j * N];
                    if (b == 0.0) continue;
                    double cs, sn, rv;
                    givens<F>(q.R[j + j * N], b, cs, sn, rv);
                    q.R[j + j * N] = rv;
                    q.R[i + j * N] = 0.0;
#pragma unroll
                    for (int k = j + 1; k < N; ++k) rotate<F, double>(cs, sn, q.R[j + k * N], q.R[i + k * N]);
                    rotate<F, double>(cs, sn, q.c[j], q.c[i]);
                }
        }
        // rows N..M-1, each rotated into the triangle as it is generated
#pragma unroll 1
        for (int i = N; i < M; ++i) {
            double J[N];
            const double r = fam.template row<F>(x, i, J);
#pragma unroll
            for (int k = 0; k < N; ++k) {
                g[k] = A::madd(J[k], r, g[k]);
                js = A::madd(J[k], J[k], js);
                jm = jmax(jm, fabs(J[k]));
                fin = fin && isfin(J[k]);
            }
            if constexpr (QR) {
                const double wr = fold_row<F, N, double>(q.R, q.c, J, -r, 0);
                rest2 = A::madd(wr, wr, rest2);
            }
            if constexpr (Mode == 2) {
                float Jf[N];
#pragma unroll
                for (int k = 0; k < N; ++k) {
                    Jf[k] = (float)J[k];
                    fits = fits && isfinite(Jf[k]);
#pragma unroll
                    for (int l = k; l < N; ++l)
                        qm.G[gram_index<N>(k, l)] = A::madd(J[k], J[l], qm.G[gram_index<N>(k, l)]);
                }
                const float rf = -(float)r;
                fits = fits && isfinite(rf);
                fold_row<F, N, float>(qm.R, qm.c, Jf, rf, 0);
            }
        }
        if constexpr (QR) q.rest2 = rest2;
        if constexpr (Mode == 2) {
#pragma unroll
            for (int k = 0; k < N; ++k) {
                qm.g[k] = g[k];
                fits = fits && isfinite(qm.R[k + k * N]);
            }
            qm.fits = fits;
        }
        finite = fin;
        // ‖J‖_F: rnorm over the M N entries, with its scaled fallback
        double jnorm;
        if (isfin(js) && js >= double(M * N) * kFloatmin) {
            jnorm = __dsqrt_rn(js);
        } else if (jm == 0.0 || !isfin(jm)) {
            jnorm = jm;
        } else {
            const int e = jexponent(jm);
            double acc = 0.0;
#pragma unroll 1
            for (int i = 0; i < M; ++i) {
                double J[N];
                fam.template row<F>(x, i, J);
#pragma unroll
                for (int k = 0; k < N; ++k) {
                    const double u = ldexp2_slow(J[k], -e);
                    acc = (i == 0 && k == 0) ? A::mul(u, u) : A::madd(u, u, acc);
                }
            }
            jnorm = ldexp2_slow(__dsqrt_rn(acc), e);
        }
        st.jnorm = jnorm;
        if (jnorm == 0.0 || fnorm == 0.0) {
            st.gradratio = 0.0;
            return;
        }
        double gnorm = rnorm<F, N>(g);
        if (isfin(gnorm) || !(isfin(jnorm) && isfin(fnorm))) {
            st.gradratio = __ddiv_rn(__ddiv_rn(gnorm, jnorm), fnorm);
            return;
        }
        // J'F overflowed: the gradient of F / 2^e (newton.jl:1293-1297)
        const int e = jexponent(fnorm);
#pragma unroll 1
        for (int i = 0; i < M; ++i) {
            double J[N];
            const double r = ldexp2_slow(fam.template row<F>(x, i, J), -e);
#pragma unroll
            for (int k = 0; k < N; ++k) g[k] = i == 0 ? A::mul(J[k], r) : A::madd(J[k], r, g[k]);
        }
        st.gradratio = __ddiv_rn(__ddiv_rn(rnorm<F, N>(g), jnorm), ldexp2_slow(fnorm, -e));
    }

    // One damped solve on the triangle: the rows sqrt(mu) e_j folded into (R0, c0), then back
    // substitution. False when the damping or the solution is not finite or R is singular.
    __device__ bool trial(const StackedQR<N>& q, double mu, double (&d)[N]) const {
        const double damp = mu < 4.0 * kEps ? 0.0 : mu;
        const double sq = __dsqrt_rn(damp);
        if (!isfin(sq) || !isfin(A::mul(sq, 1.0))) {
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = 0.0;
            return false;
        }
        double R[N * N], c[N];
#pragma unroll
        for (int k = 0; k < N * N; ++k) R[k] = q.R[k];
#pragma unroll
        for (int k = 0; k < N; ++k) c[k] = q.c[k];
        // the damping rows sqrt(mu) e_j, one at a time (a runtime loop over one copy of the
        // row fold, which skips the columns before j)
        const double sq1 = A::mul(sq, 1.0);
#pragma unroll 1
        for (int j = 0; j < N; ++j) {
            double w[N];
#pragma unroll
            for (int k = 0; k < N; ++k) w[k] = k == j ? sq1 : 0.0;
            fold_row<F, N, double>(R, c, w, 0.0, j);
        }
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = 0.0;
        bool ok = true;
#pragma unroll
        for (int i = N - 1; i >= 0; --i) {
            double s = c[i];
#pragma unroll
            for (int j = i + 1; j < N; ++j) s = A::msub(R[i + j * N], d[j], s);
            const double rii = R[i + i * N];
            ok = ok && rii != 0.0 && isfin(rii);
            d[i] = ok ? __ddiv_rn(s, rii) : 0.0;
        }
        if (!ok) {
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = 0.0;
            return false;
        }
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (!isfin(d[i])) return false;
        return true;
    }

    // The predicted reduction |F|^2 - |F + J d|^2 from the factorisation (see the file head).
    __device__ double predicted(const StackedQR<N>& q, const double (&d)[N], double fnorm) const {
        double u[N];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double s = A::mul(q.R[i + i * N], d[i]);
#pragma unroll
            for (int j = i + 1; j < N; ++j) s = A::madd(q.R[i + j * N], d[j], s);
            u[i] = s;
        }
        double cu = A::mul(q.c[0], u[0]), uu = A::mul(u[0], u[0]);
#pragma unroll
        for (int i = 1; i < N; ++i) {
            cu = A::madd(q.c[i], u[i], cu);
            uu = A::madd(u[i], u[i], uu);
        }
        double pred = A::sub(A::mul(2.0, cu), uu);
        if (pred <= 0.0) {
            double l2 = q.rest2;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const double v = A::sub(u[i], q.c[i]);
                l2 = A::madd(v, v, l2);
            }
            const double fl = __dsqrt_rn(l2);
            pred = A::mul(A::sub(fnorm, fl), A::add(fnorm, fl));
        }
        return pred;
    }

    // The mixed form's trial: the damped FP32 triangle and back substitution, then refinement
    // of d against the FP64 residual of the damped normal equations,
    // r = -J'F - (J'J + damp I) d, solved on the same triangle (R' R = J'J + damp I).
    __device__ bool trial(const MixedQR<N>& q, double mu, double (&d)[N]) const {
        const double damp = mu < 4.0 * kEps ? 0.0 : mu;
        const double sq = __dsqrt_rn(damp);
        if (!isfin(sq) || !isfin(A::mul(sq, 1.0))) {
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = 0.0;
            return false;
        }
        float R[N * N], c[N];
#pragma unroll
        for (int k = 0; k < N * N; ++k) R[k] = q.R[k];
#pragma unroll
        for (int k = 0; k < N; ++k) c[k] = q.c[k];
        const float sqf = (float)A::mul(sq, 1.0);
#pragma unroll 1
        for (int j = 0; j < N; ++j) {
            float w[N];
#pragma unroll
            for (int k = 0; k < N; ++k) w[k] = k == j ? sqf : 0.0f;
            fold_row<F, N, float>(R, c, w, 0.0f, j);
        }
        float df[N];
        bool ok = true;
#pragma unroll
        for (int i = N - 1; i >= 0; --i) {
            float s = c[i];
#pragma unroll
            for (int j = i + 1; j < N; ++j) s = Arith<F>::msub(R[i + j * N], df[j], s);
            ok = ok && R[i + i * N] != 0.0f && isfinite(R[i + i * N]);
            df[i] = ok ? s / R[i + i * N] : 0.0f;
        }
#pragma unroll
        for (int i = 0; i < N; ++i) {
            d[i] = (double)df[i];
            ok = ok && isfin(d[i]);
        }
        if (!ok) return false;
        // refinement passes (the Refinement parameters of the method: eta, maxiter)
        double r[N];
        auto residual = [&](const double (&v)[N], double (&out)[N]) {
#pragma unroll
            for (int a = 0; a < N; ++a) {
                double t = A::madd(damp, v[a], q.g[a]);
#pragma unroll
                for (int b = 0; b < N; ++b)
                    t = A::madd(q.G[a <= b ? gram_index<N>(a, b) : gram_index<N>(b, a)], v[b], t);
                out[a] = -t;
            }
        };
        residual(d, r);
        const double thr = A::mul(jmax(m.refine_eta, kSqrtEps), rnorm<F, N>(q.g));
        double rprev = rnorm<F, N>(r);
        for (int it = 0; it < m.refine_maxiter && isfin(rprev) && rprev > thr; ++it) {
            double sc = fabs(r[0]);
#pragma unroll
            for (int a = 1; a < N; ++a) sc = jmax(sc, fabs(r[a]));
            if (!(sc > 0.0) || !isfin(sc)) break;
            // R' y = r / sc (forward), then R z = y (back), in FP32
            float y[N];
#pragma unroll
            for (int a = 0; a < N; ++a) {
                float t = (float)(r[a] / sc);
#pragma unroll
                for (int b = 0; b < a; ++b) t = Arith<F>::msub(R[b + a * N], y[b], t);
                y[a] = t / R[a + a * N];
            }
#pragma unroll
            for (int a = N - 1; a >= 0; --a) {
                float t = y[a];
#pragma unroll
                for (int b = a + 1; b < N; ++b) t = Arith<F>::msub(R[a + b * N], y[b], t);
                y[a] = t / R[a + a * N];
            }
            double dc[N], rc[N];
#pragma unroll
            for (int a = 0; a < N; ++a) dc[a] = A::madd((double)y[a], sc, d[a]);
            residual(dc, rc);
            const double rn = rnorm<F, N>(rc);
            if (!(rn < rprev)) break;
#pragma unroll
            for (int a = 0; a < N; ++a) {
                d[a] = dc[a];
                r[a] = rc[a];
            }
            rprev = rn;
        }
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (!isfin(d[i])) return false;
        return true;
    }

    // The predicted reduction from the FP64 Gram matrix and gradient: -2 g'd - d'G d (the
    // reference's -2 F'(J d) - |J d|^2 in exact arithmetic); its fallback |F + J d|^2 =
    // |F|^2 + 2 g'd + d'G d.
    __device__ double predicted(const MixedQR<N>& q, const double (&d)[N], double fnorm) const {
        double gd = A::mul(q.g[0], d[0]);
#pragma unroll
        for (int a = 1; a < N; ++a) gd = A::madd(q.g[a], d[a], gd);
        double dGd = 0.0;
#pragma unroll
        for (int a = 0; a < N; ++a) {
            double t = 0.0;
#pragma unroll
            for (int b = 0; b < N; ++b)
                t = A::madd(q.G[a <= b ? gram_index<N>(a, b) : gram_index<N>(b, a)], d[b], t);
            dGd = A::madd(d[a], t, dGd);
        }
        double pred = A::sub(A::mul(-2.0, gd), dGd);
        if (pred <= 0.0) {
            const double fl2 = A::add(A::madd(2.0, gd, A::mul(fnorm, fnorm)), dGd);
            const double fl = __dsqrt_rn(fl2 > 0.0 ? fl2 : 0.0);
            pred = A::mul(A::sub(fnorm, fl), A::add(fnorm, fl));
        }
        return pred;
    }

    // The trials of one step on a factorisation (newton.jl:1906-1971): damped solve, predicted
    // and actual reduction, the gain ratio; mu grows after each rejected trial.
    template <class Q>
    __device__ void trials(const Q& q, State& st, double (&x)[N], StepInfo& info, double fnorm,
                           double mu, double mu_min_eff, bool promoted) const {
        int failures = 0;
        while (true) {
            double d[N];
            if (trial(q, mu, d)) {
                const double pred = predicted(q, d, fnorm);
                double xp[N];
#pragma unroll
                for (int i = 0; i < N; ++i) xp[i] = A::add(x[i], d[i]);
                double fnp, fmaxp;
                fnorms(xp, fnp, fmaxp);
                if (isfin(fnp) && pred > 0.0) {
                    const double ared = A::mul(A::sub(fnorm, fnp), A::add(fnorm, fnp));
                    const double rho = __ddiv_rn(ared, pred);
                    if (rho > m.lm_rho_accept) {
                        const bool limited = mu > m.lm_mu0;
                        const double mu_next = jmax(A::mul(mu, m.lm_mu_decrease), mu_min_eff);
                        const double stepnorm = rnorm<F, N>(d);
#pragma unroll
                        for (int i = 0; i < N; ++i) x[i] = xp[i];
                        st.fnorm = fnp;
                        st.fmax = fmaxp;
                        st.mu = mu_next;
                        info = {SUCCESS, fnp, stepnorm, failures, promoted, limited, false};
                        return;
                    }
                }
            }
            failures += 1;
            mu = jmax(A::mul(mu, m.lm_mu_increase), mu_min_eff);
            if (!isfin(mu) || mu > m.lm_mu_max) {
                st.mu = jmin(mu, kFloatmax);
                info = {STALLED, fnorm, 0.0, failures, promoted, false, false};
                return;
            }
        }
    }

    // The LevenbergMarquardt step, newton.jl:1897-1971. The mixed form factors in FP32 and
    // refines in FP64; a step whose rows leave the FP32 range is taken in FP64 (`promoted`).
    __device__ void step(State& st, double (&x)[N], StepInfo& info) const {
        const double fnorm = st.fnorm;
        const double mu = st.mu;
        if (!isfin(mu)) {
            info = {NONFINITE, fnorm, 0.0, 0, false, false, false};
            return;
        }
        if (fnorm == 0.0) {
            info = {SUCCESS, 0.0, 0.0, 0, false, false, false};
            return;
        }
        const double mu_min_eff = jmax(m.lm_mu_min, 4.0 * kEps);
        bool finite;
        if constexpr (Mixed) {
            MixedQR<N> qm;
            jacobian_pass_mixed(x, fnorm, st, qm, finite);
            if (!finite) {
                info = {NONFINITE, fnorm, 0.0, 0, false, false, false};
                return;
            }
            if (qm.fits) {
                trials(qm, st, x, info, fnorm, mu, mu_min_eff, false);
                return;
            }
        }
        StackedQR<N> q;
        jacobian_pass<true>(x, fnorm, st, q, finite);
        if (!finite) {
            info = {NONFINITE, fnorm, 0.0, 0, false, false, false};
            return;
        }
        trials(q, st, x, info, fnorm, mu, mu_min_eff, Mixed);
    }

    // stationary_converged, src/nonlinear/solver.jl:148-158.
    __device__ __forceinline__ bool stationary(const State& st, const DevStatus& s) const {
        if (!(s.iterations >= o.min_iterations)) return false;
        return st.jnorm > 0.0 && s.fnorm > 0.0 && st.gradratio <= o.g_tol;
    }

    // refresh_diagnostics!!, newton.jl:807-822: the diagnostics at the new iterate.
    __device__ void refresh(State& st, const double (&x)[N]) const {
        StackedQR<N> unused;
        bool finite;
        jacobian_pass<false>(x, st.fnorm, st, unused, finite);
    }

    __device__ static void close(DevStatus& s, int code, bool stationary, bool contracted) {
        s.code = code;
        s.stationary = stationary;
        s.contracted = contracted;
    }

    __device__ __forceinline__ bool residual_converged(const DevStatus& s, double ft,
                                                       double ft0) const {
        if (!(s.iterations >= o.min_iterations)) return false;
        return ft <= jmax(o.f_abstol, A::mul(o.f_reltol, ft0));
    }

    // solve!!, src/nonlinear/solver.jl:277-378, with the least-squares branches (stationarity,
    // re-measured diagnostics, the discarded step of keeps_step_start, solver.jl:183-189 and
    // 330-339), as a run that advances one step at a time: `begin` takes the start (and may
    // already close the run), each `iterate` one pass of the loop; `done` marks the close.
    // `gr` is the gradratio of the last diagnostics (newton_finish!!).
    struct Run {
        State st;
        DevStatus s;
        double ftest0, gr;
        int stalls;
        bool done;
    };

    __device__ void begin(double (&x)[N], Run& r) const {
        State& st = r.st;
        DevStatus& s = r.s;
        fnorms(x, st.fnorm, st.fmax);
        st.mu = m.lm_mu0;
        st.gradratio = kNaN;
        st.jnorm = 0.0;
        s.code = SUCCESS;
        s.iterations = 0;
        s.fnorm = st.fnorm;
        s.stepnorm = 0.0;
        s.step_failures = 0;
        s.promoted = false;
        s.stationary = false;
        s.rate = kNaN;
        s.contracted = false;
        r.gr = kNaN;
        r.stalls = 0;
        r.done = true;
        if (!isfin(st.fnorm)) {
            close(s, NONFINITE, false, false);
            return;
        }
        r.ftest0 = o.norm == 1 ? st.fmax : st.fnorm;
        if (residual_converged(s, r.ftest0, r.ftest0)) return;
        if (o.max_iterations == 0) {
            close(s, MAXITERS, false, false);
            return;
        }
        r.done = false;
    }

    __device__ void iterate(double (&x)[N], Run& r) const {
        State& st = r.st;
        DevStatus& s = r.s;
        const double ftest0 = r.ftest0;
        r.done = true;
        double xk[N];
#pragma unroll
        for (int i = 0; i < N; ++i) xk[i] = x[i];
        const DevStatus sk = s;
        StepInfo info;
        step(st, x, info);
        record(s, info);
        const State st_step = st;
        r.gr = st.gradratio;
        if (info.code == SINGULAR || info.code == NONFINITE || info.code == MAXITERS) return;
        if (info.code == LINESEARCH_FAILED && info.stepnorm == 0.0 && !stationary(st, s)) return;
        if (residual_converged(s, o.norm == 1 ? st.fmax : s.fnorm, ftest0)) {
            close(s, SUCCESS, false, false);
            return;
        }
        bool refreshed = false;
        if (stationary(st, s)) {
            refresh(st, x);
            refreshed = true;
            r.gr = st.gradratio;
            if (stationary(st, s)) {
                close(s, SUCCESS, true, false);
                return;
            }
            if (sk.iterations >= 1 && s.fnorm >= sk.fnorm && stationary(st_step, sk)) {
                // discarded_step_status, solver.jl:103-109
#pragma unroll
                for (int i = 0; i < N; ++i) x[i] = xk[i];
                const int failures = s.step_failures;
                const bool promoted = s.promoted;
                s = sk;
                s.code = SUCCESS;
                s.step_failures = failures;
                s.promoted = promoted;
                s.stationary = true;
                s.contracted = false;
                r.gr = st_step.gradratio;
                return;
            }
        }
        const bool steptested = !(info.code == STALLED || info.limited);
        const double xnorm = steptested ? rnorm<F, N>(x) : kNaN;
        bool contracted = false;
        if (!info.shortened && o.rate_test && s.iterations >= o.min_iterations) {
            const double th = jmax(s.rate, sk.rate);
            if (s.stepnorm > 0.0 && th < 1.0)
                contracted = A::mul(__ddiv_rn(th, A::sub(1.0, th)), s.stepnorm) <=
                             A::mul(o.kappa, jmax(o.x_abstol, A::mul(o.x_reltol, xnorm)));
        }
        bool stepc = false;
        if (steptested && s.iterations >= o.min_iterations) {
            stepc = s.iterations > 0 && s.stepnorm > 0.0 &&
                    s.stepnorm <= jmax(o.x_abstol, A::mul(o.x_reltol, xnorm));
            stepc = stepc || (info.code == SUCCESS && info.stepnorm == 0.0);
            stepc = stepc || (o.roundoff && s.rate >= 1.0 && sk.rate < 1.0);
        }
        if (contracted || stepc) {
            if (!refreshed) {
                refresh(st, x);
                r.gr = st.gradratio;
            }
            if (stationary(st, s)) {
                close(s, SUCCESS, true, false);
                return;
            }
            close(s, contracted ? SUCCESS : STALLED, false, contracted);
            return;
        }
        if (info.code == STALLED) {
            r.stalls += 1;
            if (r.stalls >= o.max_stalls) {
                close(s, STALLED, false, false);
                return;
            }
        } else {
            r.stalls = 0;
        }
        if (s.iterations >= o.max_iterations) {
            close(s, MAXITERS, false, false);
            return;
        }
        r.done = false;
    }

    __device__ DevStatus solve(double (&x)[N], double& gr) const {
        Run r;
        begin(x, r);
        while (!r.done) iterate(x, r);
        gr = r.gr;
        return r.s;
    }
};

}  // namespace gsb
