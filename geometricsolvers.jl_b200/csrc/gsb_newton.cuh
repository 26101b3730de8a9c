// The per-system Newton solve of the batch: one CUDA thread runs GeometricSolvers.jl's R1 loop
// `solve!!` (src/nonlinear/solver.jl:277-378) for its system, with the iterate, the residual,
// the Jacobian, its pivoted factor and the direction in registers (every array index is a
// compile-time constant after unrolling; a pivot row is selected by predicated moves).
//
// Methods: Newton with LUFactorization{TF} (TF = Float64, or Float32 with Refinement and the
// promotion to Float64 of src/nonlinear/newton.jl:1604-1720), globalization Static or
// Backtracking. Status fields, codes and every stopping test follow the reference.
#pragma once
#include <type_traits>

#include "../../include/gsb.h"
#include "gsb_families.cuh"
#include "gsb_numerics.cuh"

namespace gsb {

struct StepInfo {
    int code;
    double fnorm, stepnorm;
    int failures;
    bool promoted, limited, shortened;
};

struct DevStatus {
    int code, iterations;
    double fnorm, stepnorm;
    int step_failures;
    bool promoted, stationary;
    double rate;
    bool contracted;
    bool reused = false;  // the last step stepped along a factor an earlier step formed
};

struct DevState {
    double merit, fnorm, gradratio, jnorm;
    bool promoted;
    int slow_steps;
    // FactorAge (src/nonlinear/newton.jl:621-625) of Newton(reuse = k): the age of the held
    // factor, whether it is to be refreshed, whether the last step reused it
    int age;
    bool stalled, reused;
    double radius;  // TrustRadius of DogLeg (newton.jl:637-640); 0 while unset
};

// The step of the Newton solve: the method's own (plain, or the mixed-precision step), the step
// with factor reuse, or the DogLeg trust-region step.
// kStepTrial32: the mixed step (Float32 factor with refinement) whose line-search trials run in
// Float32, a departure from the reference that has no counterpart there (see Solver::trial).
enum StepKind : int { kStepNewton = 0, kStepReuse = 1, kStepDogLeg = 2, kStepTrial32 = 3 };

// What a step that took the common course (Backtracking's first trial accepted at alpha = 1)
// already formed for the stopping tests that follow it, with their own operands and operations:
// record's rate, the norm of the new iterate, and the quotient th / (1 - th) of the rate test.
struct StepSpec {
    bool valid;
    double rate, xnorm, q;
};

// record(status, info), src/base/status.jl:245-262.
__device__ __forceinline__ void record(DevStatus& s, const StepInfo& i) {
    s.rate = s.stepnorm > 0.0 ? __ddiv_rn(i.stepnorm, s.stepnorm) : kNaN;
    s.code = i.code;
    s.iterations += 1;
    s.fnorm = i.fnorm;
    s.stepnorm = i.stepnorm;
    s.step_failures += i.failures;
    s.promoted = s.promoted || i.promoted;
}

// Exchange x and y where r == p, as two predicated selects. Written in PTX so that the front
// end cannot turn a row exchange over unrolled rows into an indexed access, which would move the
// whole register matrix to local memory. Both selects write PTX temporaries before either
// output is written, so an output that shares a register with an input cannot corrupt it.
__device__ __forceinline__ void cswap(int r, int p, double& x, double& y) {
    double nx, ny;
    asm("{\n\t.reg .pred q;\n\t.reg .f64 t0, t1;\n\tsetp.eq.s32 q, %2, %3;\n\t"
        "selp.f64 t0, %5, %4, q;\n\tselp.f64 t1, %4, %5, q;\n\tmov.f64 %0, t0;\n\t"
        "mov.f64 %1, t1;\n\t}"
        : "=d"(nx), "=d"(ny)
        : "r"(r), "r"(p), "d"(x), "d"(y));
    x = nx;
    y = ny;
}
__device__ __forceinline__ void cswap(int r, int p, float& x, float& y) {
    float nx, ny;
    asm("{\n\t.reg .pred q;\n\t.reg .f32 t0, t1;\n\tsetp.eq.s32 q, %2, %3;\n\t"
        "selp.f32 t0, %5, %4, q;\n\tselp.f32 t1, %4, %5, q;\n\tmov.f32 %0, t0;\n\t"
        "mov.f32 %1, t1;\n\t}"
        : "=f"(nx), "=f"(ny)
        : "r"(r), "r"(p), "f"(x), "f"(y));
    x = nx;
    y = ny;
}

// The pivoted LU of src/linear/static/lu.jl:24-64 on a register matrix, with the scaling of
// factor_matrix (src/linear/factors.jl:802-811): TF = T divides by 2^e only for e < 0; another
// TF divides for every e != 0, in T, then rounds to TF.
template <bool F, int N, class TF> struct LUFactor {
    // Under fused arithmetic the factor divides by multiplying with reciprocals: one of each
    // pivot, computed once and kept in place of the pivot for the back substitution (8 FP64
    // divisions instead of 36 at n = 8, where one division costs the FP64 pipe about 14 FMAs),
    // and, for the Float32 factor of the mixed step, one of the scale s of its right-hand sides.
    // The unfused arithmetic divides as lu.jl does.
    static constexpr bool kRecip = F;
    TF a[N * N];
    int ipiv[N];
    int info;
    int e;

    // J into the Float64 factor's registers, with the two sums that grad_ratio_and_norm takes
    // over J folded while each entry is in a register: s, the squares of the entries in column
    // order, and g = J' Fx, each in the order of that function's own loops, so the results are
    // the same bits and J is read from the family once per step instead of three times.
    template <class Fam, class JS, int M>
    __device__ __forceinline__ void load(const Fam& fam, const JS& js, const double (&Fx)[M],
                                         double& s, double (&g)[N]) {
        static_assert(sizeof(TF) == sizeof(double) && M == N, "the square Float64 factor");
        for_each_J(fam, js, [&](int i, int k, double v) {
            a[i + k * N] = v;
            s = (i == 0 && k == 0) ? Arith<F>::mul(v, v) : Arith<F>::madd(v, v, s);
            g[k] = i == 0 ? Arith<F>::mul(v, Fx[0]) : Arith<F>::madd(v, Fx[i], g[k]);
        });
    }

    // factor_matrix's scaling of the loaded J (J / 2^e in place), then the elimination. The
    // same-type scaling divides only for e < 0, that is when every |J_ik| < 1 (or the largest
    // is subnormal); an entry with |J_00| >= 1 settles e = 0 without the scan of all N^2.
    __device__ __forceinline__ void eliminate() {
        static_assert(sizeof(TF) == sizeof(double), "the Float64 factor");
        if (fabs(a[0]) >= 1.0) {
            e = 0;
        } else {
            e = matrix_exponent<N * N>(a);
            if (e < 0) {
#pragma unroll
                for (int q = 0; q < N * N; ++q) a[q] = scale2_in(a[q], -e);  // -e in [1, 1023]
            } else {
                e = 0;
            }
        }
        elimination();
    }

    template <class Fam, class JS>
    __device__ __forceinline__ void factor(const Fam& fam, const JS& js) {
        // J into the factor's registers, then J / 2^e in place (factor_matrix)
        constexpr bool same = sizeof(TF) == sizeof(double);
        if constexpr (same) {
            for_each_J(fam, js, [&](int i, int k, double v) { a[i + k * N] = v; });
            eliminate();
            return;
        } else {
            unsigned long long mb = 0;
            for_each_J(fam, js, [&](int, int, double v) {
                const unsigned long long b = FBits<double>::bits(v) & ~FBits<double>::sign_mask;
                mb = b > mb ? b : mb;
            });
            double mm = FBits<double>::from(mb);
            e = (isfin(mm) && mm != 0.0) ? max(-1023, min(1023, jexponent(mm))) : 0;
            for_each_J(fam, js, [&](int i, int k, double v) {
                a[i + k * N] = TF(e == 0 ? v : scale2_in(v, -e));  // -e in [-1023, 1023]
            });
        }
        elimination();
    }

    // The pivoted elimination of the scaled matrix (lu.jl:24-64).
    __device__ __forceinline__ void elimination() {
        info = 0;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            int p = k;
            // The pivot is the first largest |a_ik|, i >= k. When every entry below the
            // diagonal has a smaller magnitude key (the high word with the sign shifted out,
            // an integer order of |x|; NaN above every finite value) than a_kk, the diagonal
            // is that pivot; the search of compares runs only otherwise.
            unsigned below = 0;
#pragma unroll
            for (int i = k + 1; i < N; ++i) below = max(below, mag_key(a[i + k * N]));
            if (k + 1 < N && !(below < mag_key(a[k + k * N]))) {
                TF amax = fabs(a[k + k * N]);
#pragma unroll
                for (int i = k + 1; i < N; ++i) {
                    TF v = fabs(a[i + k * N]);
                    if (v > amax) {
                        amax = v;
                        p = i;
                    }
                }
            }
            ipiv[k] = p;
            if (p != k) {
#pragma unroll
                for (int i = k + 1; i < N; ++i)
#pragma unroll
                    for (int j = 0; j < N; ++j) cswap(i, p, a[k + j * N], a[i + j * N]);
            }
            TF akk = a[k + k * N];
            if (akk == TF(0)) {
                if (info == 0) info = k + 1;
            } else if constexpr (kRecip) {
                // the fused factor: one reciprocal per pivot (correctly rounded, the bits of
                // 1 / akk), kept in place of the pivot for the back substitution
                const TF r = crcp(akk);
                a[k + k * N] = r;
#pragma unroll
                for (int i = k + 1; i < N; ++i) a[i + k * N] = a[i + k * N] * r;
#pragma unroll
                for (int j = k + 1; j < N; ++j)
#pragma unroll
                    for (int i = k + 1; i < N; ++i)
                        a[i + j * N] = Arith<F>::msub(a[i + k * N], a[k + j * N], a[i + j * N]);
            } else {
#pragma unroll
                for (int i = k + 1; i < N; ++i) a[i + k * N] = a[i + k * N] / akk;
#pragma unroll
                for (int j = k + 1; j < N; ++j)
#pragma unroll
                    for (int i = k + 1; i < N; ++i)
                        a[i + j * N] = Arith<F>::msub(a[i + k * N], a[k + j * N], a[i + j * N]);
            }
        }
    }

    // lu.jl:67-92.
    __device__ __forceinline__ void backsolve(TF (&x)[N]) const {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            int p = ipiv[k];
            if (p != k) {
#pragma unroll
                for (int i = k + 1; i < N; ++i) cswap(i, p, x[k], x[i]);
            }
        }
#pragma unroll
        for (int k = 0; k < N; ++k) {
            TF xk = x[k];
#pragma unroll
            for (int i = k + 1; i < N; ++i) x[i] = Arith<F>::msub(a[i + k * N], xk, x[i]);
        }
#pragma unroll
        for (int k = N - 1; k >= 0; --k) {
            TF xk = kRecip ? x[k] * a[k + k * N] : x[k] / a[k + k * N];
            x[k] = xk;
#pragma unroll
            for (int i = 0; i < k; ++i) x[i] = Arith<F>::msub(a[i + k * N], xk, x[i]);
        }
    }

    // ldiv!!: same type (factors.jl:931-936) or mixed type (factors.jl:943-949).
    __device__ __forceinline__ void ldiv(const double (&r)[N], double (&d)[N]) const {
        if constexpr (sizeof(TF) == sizeof(double)) {
            if (e == 0 && rhs_unscaled<N>(r)) {
                // rhs_exponent is 0 and so is e: no scaling on either side of the solve
                TF x[N];
#pragma unroll
                for (int i = 0; i < N; ++i) x[i] = r[i];
                backsolve(x);
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = x[i];
                return;
            }
            int k = rhs_exponent<N>(r, e);
            TF x[N];
#pragma unroll
            for (int i = 0; i < N; ++i) x[i] = k == 0 ? r[i] : scale2_in(r[i], -k);  // -k in [-6, 1023]
            backsolve(x);
            int e2 = k - e;
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = e2 == 0 ? double(x[i]) : scale2_in(double(x[i]), e2);  // e2 = k - e in [0, 1029]
        } else {
            double s = fabs(r[0]);
#pragma unroll
            for (int i = 1; i < N; ++i) s = jmax(s, fabs(r[i]));
            if (s == 0.0) {
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = 0.0;
                return;
            }
            TF x[N];
#pragma unroll
            for (int i = 0; i < N; ++i) x[i] = TF(kRecip ? __dmul_rn(r[i], __drcp_rn(s)) : __ddiv_rn(r[i], s));
            backsolve(x);
            int ex = 0;
            double frac = isfin(s) ? frexp(s, &ex) : s;
            if (!isfin(s)) ex = 0;
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = __dmul_rn(double(x[i]), frac);
            const int E = ex - e;
            if (E >= -1074 && E <= 2046) {
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = scale2_in(d[i], E);
            } else {
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = ldexp2_slow(d[i], E);
            }
        }
    }
};

// The static Householder QR of a square J without column pivoting (src/linear/static/qr.jl:
// 9-60), one thread, the factor in registers: step k reflects the scaled subcolumn onto
// -phase * sigma e_1 with tau_k = (sigma + |x_1|) / sigma in [1, 2] and the reflector's vector
// w = v / v_1 stored below the diagonal; R on and above it. The same interface as LUFactor's
// Float64 factor (load / eliminate / ldiv), so the plain step takes either. Divisions stay
// divisions under both arithmetics; GSB_FUSED only contracts the products and sums.
template <bool F, int N, class TF = double> struct QRFactor {
    using A_ = Arith<F>;
    static constexpr bool same = sizeof(TF) == sizeof(double);
    // under the fused arithmetic the mixed ldiv scales by a reciprocal (see LUFactor)
    static constexpr bool kRecip = F;
    TF a[N * N];
    TF tau[N];
    int info;
    int e;

    __device__ __forceinline__ static TF dv(TF x, TF y) {
        if constexpr (same) return __ddiv_rn(x, y);
        else return __fdiv_rn(x, y);
    }

    template <class Fam, class JS, int M>
    __device__ __forceinline__ void load(const Fam& fam, const JS& js, const double (&Fx)[M],
                                         double& s, double (&g)[N]) {
        static_assert(M == N && same, "the square Float64 factor");
        for_each_J(fam, js, [&](int i, int k, double v) {
            a[i + k * N] = v;
            s = (i == 0 && k == 0) ? A_::mul(v, v) : A_::madd(v, v, s);
            g[k] = i == 0 ? A_::mul(v, Fx[0]) : A_::madd(v, Fx[i], g[k]);
        });
    }

    // J into the factor, factor_matrix's scaling (J / 2^e, rounded to TF), the reflections
    template <class Fam, class JS> __device__ __forceinline__ void factor(const Fam& fam, const JS& js) {
        if constexpr (same) {
            for_each_J(fam, js, [&](int i, int k, double v) { a[i + k * N] = v; });
            eliminate();
        } else {
            unsigned long long mb = 0;
            for_each_J(fam, js, [&](int, int, double v) {
                const unsigned long long b = FBits<double>::bits(v) & ~FBits<double>::sign_mask;
                mb = b > mb ? b : mb;
            });
            const double mm = FBits<double>::from(mb);
            e = (isfin(mm) && mm != 0.0) ? max(-1023, min(1023, jexponent(mm))) : 0;
            for_each_J(fam, js, [&](int i, int k, double v) {
                a[i + k * N] = TF(e == 0 ? v : scale2_in(v, -e));  // -e in [-1023, 1023]
            });
            reflect();
        }
    }

    // factor_matrix's scaling (J / 2^e) of a Float64 factor, then the reflections.
    __device__ __forceinline__ void eliminate() {
        static_assert(same, "the Float64 factor");
        e = matrix_exponent<N * N>(a);
        if (e < 0) {
#pragma unroll
            for (int q = 0; q < N * N; ++q) a[q] = scale2_in(a[q], -e);  // -e in [1, 1023]
        } else {
            e = 0;
        }
        reflect();
    }

    // qr.jl:17-58: step k reflects the subcolumn, its norm taken as LAPACK's nrm2 takes it
    // (divided by its largest |a|), in TF.
    __device__ __forceinline__ void reflect() {
        info = 0;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            tau[k] = TF(0);
            TF amax = TF(0);
#pragma unroll
            for (int i = k; i < N; ++i) amax = jmax(amax, TF(fabs(a[i + k * N])));
            TF x[N];
#pragma unroll
            for (int i = 0; i < N; ++i)
                x[i] = (i >= k && amax != TF(0)) ? dv(a[i + k * N], amax) : TF(0);
            const TF sigma = A_::mul(amax, rnorm<F, N>(x));
            if (sigma != TF(0)) {
                const TF x1 = a[k + k * N];
                const TF ax1 = TF(fabs(x1));
                const TF phase = x1 == TF(0) ? TF(1) : dv(x1, ax1);
                const TF sa = A_::add(sigma, ax1);
                const TF v1 = A_::mul(phase, sa);
                const TF tk = dv(sa, sigma);
                tau[k] = tk;
#pragma unroll
                for (int i = k + 1; i < N; ++i) a[i + k * N] = dv(a[i + k * N], v1);
#pragma unroll
                for (int j = k + 1; j < N; ++j) {
                    TF t = a[k + j * N];
#pragma unroll
                    for (int i = k + 1; i < N; ++i) t = A_::madd(a[i + k * N], a[i + j * N], t);
                    t = A_::mul(t, tk);
                    a[k + j * N] = A_::sub(a[k + j * N], t);
#pragma unroll
                    for (int i = k + 1; i < N; ++i) a[i + j * N] = A_::msub(a[i + k * N], t, a[i + j * N]);
                }
                a[k + k * N] = A_::mul(-phase, sigma);
            }
            if (a[k + k * N] == TF(0) && info == 0) info = k + 1;
        }
    }

    // qr.jl:63-89: Q' r by the reflectors, then R x = Q' r.
    __device__ __forceinline__ void backsolve(TF (&x)[N]) const {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            TF t = x[k];
#pragma unroll
            for (int i = k + 1; i < N; ++i) t = A_::madd(a[i + k * N], x[i], t);
            t = A_::mul(t, tau[k]);
            x[k] = A_::sub(x[k], t);
#pragma unroll
            for (int i = k + 1; i < N; ++i) x[i] = A_::msub(a[i + k * N], t, x[i]);
        }
#pragma unroll
        for (int k = N - 1; k >= 0; --k) {
            const TF xk = dv(x[k], a[k + k * N]);
            x[k] = xk;
#pragma unroll
            for (int i = 0; i < k; ++i) x[i] = A_::msub(a[i + k * N], xk, x[i]);
        }
    }

    // ldiv!!: same type (factors.jl:931-936), as LUFactor's Float64 branch, or mixed type
    // (factors.jl:943-949), as its Float32 branch.
    __device__ __forceinline__ void ldiv(const double (&r)[N], double (&d)[N]) const {
        if constexpr (same) {
            int k = rhs_exponent<N>(r, e);
            double x[N];
#pragma unroll
            for (int i = 0; i < N; ++i) x[i] = k == 0 ? r[i] : scale2_in(r[i], -k);  // -k in [-6, 1023]
            backsolve(x);
            int e2 = k - e;
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = e2 == 0 ? x[i] : scale2_in(x[i], e2);  // e2 in [0, 1029]
        } else {
            double s = fabs(r[0]);
#pragma unroll
            for (int i = 1; i < N; ++i) s = jmax(s, fabs(r[i]));
            if (s == 0.0) {
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = 0.0;
                return;
            }
            TF x[N];
#pragma unroll
            for (int i = 0; i < N; ++i) x[i] = TF(kRecip ? __dmul_rn(r[i], __drcp_rn(s)) : __ddiv_rn(r[i], s));
            backsolve(x);
            int ex = 0;
            double frac = isfin(s) ? frexp(s, &ex) : s;
            if (!isfin(s)) ex = 0;
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = __dmul_rn(double(x[i]), frac);
            const int E = ex - e;
            if (E >= -1074 && E <= 2046) {
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = scale2_in(d[i], E);
            } else {
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = ldexp2_slow(d[i], E);
            }
        }
    }
};

// The Float64 LU of the plain step in registers, for the common case in which it needs neither
// a row exchange nor factor_matrix's scaling: every pivot is the diagonal (each a_kk's magnitude
// key above those of the entries below it, as LUFactor's search decides) and |J_00| >= 1 (so
// e = 0). factor() returns false as soon as either fails; the caller then factors with LocalLU,
// whose operations are LUFactor's, so the results are the same bits either way. Without the
// exchange and scaling code the elimination is one straight run of arithmetic, and the
// back substitution takes no permutation.
template <bool F, int N> struct DiagLU {
    double a[N * N];

    template <class Fam, class JS>
    __device__ __forceinline__ bool factor(const Fam& fam, const JS& js) {
        for_each_J(fam, js, [&](int i, int k, double v) { a[i + k * N] = v; });
        if (!(fabs(a[0]) >= 1.0)) return false;  // factor_matrix might scale
#pragma unroll
        for (int k = 0; k < N; ++k) {
            if (k + 1 < N) {
                unsigned below = 0;
#pragma unroll
                for (int i = k + 1; i < N; ++i) below = max(below, mag_key(a[i + k * N]));
                if (!(below < mag_key(a[k + k * N]))) return false;  // a row exchange might be due
            } else if (a[k + k * N] == 0.0) {
                return false;  // singular: LocalLU reports it
            }
            if constexpr (F) {
                const double r = crcp(a[k + k * N]);
                a[k + k * N] = r;
#pragma unroll
                for (int i = k + 1; i < N; ++i) a[i + k * N] = a[i + k * N] * r;
            } else {
                const double akk = a[k + k * N];
#pragma unroll
                for (int i = k + 1; i < N; ++i) a[i + k * N] = a[i + k * N] / akk;
            }
#pragma unroll
            for (int j = k + 1; j < N; ++j)
#pragma unroll
                for (int i = k + 1; i < N; ++i)
                    a[i + j * N] = Arith<F>::msub(a[i + k * N], a[k + j * N], a[i + j * N]);
        }
        return true;
    }

    __device__ __forceinline__ void backsolve(double (&x)[N]) const {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const double xk = x[k];
#pragma unroll
            for (int i = k + 1; i < N; ++i) x[i] = Arith<F>::msub(a[i + k * N], xk, x[i]);
        }
#pragma unroll
        for (int k = N - 1; k >= 0; --k) {
            const double xk = F ? x[k] * a[k + k * N] : x[k] / a[k + k * N];
            x[k] = xk;
#pragma unroll
            for (int i = 0; i < k; ++i) x[i] = Arith<F>::msub(a[i + k * N], xk, x[i]);
        }
    }

    // ldiv!! with e = 0 (factors.jl:931-936)
    __device__ __forceinline__ void ldiv(const double (&r)[N], double (&d)[N]) const {
        double x[N];
        if (rhs_unscaled<N>(r)) {
#pragma unroll
            for (int i = 0; i < N; ++i) x[i] = r[i];
            backsolve(x);
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = x[i];
            return;
        }
        const int k = rhs_exponent<N>(r, 0);
#pragma unroll
        for (int i = 0; i < N; ++i) x[i] = k == 0 ? r[i] : scale2_in(r[i], -k);  // -k in [-6, 1023]
        backsolve(x);
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = k == 0 ? x[i] : scale2_in(x[i], k);
    }
};

// The Float64 factorisation of the mixed step's rare branches (a promoted system, or the
// promotion of a failed Float32 step), with its matrix in thread-local memory instead of
// registers: the same operations in the same order as LUFactor<F, N, double> (lu.jl:24-64,
// factors.jl:802-811, 931-936), so its results are identical, while the mixed kernel's register
// budget is set by the Float32 factor it runs at every step. The loops keep runtime indices so
// that the matrix stays in memory (L1-cached) rather than in registers.
template <bool F, int N> struct LocalLU {
    double a[N * N];
    int ipiv[N];
    int info;
    int e;

    template <class Fam, class JS>
    __device__ __noinline__ void factor(const Fam& fam, const JS& js) {
#pragma unroll
        for (int k = 0; k < N; ++k)
#pragma unroll
            for (int i = 0; i < N; ++i) a[i + k * N] = fam.J(js, i, k);
        e = matrix_exponent<N * N>(a);
        if (e < 0) {
#pragma unroll 1
            for (int q = 0; q < N * N; ++q) a[q] = scale2_in(a[q], -e);  // -e in [1, 1023]
        } else {
            e = 0;
        }
        info = 0;
#pragma unroll 1
        for (int k = 0; k < N; ++k) {
            int p = k;
            double amax = fabs(a[k + k * N]);
#pragma unroll 1
            for (int i = k + 1; i < N; ++i) {
                double v = fabs(a[i + k * N]);
                if (v > amax) {
                    amax = v;
                    p = i;
                }
            }
            ipiv[k] = p;
            if (p != k) {
#pragma unroll 1
                for (int j = 0; j < N; ++j) {
                    double t = a[k + j * N];
                    a[k + j * N] = a[p + j * N];
                    a[p + j * N] = t;
                }
            }
            double akk = a[k + k * N];
            if (akk == 0.0) {
                if (info == 0) info = k + 1;
            } else if constexpr (F) {
                const double r = 1.0 / akk;
                a[k + k * N] = r;
#pragma unroll 1
                for (int i = k + 1; i < N; ++i) a[i + k * N] = a[i + k * N] * r;
#pragma unroll 1
                for (int j = k + 1; j < N; ++j)
#pragma unroll 1
                    for (int i = k + 1; i < N; ++i)
                        a[i + j * N] = Arith<F>::msub(a[i + k * N], a[k + j * N], a[i + j * N]);
            } else {
#pragma unroll 1
                for (int i = k + 1; i < N; ++i) a[i + k * N] = a[i + k * N] / akk;
#pragma unroll 1
                for (int j = k + 1; j < N; ++j)
#pragma unroll 1
                    for (int i = k + 1; i < N; ++i)
                        a[i + j * N] = Arith<F>::msub(a[i + k * N], a[k + j * N], a[i + j * N]);
            }
        }
    }

    __device__ __noinline__ void backsolve(double* x) const {
#pragma unroll 1
        for (int k = 0; k < N; ++k) {
            int p = ipiv[k];
            if (p != k) {
                double t = x[k];
                x[k] = x[p];
                x[p] = t;
            }
        }
#pragma unroll 1
        for (int k = 0; k < N; ++k) {
            double xk = x[k];
#pragma unroll 1
            for (int i = k + 1; i < N; ++i) x[i] = Arith<F>::msub(a[i + k * N], xk, x[i]);
        }
#pragma unroll 1
        for (int k = N - 1; k >= 0; --k) {
            double xk = F ? x[k] * a[k + k * N] : x[k] / a[k + k * N];
            x[k] = xk;
#pragma unroll 1
            for (int i = 0; i < k; ++i) x[i] = Arith<F>::msub(a[i + k * N], xk, x[i]);
        }
    }

    __device__ __forceinline__ void ldiv(const double (&r)[N], double (&d)[N]) const {
        int k = rhs_exponent<N>(r, e);
        double x[N];
#pragma unroll
        for (int i = 0; i < N; ++i) x[i] = k == 0 ? r[i] : scale2_in(r[i], -k);  // -k in [-6, 1023]
        backsolve(x);
        int e2 = k - e;
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = e2 == 0 ? x[i] : scale2_in(x[i], e2);  // e2 in [0, 1029]
    }
};

// PlainRef: the plain (TF = T) step refines its direction (Refinement with a Float64 factor), a
// rare configuration kept in its own instantiation so the common plain step holds no refinement
// state in registers.
// Qr selects the static Householder QR for the step's factors (QRFactorization: the plain step's
// Float64 factor, the mixed step's Float32 factor and its Float64 fallback), else the pivoted LU.
template <class Fam, bool F, bool Mixed, bool PlainRef = false, bool Qr = false,
          int Kind = kStepNewton>
struct Solver {
    static constexpr int N = Fam::N, M = Fam::M;
    using JS = typename Fam::JState;
    using A = Arith<F>;
    // The plain step's gradient ratio feeds only the status of a square system, which keeps the
    // last factorisation's; where the step parks its start iterate and residual (N >= 6, the
    // kernel's stash), the ratio is formed once, after the last step, instead of at every step.
    static constexpr bool kDeferGr = (N >= 6) && !Fam::lsq && !Mixed && Kind == kStepNewton;
    const Fam& fam;
    const GsbMethod& m;
    const GsbOptions& o;
    double* stash;  // this thread's 2N doubles of shared memory (required from N = 6), or nullptr

    __device__ Solver(const Fam& f, const GsbMethod& mm, const GsbOptions& oo, double* st)
        : fam(f), m(mm), o(oo), stash(st) {}

    // While a factor holds the registers, the iterate and the residual wait in shared memory:
    // a volatile store and a volatile load, so that their register copies are free meanwhile.
    // With aligned rows (PairsOf) the stash is 16-byte aligned and moves two entries at a time.
    template <int L> __device__ __forceinline__ void put(unsigned a, const double (&v)[L]) const {
        if constexpr (PairsOf<Fam>::value && L % 2 == 0) {
#pragma unroll
            for (int i = 0; i < L; i += 2) sts2(a + 8u * i, v[i], v[i + 1]);
        } else {
#pragma unroll
            for (int i = 0; i < L; ++i) sts(a + 8u * i, v[i]);
        }
    }
    template <int L> __device__ __forceinline__ void get(unsigned a, double (&v)[L]) const {
        if constexpr (PairsOf<Fam>::value && L % 2 == 0) {
#pragma unroll
            for (int i = 0; i < L; i += 2) lds2(a + 8u * i, v[i], v[i + 1]);
        } else {
#pragma unroll
            for (int i = 0; i < L; ++i) v[i] = lds(a + 8u * i);
        }
    }
    __device__ __forceinline__ void park(double (&x)[N], double (&Fx)[M]) const {
        if (stash == nullptr) return;
        put<N>(smem_addr(stash), x);
        put<M>(smem_addr(stash) + 8u * N, Fx);
    }
    __device__ __forceinline__ void park_x(const double (&x)[N]) const {
        if (stash == nullptr) return;
        put<N>(smem_addr(stash), x);
    }
    __device__ __forceinline__ void park_F(const double (&Fx)[M]) const {
        if (stash == nullptr) return;
        put<M>(smem_addr(stash) + 8u * N, Fx);
    }
    __device__ __forceinline__ void unpark_x(double (&x)[N]) const {
        if (stash == nullptr) return;
        get<N>(smem_addr(stash), x);
    }
    __device__ __forceinline__ void unpark_F(double (&Fx)[M]) const {
        if (stash == nullptr) return;
        get<M>(smem_addr(stash) + 8u * N, Fx);
    }

    __device__ __forceinline__ bool has_merit() const { return m.globalization == GSB_BACKTRACKING; }

    // J v as a left fold over the columns (the SMatrix product of the held Jacobian).
    __device__ __forceinline__ void jmul(const JS& js, const double (&v)[N], double (&out)[M]) const {
        if constexpr (PairsOf<Fam>::value) {
#pragma unroll
            for (int i = 0; i < M; i += 2) {
                double j0, j1;
                fam.J2(js, i, 0, j0, j1);
                double s0 = A::mul(j0, v[0]), s1 = A::mul(j1, v[0]);
#pragma unroll
                for (int k = 1; k < N; ++k) {
                    fam.J2(js, i, k, j0, j1);
                    s0 = A::madd(j0, v[k], s0);
                    s1 = A::madd(j1, v[k], s1);
                }
                out[i] = s0;
                out[i + 1] = s1;
            }
            return;
        }
#pragma unroll
        for (int i = 0; i < M; ++i) {
            double s = A::mul(fam.J(js, i, 0), v[0]);
#pragma unroll
            for (int k = 1; k < N; ++k) s = A::madd(fam.J(js, i, k), v[k], s);
            out[i] = s;
        }
    }

    // grad_ratio_and_norm, src/nonlinear/newton.jl:1287-1298.
    __device__ void grad_ratio_and_norm(const JS& js, const double (&Fx)[M], double fnorm,
                                        double& gr, double& jnorm) const {
        double s = 0.0;
        for_each_J(fam, js, [&](int i, int k, double v) {
            s = (i == 0 && k == 0) ? A::mul(v, v) : A::madd(v, v, s);
        });
        const double tiny = double(M * N) * kFloatmin;
        if (isfin(s) && s >= tiny) {
            jnorm = sqrt(s);
        } else {
            // scaled fallback of rnorm over the M*N entries
            double mx = 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k)
#pragma unroll
                for (int i = 0; i < M; ++i) mx = jmax(mx, jmax(fabs(fam.J(js, i, k)), 0.0));
            if (mx == 0.0 || !isfin(mx)) {
                jnorm = mx;
            } else {
                int e = jexponent(mx);
                double acc = 0.0;
                bool first = true;
#pragma unroll
                for (int k = 0; k < N; ++k)
#pragma unroll
                    for (int i = 0; i < M; ++i) {
                        double u = scale2_in(fam.J(js, i, k), -e);
                        acc = first ? A::mul(u, u) : A::madd(u, u, acc);
                        first = false;
                    }
                jnorm = scale2_in(sqrt(acc), e);
            }
        }
        if (jnorm == 0.0 || fnorm == 0.0) {
            gr = 0.0;
            return;
        }
        double g[N];
        for_each_J(fam, js, [&](int i, int j, double v) {
            g[j] = i == 0 ? A::mul(v, Fx[0]) : A::madd(v, Fx[i], g[j]);
        });
        double gnorm = rnorm<F, N>(g);
        if (isfin(gnorm) || !(isfin(jnorm) && isfin(fnorm))) {
            gr = __ddiv_rn(__ddiv_rn(gnorm, jnorm), fnorm);
            return;
        }
        int e = jexponent(fnorm);
        double sc = ldexp(1.0, -e);
#pragma unroll
        for (int j = 0; j < N; ++j) {
            double t = A::mul(fam.J(js, 0, j), __dmul_rn(Fx[0], sc));
#pragma unroll
            for (int i = 1; i < M; ++i) t = A::madd(fam.J(js, i, j), __dmul_rn(Fx[i], sc), t);
            g[j] = t;
        }
        gr = __ddiv_rn(__ddiv_rn(rnorm<F, N>(g), jnorm), ldexp(fnorm, -e));
    }

    // grad_ratio_and_norm's common branch from the two sums that the factor's load folds (s,
    // the squares of J's entries in column order; g = J' Fx), with both sums in the range where
    // their norms are plain square roots. False (nothing written) when either is not: the
    // function above then runs in full, with the same operations, after the solve.
    __device__ __forceinline__ bool grad_ratio_fast(double s, const double (&g)[N], double fnorm,
                                                    double& gr, double& jnorm) const {
        if (!(isfin(s) && s >= double(M * N) * kFloatmin)) return false;
        const double gs = norm2<F, N>(g);
        if (!(isfin(gs) && gs >= double(N) * kFloatmin)) return false;
        jnorm = sqrt(s);
        gr = fnorm == 0.0 ? 0.0 : __ddiv_rn(__ddiv_rn(sqrt(gs), jnorm), fnorm);
        return true;
    }

    // residual_norm, src/nonlinear/newton.jl:1274-1278.
    __device__ __forceinline__ double residual_norm(const DevState& st, const double (&Fx)[M]) const {
        if (has_merit()) {
            if (isfin(st.merit) && st.merit >= double(M) * kFloatmin) return sqrt(st.merit);
            return rnorm<F, M>(Fx);
        }
        return isnan(st.fnorm) ? rnorm<F, M>(Fx) : st.fnorm;
    }

    // The merit of the trial x + a d: the trial iterate, its residual and norm2. The Float32
    // trial form (kStepTrial32) forms the increment a d in Float32 and adds it to the Float64
    // iterate; the residual, its norm and every test on them stay Float64.
    __device__ __forceinline__ double trial(const double (&x)[N], const double (&d)[N], double a,
                                            double (&xt)[N], double (&Ft)[M]) const {
        if constexpr (Kind == kStepTrial32) {
            const float af = __double2float_rn(a);
#pragma unroll
            for (int i = 0; i < N; ++i)
                xt[i] = __dadd_rn(x[i], (double)__fmul_rn(af, __double2float_rn(d[i])));
        } else {
#pragma unroll
            for (int i = 0; i < N; ++i) xt[i] = A::madd(a, d[i], x[i]);
        }
        fam.F(xt, Ft);
        return norm2<F, M>(Ft);
    }

    // The Float32 trial form's measured slope: 2 <F(x), J(x) d> from the residual the step
    // already holds (the reference evaluates F again at x + 0 d, the same point for a finite
    // d) and the JVP, folded in Float32.
    __device__ __forceinline__ double slope0_held(const double (&x)[N], const double (&Fx)[M],
                                                  const double (&d)[N]) const {
        double Jv[M];
        fam.jvp(x, d, Jv);
        float s = __fmul_rn(__double2float_rn(Fx[0]), __double2float_rn(Jv[0]));
#pragma unroll
        for (int i = 1; i < M; ++i)
            s = __fmaf_rn(__double2float_rn(Fx[i]), __double2float_rn(Jv[i]), s);
        return 2.0 * (double)s;
    }

    // φ′(0) = 2 <F(x), J(x) d> (src/globalization/linefunction.jl:47-52).
    __device__ __forceinline__ double slope0(const double (&x)[N], const double (&d)[N]) const {
        double x0[N], F0[M], Jv[M];
#pragma unroll
        for (int i = 0; i < N; ++i) x0[i] = A::madd(0.0, d[i], x[i]);
        fam.F(x0, F0);
        fam.jvp(x0, d, Jv);
        double s = A::mul(F0[0], Jv[0]);
#pragma unroll
        for (int i = 1; i < M; ++i) s = A::madd(F0[i], Jv[i], s);
        return 2.0 * s;
    }

    // Backtracking's common course, taken without a branch on the way: its first trial at
    // alpha = 1 with the exact slope (the plain step's ExactStep, phi'(0) = -2 phi0), the trial's
    // merit, |d| and, for the stopping tests after the step, the norm of the trial iterate, the
    // rate against the previous step and the rate test's quotient, all formed side by side; then
    // the conditions under which globalize (below) takes that trial as a SUCCESS at alpha = 1,
    // tested together. True: the step is done (x, Fx, merit, info and sp are the bits globalize
    // and the loop's own tests would give). False: nothing is written, and globalize runs.
    __device__ __forceinline__ bool first_trial_accepted(double (&x)[N], double (&Fx)[M],
                                                         const double (&d)[N], double& merit,
                                                         StepInfo& info, double prev_stepnorm,
                                                         double rate_k, StepSpec& sp) const {
        const double phi0 = merit;
        double xt[N], Ft[M];
        const double pa = trial(x, d, 1.0, xt, Ft);
        const double dn2 = norm2<F, N>(d);
        const double xn2 = norm2<F, N>(xt);
        const double dn = sqrt(dn2);
        const double rate = prev_stepnorm > 0.0 ? __ddiv_rn(dn, prev_stepnorm) : kNaN;
        const double th = jmax(rate, rate_k);
        const double q = __ddiv_rn(th, __dsub_rn(1.0, th));
        const double d0 = -2.0 * phi0;
        const double tau = jmax(__dmul_rn(4.0 * kEps, fabs(phi0)), 4.0 * 4.9406564584124654e-324);
        const double demand = __dmul_rn(m.bt_c1, d0);  // (c1 * alpha) * d0 at alpha = 1
        const double dphi = __dsub_rn(pa, phi0);
        const bool ok = isfin(dn2) && dn2 >= double(N) * kFloatmin  // rnorm(d) is sqrt(dn2)
                        && isfin(phi0) && isfin(d0) && d0 < 0.0     // the search starts
                        && !(tau > fabs(d0))                         // at alpha = 1
                        && dphi <= jmin(0.0, __dadd_rn(demand, tau)) // Armijo holds
                        && isfin(pa) && dphi < -tau;                 // and it is a SUCCESS
        if (!ok) return false;
#pragma unroll
        for (int i = 0; i < N; ++i) x[i] = xt[i];
#pragma unroll
        for (int i = 0; i < M; ++i) Fx[i] = Ft[i];
        merit = pa;
        info = {SUCCESS, sqrt(pa), dn, 0, false, false, false};
        const bool xr = isfin(xn2) && xn2 >= double(N) * kFloatmin;
        sp = {true, rate, xr ? sqrt(xn2) : rnorm<F, N>(xt), q};
        return true;
    }

    // globalize!! for Static (src/globalization/linefunction.jl:114-131) and globalize_merit!!
    // with the Backtracking search (linefunction.jl:159-199, linesearch.jl:154-171,
    // backtracking.jl:62-132).
    __device__ void globalize(double (&x)[N], double (&Fx)[M], const double (&d)[N], bool exact,
                              double& merit, StepInfo& info) const {
        if (m.globalization == GSB_STATIC) {
            double s = m.static_alpha;
            double dn = rnorm<F, N>(d);
            double stepnorm = __dmul_rn(fabs(s), dn);
            if (!isfin(stepnorm)) {
                info = {NONFINITE, rnorm<F, M>(Fx), stepnorm, 0, false, false, false};
                return;
            }
            double xp[N], Fp[M];
            double fn = rnorm_from<F, M>(Fp, trial(x, d, s, xp, Fp));
            if (!isfin(fn)) {
                info = {NONFINITE, rnorm<F, M>(Fx), stepnorm, 0, false, false, false};
                return;
            }
#pragma unroll
            for (int i = 0; i < N; ++i) x[i] = xp[i];
#pragma unroll
            for (int i = 0; i < M; ++i) Fx[i] = Fp[i];
            info = {SUCCESS, fn, stepnorm, 0, false, false, false};
            return;
        }
        const double phi0 = merit;
        double dn = rnorm<F, N>(d);
        if (!isfin(dn)) {
            info = {NONFINITE, rnorm<F, M>(Fx), dn, 0, false, false, false};
            return;
        }
        // linesearch entry: trial step 1, the anchor slope, τ and the step floor
        double alpha = 1.0;
        double d0;
        if constexpr (Kind == kStepTrial32) d0 = exact ? -2.0 * phi0 : slope0_held(x, Fx, d);
        else d0 = exact ? -2.0 * phi0 : slope0(x, d);
        int code;
        double aa = alpha, pa = kNaN;
        double xt[N], Ft[M];
        if (!(isfin(phi0) && isfin(d0) && d0 < 0.0)) {
            code = (isfin(phi0) && isfin(d0)) ? (d0 > 0.0 ? LINESEARCH_FAILED : STALLED) : NONFINITE;
        } else {
            double tau = jmax(__dmul_rn(4.0 * kEps, fabs(phi0)), 4.0 * 4.9406564584124654e-324);
            // The step floor amin = max(tau / |d0|, floatmin) is taken when first needed: an
            // accepted first trial never reads it, and the start max(1, amin) is 1 whenever
            // tau <= |d0| (then tau / |d0| <= 1 rounds to at most 1).
            double amin = kNaN;
            bool have_amin = false;
            auto floor_ = [&]() {
                if (!have_amin) {
                    amin = jmax(__ddiv_rn(tau, fabs(d0)), kFloatmin);
                    have_amin = true;
                }
                return amin;
            };
            if (tau > fabs(d0)) alpha = jmin(jmax(alpha, floor_()), kInf);
            double ap = kNaN, pp = kNaN;
            int frozen = 0, trips = 0;
            code = LINESEARCH_FAILED;
            bool done = false;
            const double c1 = m.bt_c1, p = m.bt_p;
            while (!done && trips < m.bt_maxiter) {
                ++trips;
                aa = alpha;
                pa = trial(x, d, alpha, xt, Ft);
                frozen = (pa == phi0 && alpha <= kSqrtEps) ? frozen + 1 : 0;
                double demand = __dmul_rn(__dmul_rn(c1, alpha), d0);
                if (__dsub_rn(pa, phi0) <= jmin(0.0, __dadd_rn(demand, tau))) {
                    // classify
                    if (isfin(pa) && __dsub_rn(pa, phi0) < -tau) code = SUCCESS;
                    else code = fabs(__dsub_rn(pa, phi0)) <= tau ? STALLED : LINESEARCH_FAILED;
                    done = true;
                } else if (frozen >= 2) {
                    code = STALLED;
                    done = true;
                } else if (alpha <= floor_()) {
                    code = fabs(__dsub_rn(pa, phi0)) <= tau ? STALLED : LINESEARCH_FAILED;
                    done = true;
                } else {
                    double an;
                    if (isfin(pa)) {
                        // backtrack_step, backtracking.jl:62-82
                        an = kNaN;
                        double s = fabs(d0);
                        double r1 = __dadd_rn(__ddiv_rn(__dsub_rn(pa, phi0), s), alpha);
                        if (!(ap > 0.0)) {
                            if (r1 > 0.0) an = __ddiv_rn(__dmul_rn(alpha, alpha), __dmul_rn(2.0, r1));
                        } else if (isfin(pp) && alpha != ap) {
                            double q1 = __ddiv_rn(r1, __dmul_rn(alpha, alpha));
                            double q2 = __ddiv_rn(__dadd_rn(__ddiv_rn(__dsub_rn(pp, phi0), s), ap),
                                                  __dmul_rn(ap, ap));
                            double da = __dsub_rn(alpha, ap);
                            double Aq = __ddiv_rn(__dsub_rn(q1, q2), da);
                            double Bq = __ddiv_rn(__dsub_rn(__dmul_rn(alpha, q2), __dmul_rn(ap, q1)), da);
                            double disc = __dadd_rn(__dmul_rn(Bq, Bq), __dmul_rn(3.0, Aq));
                            if (disc >= 0.0)
                                an = Bq > 0.0 ? __ddiv_rn(1.0, __dadd_rn(Bq, sqrt(disc)))
                                              : __ddiv_rn(__dadd_rn(-Bq, sqrt(disc)), __dmul_rn(3.0, Aq));
                        }
                        if (!(isfin(an) && an > 0.0)) an = __dmul_rn(p, alpha);
                        an = jmin(jmax(an, __dmul_rn(0.1, alpha)), __dmul_rn(p, alpha));
                    } else {
                        an = jmin(__dmul_rn(0.1, alpha), __dmul_rn(sqrt(alpha), sqrt(amin)));
                    }
                    ap = alpha;
                    pp = pa;
                    alpha = jmax(an, amin);
                }
            }
        }
        if (code == SUCCESS) {
#pragma unroll
            for (int i = 0; i < N; ++i) x[i] = xt[i];
#pragma unroll
            for (int i = 0; i < M; ++i) Fx[i] = Ft[i];
            info = {SUCCESS, sqrt(pa), __dmul_rn(aa, dn), 0, false, false, aa < 1.0};
            merit = pa;
        } else if (code == LINESEARCH_FAILED) {
            if (isfin(pa) && pa < phi0) {
#pragma unroll
                for (int i = 0; i < N; ++i) x[i] = xt[i];
#pragma unroll
                for (int i = 0; i < M; ++i) Fx[i] = Ft[i];
                info = {LINESEARCH_FAILED, sqrt(pa), __dmul_rn(aa, dn), 1, false, false, aa < 1.0};
                merit = pa;
            } else {
                info = {LINESEARCH_FAILED, rnorm<F, M>(Fx), 0.0, 1, false, false, false};
            }
        } else if (code == STALLED) {
            info = {STALLED, rnorm<F, M>(Fx), 0.0, 0, false, false, false};
        } else {
            info = {NONFINITE, rnorm<F, M>(Fx), 0.0, 0, false, false, false};
        }
    }

    // refine_passes!! with the held Jacobian, src/nonlinear/refinement.jl:211-244; returns
    // `failed`.
    template <class Fac>
    __device__ bool refine(double (&d)[N], const Fac& fac, const JS& js, const double (&Fx)[M]) const {
        const double fnorm = rnorm<F, M>(Fx);
        if (fnorm == 0.0) return false;
        if (!isfin(fnorm)) return true;
        const double thr = __dmul_rn(jmax(m.refine_eta, kSqrtEps), fnorm);
        // r = -F - J d, formed in place of the product
        double r[N];
        jmul(js, d, r);
#pragma unroll
        for (int i = 0; i < N; ++i) r[i] = __dadd_rn(-Fx[i], -r[i]);
        double rprev = rnorm<F, N>(r);
        if (!isfin(rprev)) return true;
        if (rprev <= thr) return false;
        for (int it = 1; it <= m.refine_maxiter; ++it) {
            // the candidate d + fac \ r, formed in place of the correction
            double dc[N];
            fac.ldiv(r, dc);
#pragma unroll
            for (int i = 0; i < N; ++i) dc[i] = __dadd_rn(d[i], dc[i]);
            jmul(js, dc, r);
#pragma unroll
            for (int i = 0; i < N; ++i) r[i] = __dadd_rn(-Fx[i], -r[i]);
            const double rc = rnorm<F, N>(r);
            if (!(rc < rprev)) return true;
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = dc[i];
            rprev = rc;
            if (rc <= thr) return false;
        }
        return true;
    }

    // d = -(fac \ F) refined (Refinement with the Float64 factor): the direction, then its passes.
    template <class Fac>
    __device__ __forceinline__ void refine_neg(double (&d)[N], const Fac& fac, const JS& js,
                                               const double (&Fx)[M]) const {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = -d[i];
        refine(d, fac, js, Fx);
    }

    // The plain step (TF = T), src/nonlinear/newton.jl:1679-1688.
    __device__ void step_plain(DevState& st, double (&x)[N], double (&Fx)[M], StepInfo& info,
                               double prev_stepnorm = 0.0, double rate_k = kNaN,
                               StepSpec* sp = nullptr) const {
        if constexpr (kDeferGr) {
            // the gradient ratio is formed after the last step (stashed_grad_ratio)
            JS js;
            fam.jacobian(x, js);
            double merit = st.merit;
            double d[N];
            bool singular = false;
            park(x, Fx);
            if constexpr (Qr) {
                QRFactor<F, N> fac;
                fac.factor(fam, js);
                singular = fac.info > 0;
                if (!singular) {
                    unpark_F(Fx);
                    fac.ldiv(Fx, d);
                    if constexpr (PlainRef) refine_neg(d, fac, js, Fx);
                }
            } else {
                // the register factor without exchanges or scaling, else (rarely) the factor
                // with both in thread-local memory: the same bits
                DiagLU<F, N> fac;
                if (fac.factor(fam, js)) {
                    unpark_F(Fx);
                    fac.ldiv(Fx, d);
                    if constexpr (PlainRef) refine_neg(d, fac, js, Fx);
                } else {
                    LocalLU<F, N> lf;
                    lf.factor(fam, js);
                    singular = lf.info > 0;
                    if (!singular) {
                        unpark_F(Fx);
                        lf.ldiv(Fx, d);
                        if constexpr (PlainRef) refine_neg(d, lf, js, Fx);
                    }
                }
            }
            if (singular) {
                unpark_x(x);
                unpark_F(Fx);
                info = {SINGULAR, rnorm<F, M>(Fx), 0.0, 0, false, false, false};
            } else {
                if constexpr (!PlainRef) {
#pragma unroll
                    for (int i = 0; i < N; ++i) d[i] = -d[i];
                }
                unpark_x(x);
                if constexpr (!PlainRef) {
                    if (sp != nullptr && m.globalization == GSB_BACKTRACKING &&
                        first_trial_accepted(x, Fx, d, merit, info, prev_stepnorm, rate_k, *sp)) {
                        st.merit = merit;
                        st.fnorm = info.fnorm;
                        return;
                    }
                }
                globalize(x, Fx, d, !PlainRef, merit, info);
            }
            st.merit = merit;
            st.fnorm = info.fnorm;
            return;
        }
        double fnorm = residual_norm(st, Fx);
        JS js;
        fam.jacobian(x, js);
        double gr, jn;
        double merit = st.merit;
        constexpr bool ref = PlainRef;
        {
            typename std::conditional<Qr, QRFactor<F, N>, LUFactor<F, N, double>>::type fac;
            park_x(x);
            // grad_ratio_and_norm from the sums that the factor's load folds; its scaled
            // branches, for sums out of range, run in full once the factor is done with
            bool gr_done;
            {
                double s, g[N];
                fac.load(fam, js, Fx, s, g);
                gr_done = grad_ratio_fast(s, g, fnorm, gr, jn);
            }
            park_F(Fx);
            fac.eliminate();
            if (fac.info > 0) {
                unpark_x(x);
                unpark_F(Fx);
                if (!gr_done) grad_ratio_and_norm(js, Fx, fnorm, gr, jn);
                info = {SINGULAR, rnorm<F, M>(Fx), 0.0, 0, false, false, false};
            } else {
                double d[N];
                unpark_F(Fx);
                fac.ldiv(Fx, d);
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = -d[i];
                if constexpr (ref) refine(d, fac, js, Fx);
                if (!gr_done) grad_ratio_and_norm(js, Fx, fnorm, gr, jn);
                unpark_x(x);
                globalize(x, Fx, d, !ref, merit, info);
            }
        }
        st.gradratio = gr;
        st.jnorm = jn;
        st.merit = merit;
        st.fnorm = info.fnorm;
    }

    // The mixed-precision step (TF = Float32), src/nonlinear/newton.jl:1692-1720 with
    // mixed_newton!! :1604-1666, promote_factor!! :1332-1339, linear_residual_ratio :1422-1430
    // and read_mixed_stall :1437-1451.
    __device__ void step_mixed(DevState& st, double (&x)[N], double (&Fx)[M], StepInfo& info) const {
        double fnorm_old = residual_norm(st, Fx);
        const bool was_promoted = st.promoted;
        JS js;
        fam.jacobian(x, js);
        double gr, jn;
        grad_ratio_and_norm(js, Fx, fnorm_old, gr, jn);
        st.gradratio = gr;
        st.jnorm = jn;
        const bool ref = m.refinement == GSB_REFINEMENT;
        double d[N];
        bool ok = true;
        int failures = 0;
        double lin_rel = 0.0;
        bool md_promoted = was_promoted;
        bool fallback = was_promoted;
        park_x(x);
        if (!was_promoted) {
            typename std::conditional<Qr, QRFactor<F, N, float>, LUFactor<F, N, float>>::type fac;
            fac.factor(fam, js);
            bool ref_failed;
            if (fac.info > 0) {
                ref_failed = true;
            } else {
                fac.ldiv(Fx, d);
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = -d[i];
                ref_failed = ref ? refine(d, fac, js, Fx) : false;
            }
            if (ref_failed || fac.info > 0) {
                failures += 1;
                md_promoted = true;
                fallback = true;
            } else if (!Fam::lsq) {
                if (fnorm_old == 0.0 || !isfin(fnorm_old)) {
                    lin_rel = 0.0;
                } else {
                    double Jd[N], lin[N];
                    jmul(js, d, Jd);
#pragma unroll
                    for (int i = 0; i < N; ++i) lin[i] = __dadd_rn(Fx[i], Jd[i]);
                    lin_rel = __ddiv_rn(rnorm<F, N>(lin), fnorm_old);
                }
            }
        }
        if (fallback) {
            // the factorisation in the working precision: at every step once promoted (with the
            // refinement passes), and as the promotion of a failed Float32 step (without them)
            // the register factor for small systems; thread-local memory from n = 6 on
            using FT = typename std::conditional<
                Qr, QRFactor<F, N, double>,
                typename std::conditional<(N >= 6), LocalLU<F, N>, LUFactor<F, N, double>>::type>::type;
            FT ft;
            ft.factor(fam, js);
            if (ft.info > 0) {
                ok = false;
            } else {
                ft.ldiv(Fx, d);
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = -d[i];
                if (was_promoted && ref) refine(d, ft, js, Fx);
            }
        }
        unpark_x(x);
        if (!ok) {
            st.promoted = md_promoted;
            info = {SINGULAR, rnorm<F, M>(Fx), 0.0, failures, md_promoted, false, false};
            return;
        }
        const bool promoted_step = md_promoted && !was_promoted;
        const bool exact_step = md_promoted && !Fam::lsq;
        double merit = st.merit;
        globalize(x, Fx, d, exact_step, merit, info);
        info.failures += failures;
        if (promoted_step) {
            info.promoted = true;
            st.promoted = true;
            st.slow_steps = 0;
        } else if (!was_promoted) {
            const double eta_lin = 1e-4;
            if (info.fnorm > __dmul_rn(0.5, fnorm_old) && lin_rel > eta_lin) {
                int slow = st.slow_steps + 1;
                if (slow >= 2) {
                    st.promoted = true;
                    st.slow_steps = 0;
                    info.failures += 1;
                    info.promoted = true;
                } else {
                    st.promoted = false;
                    st.slow_steps = slow;
                }
            } else {
                st.promoted = false;
                st.slow_steps = 0;
            }
        }
        st.merit = merit;
        st.fnorm = info.fnorm;
    }

    // newton_step!! with reuse = k (Float64 factor, no refinement), src/nonlinear/newton.jl:
    // 1783-1820: while the held factor is younger than k steps and the last step did not stall,
    // the step solves with it and searches along that direction with the measured slope; a
    // search that fails without a step is taken again, in the same step, from a fresh factor at
    // the same point, which the steps after it hold (reuse_result, :1811-1820).
    __device__ void step_reuse(DevState& st, double (&x)[N], double (&Fx)[M], StepInfo& info,
                               LocalLU<F, N>& held) const {
        const int age_fresh = m.reuse == 1 ? 0 : 1;  // fresh_age, newton.jl:629
        if (!(st.age == 0 || st.stalled)) {
            const int age_next = st.age + 1 >= m.reuse ? 0 : st.age + 1;  // next_age, :632-633
            double d[N];
            held.ldiv(Fx, d);
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = -d[i];
            double xr[N], Fr[M];
#pragma unroll
            for (int i = 0; i < N; ++i) xr[i] = x[i];
#pragma unroll
            for (int i = 0; i < M; ++i) Fr[i] = Fx[i];
            double merit = st.merit;
            StepInfo ri;
            globalize(xr, Fr, d, false, merit, ri);  // newton_line with fresh = false
            if (!(ri.code == LINESEARCH_FAILED && ri.stepnorm == 0.0)) {
#pragma unroll
                for (int i = 0; i < N; ++i) x[i] = xr[i];
#pragma unroll
                for (int i = 0; i < M; ++i) Fx[i] = Fr[i];
                info = ri;
                st.merit = merit;
                st.fnorm = info.fnorm;
                st.reused = true;
                st.age = age_next;
                st.stalled = ri.code == STALLED;
                return;
            }
        }
        // a fresh factor (newton_factor, newton_globalize) at x
        const double fnorm = residual_norm(st, Fx);
        JS js;
        fam.jacobian(x, js);
        double gr, jn;
        grad_ratio_and_norm(js, Fx, fnorm, gr, jn);
        held.factor(fam, js);
        double merit = st.merit;
        if (held.info > 0) {
            info = {SINGULAR, rnorm<F, M>(Fx), 0.0, 0, false, false, false};
        } else {
            double d[N];
            held.ldiv(Fx, d);
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = -d[i];
            globalize(x, Fx, d, true, merit, info);
        }
        st.gradratio = gr;
        st.jnorm = jn;
        st.merit = merit;
        st.fnorm = info.fnorm;
        st.reused = false;
        st.age = info.code == SINGULAR ? 0 : age_fresh;
        st.stalled = info.code == STALLED;
    }

    // J' v as a left fold down each column (the product with the adjoint of the SMatrix).
    __device__ __forceinline__ void jtmul(const JS& js, const double (&v)[M], double (&out)[N]) const {
#pragma unroll
        for (int j = 0; j < N; ++j) {
            double t = A::mul(fam.J(js, 0, j), v[0]);
#pragma unroll
            for (int i = 1; i < M; ++i) t = A::madd(fam.J(js, i, j), v[i], t);
            out[j] = t;
        }
    }

    // newton_step!! with DogLeg, src/nonlinear/newton.jl:1725-1747: one Jacobian, one factor, the
    // Newton direction (none when the factor fails or its norm is zero or not finite), then the
    // trial loop of dogleg_step on the Jacobian, with the radius the state carries.
    __device__ void step_dogleg(DevState& st, double (&x)[N], double (&Fx)[M], StepInfo& info) const {
        const double fnorm = residual_norm(st, Fx);
        JS js;
        fam.jacobian(x, js);
        double gr, jn;
        grad_ratio_and_norm(js, Fx, fnorm, gr, jn);
        double d[N];
        bool newton = false;
        {
            LUFactor<F, N, double> fac;
            fac.factor(fam, js);
            if (fac.info == 0) {  // dogleg_direction, :1751-1756
                fac.ldiv(Fx, d);
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = -d[i];
                const double nd = rnorm<F, N>(d);
                newton = isfin(nd) && nd != 0.0;
            }
        }
        dogleg_step(js, x, Fx, d, newton, st.radius, info);
        st.gradratio = gr;
        st.jnorm = jn;
        st.fnorm = info.fnorm;
    }

    // dogleg_step, src/globalization/dogleg.jl:113-215 (Procedure 4.1 of Pawlowski, Simonis,
    // Walker and Shadid 2008): the Newton step inside the radius, else the Cauchy point cut to
    // it, else the point of norm delta on the segment between them; a trial is accepted when
    // pred = |F| - |F + J s| > 0 and ared = |F| - |F(x + s)| >= 1e-4 pred, with the radius
    // rules of that procedure. The Cauchy direction comes from the unit residual.
    __device__ void dogleg_step(const JS& js, double (&x)[N], double (&Fx)[M], const double (&sN)[N],
                                bool newton, double& delta, StepInfo& info) const {
        const double lo = 1e-6, hi = 1e10;
        const double fnorm = rnorm<F, M>(Fx);
        if (fnorm == 0.0) {
            info = {SUCCESS, fnorm, 0.0, 0, false, false, false};
            return;
        }
        const double nN = newton ? rnorm<F, N>(sN) : kInf;
        const double inv_f = __ddiv_rn(1.0, fnorm);
        double u[M], gh[N], Jg[M];
#pragma unroll
        for (int i = 0; i < M; ++i) u[i] = __dmul_rn(inv_f, Fx[i]);
        jtmul(js, u, gh);
        const double gnorm = rnorm<F, N>(gh);
        const double inv_g = __ddiv_rn(1.0, gnorm);
#pragma unroll
        for (int j = 0; j < N; ++j) gh[j] = __dmul_rn(inv_g, gh[j]);
        jmul(js, gh, Jg);
        const double jnorm = rnorm<F, M>(Jg);
        const bool cauchy = gnorm != 0.0 && isfin(gnorm) && jnorm != 0.0 && isfin(jnorm);
        const double nC = __dmul_rn(fnorm, __ddiv_rn(__ddiv_rn(gnorm, jnorm), jnorm));
        if (delta == 0.0 && (newton || cauchy)) {
            const double n0 = newton ? nN : nC;
            delta = n0 < lo ? 2.0 * lo : jmin(jmax(n0, lo), hi);
        }
        while (true) {
            double sv[N];
            bool boundary;
            if (newton && nN <= delta) {
#pragma unroll
                for (int j = 0; j < N; ++j) sv[j] = sN[j];
                boundary = nN >= delta;
            } else if (!cauchy) {
                info = {STALLED, fnorm, 0.0, 0, false, false, false};
                return;
            } else if (!newton || nC >= delta) {
                const double a = -jmin(nC, delta);
#pragma unroll
                for (int j = 0; j < N; ++j) sv[j] = __dmul_rn(a, gh[j]);
                boundary = nC >= delta;
            } else {
                double a[N], b[N];
                const double ca = -__ddiv_rn(nC, delta);
#pragma unroll
                for (int j = 0; j < N; ++j) a[j] = __dmul_rn(ca, gh[j]);
#pragma unroll
                for (int j = 0; j < N; ++j) b[j] = A::madd(nC, gh[j], sN[j]);
                const double inv_b = __ddiv_rn(1.0, rnorm<F, N>(b));
#pragma unroll
                for (int j = 0; j < N; ++j) b[j] = __dmul_rn(inv_b, b[j]);
                double ab = A::mul(a[0], b[0]);
#pragma unroll
                for (int j = 1; j < N; ++j) ab = A::madd(a[j], b[j], ab);
                const double c = __dsub_rn(1.0, norm2<F, N>(a));
                const double ab2 = __dmul_rn(ab, ab);
                const double t = __ddiv_rn(c, __dadd_rn(ab, __dsqrt_rn(__dadd_rn(ab2, c))));
                const double dt = __dmul_rn(delta, t);
#pragma unroll
                for (int j = 0; j < N; ++j) sv[j] = A::madd(delta, a[j], A::mul(dt, b[j]));
                boundary = true;
            }
            double Js[M], Fl[M];
            jmul(js, sv, Js);
#pragma unroll
            for (int i = 0; i < M; ++i) Fl[i] = __dadd_rn(Fx[i], Js[i]);
            const double pred = __dsub_rn(fnorm, rnorm<F, M>(Fl));
            double xp[N], Fp[M];
#pragma unroll
            for (int j = 0; j < N; ++j) xp[j] = __dadd_rn(x[j], sv[j]);
            fam.F(xp, Fp);
            const double fnp = rnorm<F, M>(Fp);
            const double ared = __dsub_rn(fnorm, fnp);
            if (pred > 0.0 && ared >= __dmul_rn(1e-4, pred)) {
                const bool limited = !(newton && nN <= delta);
                const double rho = __ddiv_rn(ared, pred);
                if (rho < 0.1)
                    delta = nN < delta ? jmax(nN, lo) : jmax(__dmul_rn(0.25, delta), lo);
                else if (rho > 0.75 && boundary)
                    delta = jmin(__dmul_rn(4.0, delta), hi);
                const double stepnorm = rnorm<F, N>(sv);
#pragma unroll
                for (int j = 0; j < N; ++j) x[j] = xp[j];
#pragma unroll
                for (int i = 0; i < M; ++i) Fx[i] = Fp[i];
                info = {SUCCESS, fnp, stepnorm, 0, false, limited, false};
                return;
            }
            if (delta == lo) {
                info = {LINESEARCH_FAILED, fnorm, 0.0, 1, false, false, false};
                return;
            }
            delta = jmax(__dmul_rn(0.25, delta), lo);
        }
    }

    __device__ __forceinline__ bool residual_converged(const DevStatus& s, double ftest,
                                                       double ftest0) const {
        if (!(s.iterations >= o.min_iterations)) return false;
        return ftest <= jmax(o.f_abstol, __dmul_rn(o.f_reltol, ftest0));
    }

    // The gradient ratio of the last step (grad_ratio_and_norm, newton.jl:1287-1298) from the
    // iterate and residual that step parked at its start: the Jacobian there, the two sums that
    // the factor's load would have folded (the squares of J's entries in column order, J' F), in
    // the same order, and the residual norm that the step read (its merit is norm2 of that
    // residual, the same fold), so the ratio has the bits the step itself would have formed.
    __device__ double stashed_grad_ratio() const {
        double xs[N], Fs[M];
        unpark_x(xs);
        unpark_F(Fs);
        double fnorm;
        if (has_merit()) {
            const double m2 = norm2<F, M>(Fs);
            fnorm = (isfin(m2) && m2 >= double(M) * kFloatmin) ? sqrt(m2) : rnorm<F, M>(Fs);
        } else {
            fnorm = rnorm<F, M>(Fs);
        }
        JS js;
        fam.jacobian(xs, js);
        double s = 0.0, g[N];
        for_each_J(fam, js, [&](int i, int k, double v) {
            s = (i == 0 && k == 0) ? A::mul(v, v) : A::madd(v, v, s);
            g[k] = i == 0 ? A::mul(v, Fs[0]) : A::madd(v, Fs[i], g[k]);
        });
        double gr, jn;
        if (!grad_ratio_fast(s, g, fnorm, gr, jn)) grad_ratio_and_norm(js, Fs, fnorm, gr, jn);
        return gr;
    }

    // solve!!, src/nonlinear/solver.jl:277-378. Returns the status; `gr` is the gradratio of
    // the last factorisation (newton_finish!!, src/nonlinear/newton.jl:1165-1184).
    __device__ DevStatus solve(double (&x)[N], double& gr_out) const {
        DevStatus s = solve_steps(x, gr_out);
        if constexpr (kDeferGr) {
            if (s.iterations > 0) gr_out = stashed_grad_ratio();
        }
        return s;
    }

    __device__ DevStatus solve_steps(double (&x)[N], double& gr_out) const {
        double Fx[M];
        fam.F(x, Fx);
        double n2 = norm2<F, M>(Fx);
        double fnorm0 = rnorm_from<F, M>(Fx, n2);
        DevState st;
        st.merit = has_merit() ? n2 : kNaN;
        st.fnorm = fnorm0;
        st.gradratio = kNaN;
        st.jnorm = 0.0;
        st.promoted = false;
        st.slow_steps = 0;
        st.age = 0;  // reset_rule: FactorAge(0, false, false), TrustRadius(radius0, radius0)
        st.stalled = false;
        st.reused = false;
        st.radius = m.dogleg_radius;
        // the factor that steps with reuse hold from one step to the next (thread-local memory)
        typename std::conditional<Kind == kStepReuse, LocalLU<F, N>, char>::type held;
        DevStatus s;
        s.code = SUCCESS;
        s.iterations = 0;
        s.fnorm = fnorm0;
        s.stepnorm = 0.0;
        s.step_failures = 0;
        s.promoted = false;
        s.stationary = false;
        s.rate = kNaN;
        s.contracted = false;
        s.reused = false;
        gr_out = kNaN;
        if (!isfin(fnorm0)) {
            s.code = NONFINITE;
            return s;
        }
        const double ftest0 = o.norm == 1 ? rmaxnorm<M>(Fx) : fnorm0;
        if (residual_converged(s, ftest0, ftest0)) return s;
        if (o.max_iterations == 0) {
            s.code = MAXITERS;
            return s;
        }
        int stalls = 0;
        while (true) {
            const double rate_k = s.rate;
            StepInfo info;
            StepSpec sp;
            sp.valid = false;
            if constexpr (Kind == kStepReuse) step_reuse(st, x, Fx, info, held);
            else if constexpr (Kind == kStepDogLeg) step_dogleg(st, x, Fx, info);
            else if (Mixed) step_mixed(st, x, Fx, info);
            else step_plain(st, x, Fx, info, s.stepnorm, rate_k, &sp);
            if (sp.valid) {
                // record(s, info) with the rate the step formed from the same operands
                s.rate = sp.rate;
                s.code = info.code;
                s.iterations += 1;
                s.fnorm = info.fnorm;
                s.stepnorm = info.stepnorm;
                s.step_failures += info.failures;
                s.promoted = s.promoted || info.promoted;
            } else {
                record(s, info);
            }
            gr_out = st.gradratio;
            if constexpr (Kind == kStepReuse) {
                // observe_rate!! (newton.jl:1205-1210): a step along a reused factor at a rate
                // >= 1 refreshes the factor at the next step (a NaN rate refreshes nothing)
                if (st.reused && s.rate >= 1.0) st.stalled = true;
                s.reused = st.reused;
            }
            if (info.code == SINGULAR || info.code == NONFINITE || info.code == MAXITERS) return s;
            if (info.code == LINESEARCH_FAILED && info.stepnorm == 0.0) return s;
            double ft = o.norm == 1 ? rmaxnorm<M>(Fx) : s.fnorm;
            if (residual_converged(s, ft, ftest0)) {
                s.code = SUCCESS;
                s.stationary = false;
                s.contracted = false;
                return s;
            }
            const bool steptested = !(info.code == STALLED || info.limited);
            const double xnorm = steptested ? (sp.valid ? sp.xnorm : rnorm<F, N>(x)) : kNaN;
            bool contracted = false;
            if (!info.shortened && o.rate_test && s.iterations >= o.min_iterations) {
                double th = jmax(s.rate, rate_k);
                if (s.stepnorm > 0.0 && th < 1.0) {
                    const double q = sp.valid ? sp.q : __ddiv_rn(th, __dsub_rn(1.0, th));
                    contracted = __dmul_rn(q, s.stepnorm) <=
                                 __dmul_rn(o.kappa, jmax(o.x_abstol, __dmul_rn(o.x_reltol, xnorm)));
                }
            }
            bool stepc = false;
            if (steptested && s.iterations >= o.min_iterations) {
                stepc = s.iterations > 0 && s.stepnorm > 0.0 &&
                        s.stepnorm <= jmax(o.x_abstol, __dmul_rn(o.x_reltol, xnorm));
                stepc = stepc || (info.code == SUCCESS && info.stepnorm == 0.0);
                stepc = stepc || (o.roundoff && s.rate >= 1.0 && rate_k < 1.0);
            }
            if (contracted || stepc) {
                s.code = contracted ? SUCCESS : STALLED;
                s.stationary = false;
                s.contracted = contracted;
                return s;
            }
            if (info.code == STALLED) {
                stalls += 1;
                if (stalls >= o.max_stalls) {
                    s.code = STALLED;
                    s.stationary = false;
                    s.contracted = false;
                    return s;
                }
            } else {
                stalls = 0;
            }
            if (s.iterations >= o.max_iterations) {
                s.code = MAXITERS;
                s.stationary = false;
                s.contracted = false;
                return s;
            }
        }
    }
};

}  // namespace gsb
