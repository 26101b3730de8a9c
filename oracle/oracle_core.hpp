// ORACLE — test infrastructure only. A CPU restatement, in plain C++17, of the R1 solve that
// GeometricSolvers.jl runs once per work item of `solve_batch!`. Only tests/, the smoke check
// and bench.py's CPU-baseline leg may load it; the product never does.
//
// Arithmetic follows Julia's semantics: every operation is rounded on its own (the build passes
// -ffp-contract=off), max/min propagate NaN, sums of static vectors are left folds. Each function
// cites the reference file:line it restates (paths within the GeometricSolvers.jl project).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace orc {

constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();
constexpr double kEps = std::numeric_limits<double>::epsilon();
constexpr double kFloatmin = std::numeric_limits<double>::min();
constexpr double kFloatmax = std::numeric_limits<double>::max();

enum Code : int { SUCCESS = 0, STALLED = 1, MAXITERS = 2, SINGULAR = 3, NONFINITE = 4,
                  LINESEARCH_FAILED = 5 };

// Julia's max/min on floats: NaN propagates, max(-0.0, 0.0) = 0.0, min(-0.0, 0.0) = -0.0.
template <class T> inline T jmax(T a, T b) {
    if (a != a) return a;
    if (b != b) return b;
    if (a == b) return std::signbit(a) ? b : a;
    return a > b ? a : b;
}
template <class T> inline T jmin(T a, T b) {
    if (a != a) return a;
    if (b != b) return b;
    if (a == b) return std::signbit(a) ? a : b;
    return a < b ? a : b;
}

template <class T> struct FBits;
template <> struct FBits<double> {
    using U = uint64_t;
    static constexpr int sig = 52, ebits = 11, raw_max = 2047, emax = 1023;
    static constexpr U sign_mask = 1ull << 63, exp_mask = 0x7ffull << 52,
                       sig_mask = (1ull << 52) - 1;
    static int clz(U x) { return __builtin_clzll(x); }
};
template <> struct FBits<float> {
    using U = uint32_t;
    static constexpr int sig = 23, ebits = 8, raw_max = 255, emax = 127;
    static constexpr U sign_mask = 1u << 31, exp_mask = 0xffu << 23, sig_mask = (1u << 23) - 1;
    static int clz(U x) { return __builtin_clz(x); }
};

template <class T> inline typename FBits<T>::U to_bits(T x) {
    typename FBits<T>::U u;
    std::memcpy(&u, &x, sizeof(T));
    return u;
}
template <class T> inline T from_bits(typename FBits<T>::U u) {
    T x;
    std::memcpy(&x, &u, sizeof(T));
    return x;
}

// `a * 2^e`, exact unless the result leaves the range, rounded to nearest-even into the
// subnormals. src/linear/factors.jl:726-758.
template <class T> inline T ldexp2(T x, long e) {
    using B = FBits<T>;
    using U = typename B::U;
    U xu = to_bits(x);
    U sign = xu & B::sign_mask;
    U xs = xu & ~B::sign_mask;
    if (xs >= B::exp_mask) return x;
    if (xs == 0) return x;
    long k = (long)(xs >> B::sig);
    if (k == 0) {
        int m = B::clz(xs) - B::ebits;
        xs <<= m;
        k = 1 - m;
    }
    U sig = (xs & B::sig_mask) | (U(1) << B::sig);
    k += e;
    if (k >= B::raw_max) return from_bits<T>(sign | B::exp_mask);
    if (k > 0) return from_bits<T>(sign | (U(k) << B::sig) | (sig & B::sig_mask));
    if (k <= -B::sig - 1) return from_bits<T>(sign);
    int shift = int(1 - k);
    U lower = sig & ((U(1) << shift) - U(1));
    U half = U(1) << (shift - 1);
    U sub = sig >> shift;
    if (lower > half || (lower == half && (sub & 1))) sub += 1;
    return from_bits<T>(sign | sub);
}

// Julia's `exponent` of a finite nonzero float: the exponent of its leading bit.
template <class T> inline int jexponent(T x) { return std::ilogb(x); }

// ─── reductions, src/base/reductions.jl ────────────────────────────────────────────────────

// norm2: sum(abs2, a) as a left fold. reductions.jl:19-22.
template <class T> inline T norm2(const T* a, int n) {
    if (n == 0) return T(0);
    T s = a[0] * a[0];
    for (int i = 1; i < n; ++i) s = s + a[i] * a[i];
    return s;
}

// rnorm with the scaled fallback below n*floatmin or on overflow. reductions.jl:348-364.
// The scaled sum accumulates in promote_type(R, Float32) = R for Float32 and Float64.
template <class T> inline T rnorm(const T* a, int n) {
    T s = norm2(a, n);
    if (std::isfinite(s) && s >= T(n) * std::numeric_limits<T>::min()) return std::sqrt(s);
    if (n == 0) return T(0);
    T m = std::fabs(a[0]);
    m = jmax(m, T(0));  // max(abs(real), abs(imag)) with imag = 0
    for (int i = 1; i < n; ++i) m = jmax(m, jmax(std::fabs(a[i]), T(0)));
    if (m == T(0) || !std::isfinite(m)) return m;
    int e = jexponent(m);
    T t = ldexp2(a[0], -e);
    T acc = t * t;
    for (int i = 1; i < n; ++i) {
        T u = ldexp2(a[i], -e);
        acc = acc + u * u;
    }
    return ldexp2(std::sqrt(acc), e);
}

// rmaxnorm: maximum(abs, a). reductions.jl:374.
template <class T> inline T rmaxnorm(const T* a, int n) {
    if (n == 0) return T(0);
    T m = std::fabs(a[0]);
    for (int i = 1; i < n; ++i) m = jmax(m, std::fabs(a[i]));
    return m;
}

// rdot: the real inner product, a left fold. reductions.jl:384-392.
template <class T> inline T rdot(const T* a, const T* b, int n) {
    if (n == 0) return T(0);
    T s = a[0] * b[0];
    for (int i = 1; i < n; ++i) s = s + a[i] * b[i];
    return s;
}

// ─── scaling, src/linear/factors.jl ─────────────────────────────────────────────────────────

template <class T> inline typename FBits<T>::U abs_bits(T x) {
    return to_bits(x) & ~FBits<T>::sign_mask;
}

// matrix_exponent: exponent of the largest |entry|, clamped, 0 for zero or non-finite.
// factors.jl:833-843.
template <class T> inline int matrix_exponent(const T* a, int len) {
    using U = typename FBits<T>::U;
    U mb = 0;
    for (int i = 0; i < len; ++i) {
        U b = abs_bits(a[i]);
        mb = b > mb ? b : mb;
    }
    T m = from_bits<T>(mb);
    if (!(std::isfinite(m) && m != T(0))) return 0;
    int e = jexponent(m);
    int emax = FBits<T>::emax;
    return e > emax ? emax : (e < -emax ? -emax : e);
}

// headroom(n) = 2 + ceil(log2 n) bits. factors.jl:890.
inline int headroom(int n) {
    unsigned long long v = (unsigned long long)(n - 1);
    int lz = v == 0 ? 64 : __builtin_clzll(v);
    return 2 + 64 - lz;
}

inline int jclamp(int x, int lo, int hi) { return x > hi ? hi : (x < lo ? lo : x); }

// rhs_exponent(r, e). factors.jl:880-885.
template <class T> inline int rhs_exponent(const T* r, int n, int e) {
    if (n == 0) return 0;
    int emax = FBits<T>::emax;
    int m = matrix_exponent(r, n);
    int a = jclamp(m, e < 0 ? e : 0, 0);
    int b = m - (emax - headroom(n));
    return a > b ? a : b;
}

// factor_matrix(F, J): J / 2^e in the factor type F, and e. factors.jl:802-811. `same` is
// F === T (the element type of J).
template <class TF> inline int factor_matrix(const double* J, int len, TF* out) {
    int e = len == 0 ? 0 : matrix_exponent(J, len);
    constexpr bool same = std::is_same<TF, double>::value;
    if (e == 0 || (same && !(e < 0))) {
        for (int i = 0; i < len; ++i) out[i] = TF(J[i]);
        return 0;
    }
    for (int i = 0; i < len; ++i) out[i] = TF(ldexp2(J[i], -e));
    return e;
}

// ─── static factors, src/linear/static/{lu,qr}.jl and src/linear/factors.jl:134-155 ──────────

template <int N, class TF> struct LUFac {
    TF A[N * N];  // column-major; U on and above the diagonal, multipliers below
    int32_t ipiv[N];
    int32_t info;
    int32_t e;
};

// Partial-pivot LU, first largest |a|, info = first zero pivot, no early exit. lu.jl:24-64.
template <int N, class TF> inline void lu_factor(const double* J, LUFac<N, TF>& f) {
    f.e = factor_matrix<TF>(J, N * N, f.A);
    TF* A = f.A;
    f.info = 0;
    for (int k = 0; k < N; ++k) {
        int p = k;
        TF amax = std::fabs(A[k + k * N]);
        for (int i = k + 1; i < N; ++i) {
            TF a = std::fabs(A[i + k * N]);
            if (a > amax) {
                amax = a;
                p = i;
            }
        }
        f.ipiv[k] = p;
        if (p != k)
            for (int j = 0; j < N; ++j) {
                TF t = A[k + j * N];
                A[k + j * N] = A[p + j * N];
                A[p + j * N] = t;
            }
        TF akk = A[k + k * N];
        if (akk == TF(0)) {
            if (f.info == 0) f.info = k + 1;
        } else {
            for (int i = k + 1; i < N; ++i) A[i + k * N] = A[i + k * N] / akk;
            for (int j = k + 1; j < N; ++j)
                for (int i = k + 1; i < N; ++i)
                    A[i + j * N] = A[i + j * N] - A[i + k * N] * A[k + j * N];
        }
    }
}

// lu.jl:67-92.
template <int N, class TF> inline void lu_backsolve(const LUFac<N, TF>& f, TF* x) {
    const TF* A = f.A;
    if constexpr (N > 1)
        for (int k = 0; k < N; ++k) {
            int p = f.ipiv[k];
            if (p != k) {
                TF t = x[k];
                x[k] = x[p];
                x[p] = t;
            }
        }
    for (int k = 0; k < N; ++k) {
        TF xk = x[k];
        for (int i = k + 1; i < N; ++i) x[i] = x[i] - A[i + k * N] * xk;
    }
    for (int k = N - 1; k >= 0; --k) {
        TF xk = x[k] / A[k + k * N];
        x[k] = xk;
        for (int i = 0; i < k; ++i) x[i] = x[i] - A[i + k * N] * xk;
    }
}

template <int N, class TF> struct QRFac {
    TF A[N * N];
    TF tau[N];
    int32_t info;
    int32_t e;
};

// Householder QR without pivoting, tau in [1, 2]. qr.jl:9-60.
template <int N, class TF> inline void qr_factor(const double* J, QRFac<N, TF>& f) {
    f.e = factor_matrix<TF>(J, N * N, f.A);
    TF* A = f.A;
    f.info = 0;
    for (int k = 0; k < N; ++k) f.tau[k] = TF(0);
    for (int k = 0; k < N; ++k) {
        TF amax = TF(0);
        for (int i = k; i < N; ++i) amax = jmax(amax, TF(std::fabs(A[i + k * N])));
        TF x[N];
        for (int i = 0; i < N; ++i)
            x[i] = (i >= k && amax != TF(0)) ? A[i + k * N] / amax : TF(0);
        TF sigma = amax * rnorm(x, N);
        if (sigma != TF(0)) {
            TF x1 = A[k + k * N];
            TF phase = x1 == TF(0) ? TF(1) : x1 / TF(std::fabs(x1));
            TF v1 = phase * (sigma + TF(std::fabs(x1)));
            TF tk = (sigma + TF(std::fabs(x1))) / sigma;
            f.tau[k] = tk;
            for (int i = k + 1; i < N; ++i) A[i + k * N] = A[i + k * N] / v1;
            for (int j = k + 1; j < N; ++j) {
                TF s = A[k + j * N];
                for (int i = k + 1; i < N; ++i) s = s + A[i + k * N] * A[i + j * N];
                s = s * tk;
                A[k + j * N] = A[k + j * N] - s;
                for (int i = k + 1; i < N; ++i) A[i + j * N] = A[i + j * N] - A[i + k * N] * s;
            }
            A[k + k * N] = -phase * sigma;
        }
        if (A[k + k * N] == TF(0) && f.info == 0) f.info = k + 1;
    }
}

// qr.jl:63-89.
template <int N, class TF> inline void qr_backsolve(const QRFac<N, TF>& f, TF* x) {
    const TF* A = f.A;
    for (int k = 0; k < N; ++k) {
        TF s = x[k];
        for (int i = k + 1; i < N; ++i) s = s + A[i + k * N] * x[i];
        s = s * f.tau[k];
        x[k] = x[k] - s;
        for (int i = k + 1; i < N; ++i) x[i] = x[i] - A[i + k * N] * s;
    }
    for (int k = N - 1; k >= 0; --k) {
        TF xk = x[k] / A[k + k * N];
        x[k] = xk;
        for (int i = 0; i < k; ++i) x[i] = x[i] - A[i + k * N] * xk;
    }
}

// A factor of either kind, in TF. `qr` selects QRFactorization.
template <int N, class TF> struct Factor {
    bool qr;
    LUFac<N, TF> lu;
    QRFac<N, TF> q;
    int32_t info() const { return qr ? q.info : lu.info; }
    int32_t e() const { return qr ? q.e : lu.e; }
    void factor(const double* J, bool use_qr) {
        qr = use_qr;
        if (qr) qr_factor<N, TF>(J, q);
        else lu_factor<N, TF>(J, lu);
    }
    void backsolve(TF* x) const {
        if (qr) qr_backsolve<N, TF>(q, x);
        else lu_backsolve<N, TF>(lu, x);
    }
};

// Same-type ldiv!!: r scaled by 2^-k, solved, scaled back by 2^(k - e). factors.jl:931-936,
// with unscale :916-919.
template <int N> inline void ldiv_same(const Factor<N, double>& f, const double* r, double* d) {
    int k = rhs_exponent(r, N, f.e());
    for (int i = 0; i < N; ++i) d[i] = k == 0 ? r[i] : ldexp2(r[i], -k);
    f.backsolve(d);
    int e2 = k - f.e();
    if (e2 != 0)
        for (int i = 0; i < N; ++i) d[i] = ldexp2(d[i], e2);
}

// Mixed-type ldiv!!: r / max|r| rounded to TF, solved, multiplied by frac 2^(ex - e) in the
// wider type. factors.jl:943-949.
template <int N, class TF> inline void ldiv_mixed(const Factor<N, TF>& f, const double* r,
                                                  double* d) {
    double s = std::fabs(r[0]);
    for (int i = 1; i < N; ++i) s = jmax(s, std::fabs(r[i]));
    if (s == 0.0) {
        for (int i = 0; i < N; ++i) d[i] = 0.0;
        return;
    }
    TF x[N];
    for (int i = 0; i < N; ++i) x[i] = TF(r[i] / s);
    f.backsolve(x);
    int ex = 0;
    double frac = std::frexp(s, &ex);
    if (!std::isfinite(s)) ex = 0;
    for (int i = 0; i < N; ++i) d[i] = ldexp2(double(x[i]) * frac, (long)ex - f.e());
}

template <int N, class TF> inline void ldiv(const Factor<N, TF>& f, const double* r, double* d) {
    if constexpr (std::is_same<TF, double>::value) ldiv_same<N>(f, r, d);
    else ldiv_mixed<N, TF>(f, r, d);
}

// Julia's LinearAlgebra.givens(f, g, 1, 2) for real arguments (LAPACK's DLARTG algorithm, as
// Julia's givensAlgorithm states it); returns (c, s, r). Third-party: Julia stdlib.
inline void givens(double f, double g, double& cs, double& sn, double& r) {
    const double safmn2 = std::ldexp(1.0, -485), safmx2 = std::ldexp(1.0, 485);
    if (g == 0.0) {
        cs = 1.0; sn = 0.0; r = f;
    } else if (f == 0.0) {
        cs = 0.0; sn = 1.0; r = g;
    } else {
        double f1 = f, g1 = g;
        double scale = jmax(std::fabs(f1), std::fabs(g1));
        if (scale >= safmx2) {
            int count = 0;
            while (true) {
                ++count;
                f1 *= safmn2;
                g1 *= safmn2;
                scale = jmax(std::fabs(f1), std::fabs(g1));
                if (scale < safmx2 || count >= 20) break;
            }
            r = std::sqrt(f1 * f1 + g1 * g1);
            cs = f1 / r;
            sn = g1 / r;
            for (int i = 0; i < count; ++i) r *= safmx2;
        } else if (scale <= safmn2) {
            int count = 0;
            while (true) {
                ++count;
                f1 *= safmx2;
                g1 *= safmx2;
                scale = jmax(std::fabs(f1), std::fabs(g1));
                if (scale > safmn2) break;
            }
            r = std::sqrt(f1 * f1 + g1 * g1);
            cs = f1 / r;
            sn = g1 / r;
            for (int i = 0; i < count; ++i) r *= safmn2;
        } else {
            r = std::sqrt(f1 * f1 + g1 * g1);
            cs = f1 / r;
            sn = g1 / r;
        }
        if (std::fabs(f) > std::fabs(g) && cs < 0) {
            cs = -cs; sn = -sn; r = -r;
        }
    }
}

}  // namespace orc
