// Device residual families, selected by the GsbFamily tag. Each family gives:
//   F(x, out)            the residual, in the family's own operation order;
//   jacobian(x, js)      the forward-mode dual Jacobian (the N-partial pass of
//                        src/ad/forwarddiff_static.jl:50-65), held in a JState;
//   J(js, i, k)          entry (i, k) of that Jacobian (i, k compile-time after unrolling);
//   jvp(x, v, out)       the 1-partial dual pass, J(x) v (src/ad/jvp.jl:96-107).
// A family whose dual partials have structure holds only what the seeds leave nonzero: the
// cubic family's Jacobian is A off the diagonal exactly (each off-diagonal partial is A_ik
// plus products with zero seeds), so its JState is the diagonal, and A is read from the
// family's parameter block.
#pragma once

#include "gsb_dual.cuh"
#include "gsb_numerics.cuh"

namespace gsb {

// ─── GSB_FAMILY_CUBIC_AFFINE: F(x) = A x + 0.1 x.^3 - b, p = (A column-major n*n, b) ───────
// Row i: t = fma(A_in, x_n, ... fma(A_i2, x_2, A_i1 x_1)); F_i = fma(0.1, (x_i x_i) x_i, t) - b_i.
// Dual rules: the product of duals a*b has partials a.p b.v + b.p a.v, so with the seed
// e_i the partial of (x_i x_i) x_i is (x_i + x_i) x_i + x_i x_i, and
// J_ii = fma(0.1, that, A_ii).
// Rows: the block sits in a shared-memory row whose start is 16-byte aligned (the kernel stages
// it with one bulk copy and a row stride of 2 mod 4 doubles), and A and b are read two entries
// at a time (A(i, k), A(i+1, k) for even i), 16-byte loads that are free of bank conflicts at that
// stride; N is even. The arithmetic is the same, row by row and in the same order.
template <int N_, bool SharedA = false, bool Rows = false> struct CubicAffineT {
    static constexpr int N = N_, M = N_;
    // Parameters of a system: (A, b), or with SharedA (BatchParams, src/nonlinear/batched.jl:
    // 34-47) only b, A being the batch's shared block.
    static constexpr int NP = SharedA ? N_ : N_ * N_ + N_;
    static constexpr int kShared = SharedA ? N_ * N_ : 0;  // doubles of the CTA-shared block
    static constexpr bool lsq = false;
    static constexpr bool kPairs = Rows;
    static_assert(!Rows || (N_ % 2 == 0 && !SharedA), "paired reads: even N, a per-system A");
    const double* p;            // this system's parameter block in shared memory
    const double* a = nullptr;  // the shared A (column-major) in shared memory, with SharedA
    struct JState {
        double diag[N];
    };
    // The block stays in shared memory and is read at each use (a volatile shared load), rather
    // than hoisted out of the Newton loop into registers, which the factor needs.
    __device__ __forceinline__ double par(int k) const { return lds(smem_addr(p) + 8u * k); }
    __device__ __forceinline__ double A(int i, int k) const {
        if constexpr (SharedA) return lds(smem_addr(a) + 8u * (i + k * N));
        return par(i + k * N);
    }
    __device__ __forceinline__ double bv(int i) const { return SharedA ? par(i) : par(N * N + i); }
    // (A(i, k), A(i+1, k)) and (b_i, b_i+1) for even i, with Rows
    __device__ __forceinline__ void A2(int i, int k, double& v0, double& v1) const {
        lds2(smem_addr(p) + 8u * (i + k * N), v0, v1);
    }
    __device__ __forceinline__ void b2(int i, double& v0, double& v1) const {
        lds2(smem_addr(p) + 8u * (N * N + i), v0, v1);
    }
    __device__ __forceinline__ void F(const double (&x)[N], double (&out)[M]) const {
        if constexpr (Rows) {
#pragma unroll
            for (int i = 0; i < N; i += 2) {
                double a0, a1;
                A2(i, 0, a0, a1);
                double t0 = __dmul_rn(a0, x[0]), t1 = __dmul_rn(a1, x[0]);
#pragma unroll
                for (int j = 1; j < N; ++j) {
                    A2(i, j, a0, a1);
                    t0 = __fma_rn(a0, x[j], t0);
                    t1 = __fma_rn(a1, x[j], t1);
                }
                const double c0 = __dmul_rn(__dmul_rn(x[i], x[i]), x[i]);
                const double c1 = __dmul_rn(__dmul_rn(x[i + 1], x[i + 1]), x[i + 1]);
                double b0, b1;
                b2(i, b0, b1);
                out[i] = __dsub_rn(__fma_rn(0.1, c0, t0), b0);
                out[i + 1] = __dsub_rn(__fma_rn(0.1, c1, t1), b1);
            }
            return;
        }
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double t = __dmul_rn(A(i, 0), x[0]);
#pragma unroll
            for (int j = 1; j < N; ++j) t = __fma_rn(A(i, j), x[j], t);
            double c = __dmul_rn(__dmul_rn(x[i], x[i]), x[i]);
            out[i] = __dsub_rn(__fma_rn(0.1, c, t), bv(i));
        }
    }
    // A(i, i): with Rows, from the aligned pair that holds it
    __device__ __forceinline__ double Aii(int i) const {
        if constexpr (Rows) {
            double v0, v1;
            if (i % 2 == 0) {
                A2(i, i, v0, v1);
                return v0;
            }
            A2(i - 1, i, v0, v1);
            return v1;
        }
        return A(i, i);
    }
    __device__ __forceinline__ void jacobian(const double (&x)[N], JState& js) const {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double v = x[i];
            double cp = __dadd_rn(__dmul_rn(__dadd_rn(v, v), v), __dmul_rn(v, v));
            js.diag[i] = __fma_rn(0.1, cp, Aii(i));
        }
    }
    __device__ __forceinline__ double J(const JState& js, int i, int k) const {
        return i == k ? js.diag[i] : A(i, k);
    }
    // (J(i, k), J(i+1, k)) for even i, with Rows
    __device__ __forceinline__ void J2(const JState& js, int i, int k, double& v0, double& v1) const {
        A2(i, k, v0, v1);
        if (i == k) v0 = js.diag[i];
        if (i + 1 == k) v1 = js.diag[i + 1];
    }
    __device__ __forceinline__ void jvp(const double (&x)[N], const double (&v)[N],
                                        double (&out)[M]) const {
        auto rest = [&](int i, double t) {
            double xv = __dmul_rn(v[i], x[i]);
            double x2p = __dadd_rn(xv, xv);
            double cp = __dadd_rn(__dmul_rn(x2p, x[i]), __dmul_rn(v[i], __dmul_rn(x[i], x[i])));
            return __fma_rn(0.1, cp, t);
        };
        if constexpr (Rows) {
#pragma unroll
            for (int i = 0; i < N; i += 2) {
                double a0, a1;
                A2(i, 0, a0, a1);
                double t0 = __dmul_rn(a0, v[0]), t1 = __dmul_rn(a1, v[0]);
#pragma unroll
                for (int j = 1; j < N; ++j) {
                    A2(i, j, a0, a1);
                    t0 = __fma_rn(a0, v[j], t0);
                    t1 = __fma_rn(a1, v[j], t1);
                }
                out[i] = rest(i, t0);
                out[i + 1] = rest(i + 1, t1);
            }
            return;
        }
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double t = __dmul_rn(A(i, 0), v[0]);
#pragma unroll
            for (int j = 1; j < N; ++j) t = __fma_rn(A(i, j), v[j], t);
            out[i] = rest(i, t);
        }
    }
};
template <int N> using CubicAffine = CubicAffineT<N, false>;
template <int N> using CubicAffineSharedA = CubicAffineT<N, true>;
template <int N> using CubicAffineRows = CubicAffineT<N, false, true>;

// The shared block of a family (0 doubles for families without one).
template <class Fam, class = void> struct SharedLen {
    static constexpr int value = 0;
};
template <class Fam> struct SharedLen<Fam, decltype(void(Fam::kShared))> {
    static constexpr int value = Fam::kShared;
};

// Whether a family reads its block in aligned pairs (and needs 16-byte aligned rows).
template <class Fam, class = void> struct PairsOf {
    static constexpr bool value = false;
};
template <class Fam> struct PairsOf<Fam, decltype(void(Fam::kPairs))> {
    static constexpr bool value = Fam::kPairs;
};

// Every entry of a family's Jacobian, column by column and down each column (the order of the
// factor's load and of grad_ratio_and_norm's sums): body(i, k, J(i, k)). A family with aligned
// pairs reads (J(i, k), J(i+1, k)) at once.
template <class Fam, class Body>
__device__ __forceinline__ void for_each_J(const Fam& fam, const typename Fam::JState& js, Body body) {
#pragma unroll
    for (int k = 0; k < Fam::N; ++k) {
        if constexpr (PairsOf<Fam>::value) {
#pragma unroll
            for (int i = 0; i < Fam::M; i += 2) {
                double v0, v1;
                fam.J2(js, i, k, v0, v1);
                body(i, k, v0);
                body(i + 1, k, v1);
            }
        } else {
#pragma unroll
            for (int i = 0; i < Fam::M; ++i) body(i, k, fam.J(js, i, k));
        }
    }
}

// A family with an analytic Jacobian (the problem's `J`, src/ad/forwarddiff_static.jl:36-38)
// holds the full matrix; its JVP is J(x) v as a left fold (src/ad/jvp.jl:88-91).
template <int N_, int M_> struct FullJState {
    double J[M_ * N_];
};

// ─── a family given by its residual alone ───────────────────────────────────────────────────
// Fn::eval<S>(fam, x, out) writes the residual for any scalar S with the operations of
// gsb_dual.cuh; the family evaluates it on Real for F, on Dual<N> seeded with the identity for
// the Jacobian (one N-partial pass, src/ad/forwarddiff_static.jl:50-65) and on Dual<1> seeded
// with v for the JVP (src/ad/jvp.jl:96-107). Parameters (Fn::NP doubles per system) are read
// from the system's shared-memory row with par(k).
template <class Fn> struct DualFamily {
    static constexpr int N = Fn::N, M = Fn::N, NP = Fn::NP;
    static constexpr bool lsq = false;
    const double* p;
    using JState = FullJState<N, M>;
    __device__ __forceinline__ double par(int k) const { return lds(smem_addr(p) + 8u * k); }
    __device__ __forceinline__ void F(const double (&x)[N], double (&out)[M]) const {
        Real xr[N], r[M];
#pragma unroll
        for (int i = 0; i < N; ++i) xr[i] = Real{x[i]};
        Fn::eval(*this, xr, r);
#pragma unroll
        for (int i = 0; i < M; ++i) out[i] = r[i].v;
    }
    __device__ __forceinline__ void jacobian(const double (&x)[N], JState& js) const {
        Dual<N> xd[N], rd[M];
#pragma unroll
        for (int j = 0; j < N; ++j) {
            xd[j].v = x[j];
#pragma unroll
            for (int k = 0; k < N; ++k) xd[j].p[k] = k == j ? 1.0 : 0.0;
        }
        Fn::eval(*this, xd, rd);
#pragma unroll
        for (int j = 0; j < N; ++j)
#pragma unroll
            for (int i = 0; i < M; ++i) js.J[i + j * M] = rd[i].p[j];
    }
    __device__ __forceinline__ double J(const JState& js, int i, int k) const { return js.J[i + k * M]; }
    __device__ __forceinline__ void jvp(const double (&x)[N], const double (&v)[N],
                                        double (&out)[M]) const {
        Dual<1> xd[N], rd[M];
#pragma unroll
        for (int j = 0; j < N; ++j) {
            xd[j].v = x[j];
            xd[j].p[0] = v[j];
        }
        Fn::eval(*this, xd, rd);
#pragma unroll
        for (int i = 0; i < M; ++i) out[i] = rd[i].p[0];
    }
};

// The cubic-affine residual of CubicAffineT written as a template over its scalar: each row
// fma(A_in, x_n, ... fma(A_i2, x_2, A_i1 x_1)), then fma(0.1, (x_i x_i) x_i, row) - b_i, the
// same operations as the written-out family, whose Jacobian rule this family's dual pass checks.
template <int N_> struct CubicAffineFn {
    static constexpr int N = N_, NP = N_ * N_ + N_;
    template <class Fam, class S>
    __device__ __forceinline__ static void eval(const Fam& f, const S (&x)[N], S (&out)[N]) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            S t = f.par(i) * x[0];
#pragma unroll
            for (int j = 1; j < N; ++j) t = fmac(f.par(i + j * N), x[j], t);
            S c = x[i] * x[i] * x[i];
            out[i] = fmac(0.1, c, t) - f.par(N * N + i);
        }
    }
};

// Wood's function (problem 4 of the reference's standard set, test/helpers/standard_problems.jl)
// with the coupling weight of its second and fourth residuals (20.2 in the standard problem) as
// the one parameter w of a system.
struct WoodFn {
    static constexpr int N = 4, NP = 1;
    template <class Fam, class S>
    __device__ __forceinline__ static void eval(const Fam& f, const S (&x)[4], S (&out)[4]) {
        const double w = f.par(0);
        const S t1 = x[1] - x[0] * x[0];
        const S t2 = x[3] - x[2] * x[2];
        out[0] = -200.0 * x[0] * t1 - (1.0 - x[0]);
        out[1] = 200.0 * t1 + w * (x[1] - 1.0) + 19.8 * (x[3] - 1.0);
        out[2] = -180.0 * x[2] * t2 - (1.0 - x[2]);
        out[3] = 180.0 * t2 + w * (x[3] - 1.0) + 19.8 * (x[1] - 1.0);
    }
};

// ─── test/nonlinear/batched.jl:54-90: the six-outcome residual, p = outcome 1..6 ───────────
struct Hetero6 {
    static constexpr int N = 2, M = 2, NP = 1;
    static constexpr bool lsq = false;
    const double* p;
    using JState = FullJState<2, 2>;
    __device__ __forceinline__ int code() const { return int(p[0]); }
    __device__ __forceinline__ void F(const double (&x)[2], double (&out)[2]) const {
        switch (code()) {
        case 1: out[0] = __dsub_rn(x[0], 2.0); out[1] = __dsub_rn(x[1], 3.0); break;
        case 2: out[0] = 1.0; out[1] = 1.0; break;
        case 3: out[0] = __dsub_rn(x[0], 100.0); out[1] = __dsub_rn(x[1], 100.0); break;
        case 4: out[0] = 1.0; out[1] = 1.0; break;
        case 5: out[0] = kNaN; out[1] = kNaN; break;
        default:
            out[0] = __dadd_rn(__dmul_rn(x[0], x[0]), 1.0);
            out[1] = __dadd_rn(__dmul_rn(x[1], x[1]), 1.0);
            break;
        }
    }
    __device__ __forceinline__ void jacobian(const double (&)[2], JState& js) const {
        double d;
        switch (code()) {
        case 1: d = 1.0; break;
        case 2: d = 1e16; break;
        case 3: d = 2.0; break;
        case 4: d = 0.0; break;
        case 5: d = 1.0; break;
        default: d = -1.0; break;
        }
        js.J[0] = d; js.J[1] = 0.0; js.J[2] = 0.0; js.J[3] = d;
    }
    __device__ __forceinline__ double J(const JState& js, int i, int k) const {
        return js.J[i + 2 * k];
    }
    __device__ __forceinline__ void jvp(const double (&x)[2], const double (&v)[2],
                                        double (&out)[2]) const {
        JState js;
        jacobian(x, js);
#pragma unroll
        for (int i = 0; i < 2; ++i) out[i] = __dadd_rn(__dmul_rn(js.J[i], v[0]), __dmul_rn(js.J[i + 2], v[1]));
    }
};

// ─── test/nonlinear/batched.jl:92-104: the coupled residual, p = (p1, p2) ──────────────────
struct Coupled2 {
    static constexpr int N = 2, M = 2, NP = 2;
    static constexpr bool lsq = false;
    const double* p;
    using JState = FullJState<2, 2>;
    __device__ __forceinline__ void F(const double (&x)[2], double (&out)[2]) const {
        out[0] = __dsub_rn(__dadd_rn(x[0], __ddiv_rn(__dmul_rn(x[1], x[1]), 8.0)), p[0]);
        out[1] = __dsub_rn(__dadd_rn(x[1], __ddiv_rn(__dmul_rn(x[0], x[0]), 8.0)), p[1]);
    }
    __device__ __forceinline__ void jacobian(const double (&x)[2], JState& js) const {
        js.J[0] = 1.0;
        js.J[1] = __ddiv_rn(x[0], 4.0);
        js.J[2] = __ddiv_rn(x[1], 4.0);
        js.J[3] = 1.0;
    }
    __device__ __forceinline__ double J(const JState& js, int i, int k) const {
        return js.J[i + 2 * k];
    }
    __device__ __forceinline__ void jvp(const double (&x)[2], const double (&v)[2],
                                        double (&out)[2]) const {
        JState js;
        jacobian(x, js);
#pragma unroll
        for (int i = 0; i < 2; ++i) out[i] = __dadd_rn(__dmul_rn(js.J[i], v[0]), __dmul_rn(js.J[i + 2], v[1]));
    }
};

}  // namespace gsb
