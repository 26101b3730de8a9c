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

#include "gsb_numerics.cuh"

namespace gsb {

// ─── GSB_FAMILY_CUBIC_AFFINE: F(x) = A x + 0.1 x.^3 - b, p = (A column-major n*n, b) ───────
// Row i: t = fma(A_in, x_n, ... fma(A_i2, x_2, A_i1 x_1)); F_i = fma(0.1, (x_i x_i) x_i, t) - b_i.
// Dual rules: the product of duals a*b has partials a.p b.v + b.p a.v, so with the seed
// e_i the partial of (x_i x_i) x_i is (x_i + x_i) x_i + x_i x_i, and
// J_ii = fma(0.1, that, A_ii).
template <int N_, bool SharedA = false> struct CubicAffineT {
    static constexpr int N = N_, M = N_;
    // Parameters of a system: (A, b), or with SharedA (BatchParams, src/nonlinear/batched.jl:
    // 34-47) only b, A being the batch's shared block.
    static constexpr int NP = SharedA ? N_ : N_ * N_ + N_;
    static constexpr int kShared = SharedA ? N_ * N_ : 0;  // doubles of the CTA-shared block
    static constexpr bool lsq = false;
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
    __device__ __forceinline__ void F(const double (&x)[N], double (&out)[M]) const {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double t = __dmul_rn(A(i, 0), x[0]);
#pragma unroll
            for (int j = 1; j < N; ++j) t = __fma_rn(A(i, j), x[j], t);
            double c = __dmul_rn(__dmul_rn(x[i], x[i]), x[i]);
            out[i] = __dsub_rn(__fma_rn(0.1, c, t), bv(i));
        }
    }
    __device__ __forceinline__ void jacobian(const double (&x)[N], JState& js) const {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double v = x[i];
            double cp = __dadd_rn(__dmul_rn(__dadd_rn(v, v), v), __dmul_rn(v, v));
            js.diag[i] = __fma_rn(0.1, cp, A(i, i));
        }
    }
    __device__ __forceinline__ double J(const JState& js, int i, int k) const {
        return i == k ? js.diag[i] : A(i, k);
    }
    __device__ __forceinline__ void jvp(const double (&x)[N], const double (&v)[N],
                                        double (&out)[M]) const {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double t = __dmul_rn(A(i, 0), v[0]);
#pragma unroll
            for (int j = 1; j < N; ++j) t = __fma_rn(A(i, j), v[j], t);
            double xv = __dmul_rn(v[i], x[i]);
            double x2p = __dadd_rn(xv, xv);
            double cp = __dadd_rn(__dmul_rn(x2p, x[i]), __dmul_rn(v[i], __dmul_rn(x[i], x[i])));
            out[i] = __fma_rn(0.1, cp, t);
        }
    }
};
template <int N> using CubicAffine = CubicAffineT<N, false>;
template <int N> using CubicAffineSharedA = CubicAffineT<N, true>;

// The shared block of a family (0 doubles for families without one).
template <class Fam, class = void> struct SharedLen {
    static constexpr int value = 0;
};
template <class Fam> struct SharedLen<Fam, decltype(void(Fam::kShared))> {
    static constexpr int value = Fam::kShared;
};

// A family with an analytic Jacobian (the problem's `J`, src/ad/forwarddiff_static.jl:36-38)
// holds the full matrix; its JVP is J(x) v as a left fold (src/ad/jvp.jl:88-91).
template <int N_, int M_> struct FullJState {
    double J[M_ * N_];
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
