// ORACLE — test infrastructure only, never linked into the product. liboracle.so: the CPU
// restatement of GeometricSolvers.jl's R2 batch (`solve_batch!`, src/nonlinear/batched.jl:
// 171-195: one R1 `solve!!` per system) behind the same C-ABI structs as libgsb, so that a test
// runs both on the same inputs. The batch loop splits the systems into one contiguous range per
// thread, the static schedule of the reference's own host R1 loop
// (`Threads.@threads :static`, scripts/r2_throughput.jl:107-136).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <thread>
#include <vector>

#include "../include/gsb.h"
#include "oracle_solver.hpp"
#include "oracle_standard.hpp"

using namespace orc;

namespace {

// Oracle-only test families (pins from the reference's tests).
enum { FAM_QUADMOD2 = 200, FAM_CUBICDIAG2 = 201 };

Opts to_opts(const GsbOptions* g) {
    Opts o;
    o.f_abstol = g->f_abstol;
    o.f_reltol = g->f_reltol;
    o.x_abstol = g->x_abstol;
    o.x_reltol = g->x_reltol;
    o.min_iterations = g->min_iterations;
    o.max_iterations = g->max_iterations;
    o.max_stalls = g->max_stalls;
    o.maxnorm = g->norm == 1;
    o.g_tol = g->g_tol;
    o.kappa = g->kappa;
    o.roundoff = g->roundoff != 0;
    o.rate_test = g->rate_test != 0;
    return o;
}

Meth to_meth(const GsbMethod* g) {
    Meth m;
    m.qr = g->linsolve == GSB_QR;
    m.f32 = g->factor_precision == GSB_F32;
    m.refine = g->refinement == GSB_REFINEMENT;
    m.refine_maxiter = g->refine_maxiter;
    m.refine_eta = g->refine_eta;
    m.glob = g->globalization;
    m.static_alpha = g->static_alpha;
    m.bt_c1 = g->bt_c1;
    m.bt_p = g->bt_p;
    m.bt_maxiter = g->bt_maxiter;
    m.mu0 = g->lm_mu0;
    m.mu_min = g->lm_mu_min;
    m.mu_max = g->lm_mu_max;
    m.mu_decrease = g->lm_mu_decrease;
    m.mu_increase = g->lm_mu_increase;
    m.rho_accept = g->lm_rho_accept;
    m.reuse = g->reuse;
    m.dl_radius = g->dogleg_radius;
    return m;
}

void to_status(const Status& s, GsbStatus64* out) {
    std::memset(out, 0, sizeof(*out));
    out->code = (uint8_t)s.code;
    out->f_calls = 0;
    out->iterations = s.iterations;
    out->fnorm = s.fnorm;
    out->stepnorm = s.stepnorm;
    out->step_failures = s.step_failures;
    out->promoted = s.promoted;
    out->stationary = s.stationary;
    out->jvp_calls = 0;
    out->rank = s.rank;
    out->nullnorm = s.nullnorm;
    out->gradratio = s.gradratio;
    out->rate = s.rate;
    out->contracted = s.contracted;
    out->reused = s.reused;
}

struct Batch {
    double* X;
    int x_layout;
    void* S;
    int s_kind;
    const double* P;
    int p_layout;
    const int64_t* order;
    int order_base;
    int64_t nsys;
    const double* shared;
};

inline double& xref(const Batch& b, int64_t s, int k, int n) {
    return b.x_layout == GSB_SOA ? b.X[(int64_t)k * b.nsys + s] : b.X[s * n + k];
}
inline double pget(const Batch& b, int64_t s, int k, int np) {
    return b.p_layout == GSB_SOA ? b.P[(int64_t)k * b.nsys + s] : b.P[s * np + k];
}

// One system: gather, solve!!, scatter (src/nonlinear/batched.jl:171-179).
template <class Prob, class Make>
void run_batch(const Batch& b, const Meth& m, const Opts& o, int np, Make make, int nthreads) {
    constexpr int N = Prob::N;
    auto work = [&](int64_t lo, int64_t hi) {
        std::vector<double> p(np > 0 ? np : 1);
        for (int64_t i = lo; i < hi; ++i) {
            int64_t idx = b.order ? b.order[i] - b.order_base : i;
            double x[N];
            for (int k = 0; k < N; ++k) x[k] = xref(b, idx, k, N);
            for (int k = 0; k < np; ++k) p[k] = pget(b, idx, k, np);
            Prob prob = make(p.data(), b.shared);
            Solver<Prob> s(prob, m, o);
            Status st = s.solve(x);
            for (int k = 0; k < N; ++k) xref(b, idx, k, N) = x[k];
            if (b.s_kind == GSB_STATUS64) to_status(st, (GsbStatus64*)b.S + idx);
            else ((uint8_t*)b.S)[idx] = (uint8_t)st.code;
        }
    };
    int nt = nthreads < 1 ? 1 : nthreads;
    if (nt == 1 || b.nsys < 2) {
        work(0, b.nsys);
        return;
    }
    std::vector<std::thread> pool;
    int64_t chunk = (b.nsys + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        int64_t lo = t * chunk, hi = lo + chunk < b.nsys ? lo + chunk : b.nsys;
        if (lo >= hi) break;
        pool.emplace_back(work, lo, hi);
    }
    for (auto& th : pool) th.join();
}

template <int N> int run_cubic(const Batch& b, const Meth& m, const Opts& o, int nt) {
    run_batch<CubicAffine<N>>(b, m, o, N * N + N,
                              [](const double* p, const double*) { return CubicAffine<N>{p}; }, nt);
    return 0;
}

int64_t param_count(int family, int n, int m) {
    switch (family) {
    case GSB_FAMILY_CUBIC_AFFINE: return (int64_t)n * n + n;
    case GSB_FAMILY_EXPSUM3_LSQ: return m;
    case GSB_FAMILY_IRK3_HENON_HEILES: return 4;
    case GSB_FAMILY_HETERO6: return 1;
    case GSB_FAMILY_COUPLED2: return 2;
    case GSB_FAMILY_WOOD: return 1;
    case GSB_FAMILY_CUBIC_AFFINE_DUAL: return (int64_t)n * n + n;
    case FAM_QUADMOD2: return 6;
    case FAM_CUBICDIAG2: return 8;
    default: return -1;
    }
}

}  // namespace

extern "C" {

int oracle_abi_version(void) { return GSB_ABI_VERSION; }

int oracle_max_threads(void) { return (int)std::thread::hardware_concurrency(); }

// The error of gsb_exp::exp (the exponential-sum family's exp, shared with the batch kernel)
// against long double expl on n arguments: a quarter uniform in [-1, 1], a quarter in [-40, 5]
// (the fit's range) and half uniform in [lo, hi]. Writes the largest error in ulp of the exact
// value (as far as expl resolves it), its argument and the count of results that differ from
// expl rounded to double. Normal results only.
int oracle_exp_check(int64_t n, uint64_t seed, double lo, double hi, double* max_ulp,
                     double* worst_x, int64_t* not_nearest) {
    const int nt = std::max(1, (int)std::thread::hardware_concurrency());
    std::vector<double> mu(nt, 0.0), wx(nt, 0.0);
    std::vector<int64_t> nn(nt, 0);
    std::vector<std::thread> th;
    for (int w = 0; w < nt; ++w) {
        th.emplace_back([&, w] {
            uint64_t st = seed * 0x9E3779B97F4A7C15ull + (uint64_t)w * 0xD1B54A32D192ED03ull + 1;
            auto next = [&] {  // splitmix64
                uint64_t z = (st += 0x9E3779B97F4A7C15ull);
                z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
                z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
                return (double)((z ^ (z >> 31)) >> 11) * 0x1.0p-53;
            };
            for (int64_t i = w; i < n; i += nt) {
                const double u = next();
                const double x = (i % 4 == 0) ? -1.0 + 2.0 * u
                                 : (i % 4 == 1) ? -40.0 + 45.0 * u : lo + (hi - lo) * u;
                const double a = gsb_exp::exp(x);
                const long double r = expl((long double)x);
                if (!(r >= (long double)2.2250738585072014e-308) || !std::isfinite((double)r))
                    continue;
                int ex;
                frexpl(r, &ex);
                const double err = (double)(fabsl((long double)a - r) / ldexpl(1.0L, ex - 53));
                if (err > mu[w]) {
                    mu[w] = err;
                    wx[w] = x;
                }
                if ((double)r != a) ++nn[w];
            }
        });
    }
    for (auto& t : th) t.join();
    *max_ulp = 0.0;
    *worst_x = 0.0;
    *not_nearest = 0;
    for (int w = 0; w < nt; ++w) {
        if (mu[w] > *max_ulp) {
            *max_ulp = mu[w];
            *worst_x = wx[w];
        }
        *not_nearest += nn[w];
    }
    return 0;
}

double oracle_exp(double x) { return gsb_exp::exp(x); }

// The CPU batch over host arrays, with the arguments of gsb_solve_batch; nthreads <= 0 takes
// every hardware thread.
int oracle_solve_batch(const GsbProblem* prob, const GsbMethod* method, const GsbOptions* opt,
                       double* X, int32_t x_layout, void* S, int32_t s_kind, const double* P,
                       int32_t p_layout, const int64_t* order, int32_t order_base, int64_t nsys,
                       int32_t nthreads) {
    if (nsys == 0) return 0;
    Batch b{X, x_layout, S, s_kind, P, p_layout, order, order_base, nsys, prob->shared};
    Meth m = to_meth(method);
    Opts o = to_opts(opt);
    int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
    const int n = prob->n;
    switch (prob->family) {
    case GSB_FAMILY_CUBIC_AFFINE:
        switch (n) {
        case 1: return run_cubic<1>(b, m, o, nt);
        case 2: return run_cubic<2>(b, m, o, nt);
        case 3: return run_cubic<3>(b, m, o, nt);
        case 4: return run_cubic<4>(b, m, o, nt);
        case 5: return run_cubic<5>(b, m, o, nt);
        case 6: return run_cubic<6>(b, m, o, nt);
        case 7: return run_cubic<7>(b, m, o, nt);
        case 8: return run_cubic<8>(b, m, o, nt);
        case 10: return run_cubic<10>(b, m, o, nt);
        case 12: return run_cubic<12>(b, m, o, nt);
        case 16: return run_cubic<16>(b, m, o, nt);
        case 24: return run_cubic<24>(b, m, o, nt);
        case 32: return run_cubic<32>(b, m, o, nt);
        default: return GSB_ERR_UNSUPPORTED;
        }
    case GSB_FAMILY_EXPSUM3_LSQ:
        if (n != 6 || prob->m != 64) return GSB_ERR_UNSUPPORTED;
        run_batch<ExpSum3<64>>(b, m, o, 64,
                               [](const double* p, const double* sh) { return ExpSum3<64>{p, sh}; },
                               nt);
        return 0;
    case GSB_FAMILY_IRK3_HENON_HEILES:
        if (n != 12) return GSB_ERR_UNSUPPORTED;
        run_batch<IrkHenonHeiles>(
            b, m, o, 4, [](const double* p, const double* sh) { return IrkHenonHeiles{p, sh}; }, nt);
        return 0;
    case GSB_FAMILY_HETERO6:
        run_batch<Hetero6>(b, m, o, 1, [](const double* p, const double*) { return Hetero6{p}; },
                           nt);
        return 0;
    case GSB_FAMILY_COUPLED2:
        run_batch<Coupled2>(b, m, o, 2, [](const double* p, const double*) { return Coupled2{p}; },
                            nt);
        return 0;
    case GSB_FAMILY_WOOD:
        if (n != 4) return GSB_ERR_UNSUPPORTED;
        run_batch<Wood>(b, m, o, 1, [](const double* p, const double*) { return Wood{p}; }, nt);
        return 0;
    case GSB_FAMILY_CUBIC_AFFINE_DUAL:  // the oracle's cubic family already takes dual passes
        switch (n) {
        case 2: return run_cubic<2>(b, m, o, nt);
        case 3: return run_cubic<3>(b, m, o, nt);
        case 4: return run_cubic<4>(b, m, o, nt);
        default: return GSB_ERR_UNSUPPORTED;
        }
    case FAM_QUADMOD2:
        run_batch<QuadMod2>(b, m, o, 6, [](const double* p, const double*) { return QuadMod2{p}; },
                            nt);
        return 0;
    case FAM_CUBICDIAG2:
        run_batch<CubicDiag2>(b, m, o, 8,
                              [](const double* p, const double*) { return CubicDiag2{p}; }, nt);
        return 0;
    default: return GSB_ERR_UNSUPPORTED;
    }
}

int64_t oracle_param_count(int32_t family, int32_t n, int32_t m) { return param_count(family, n, m); }

// One cell of the standard test set: problem `number` (1..23) from x0 with column 0 "Newton
// Static LU" or 1 "Newton Backtracking LU", default Options with max_iterations; returns the
// size n of the problem or a negative value. f_evals counts primal residual evaluations, as the
// reference's CountedResidual does (test/helpers/standard_cells.jl:82-96).
int oracle_standard_cell(int32_t number, const double* x0, int32_t column, int32_t max_iterations,
                         double* x_out, GsbStatus64* st, int64_t* f_evals, int64_t* dual_evals) {
    GsbOptions go;
    go.f_abstol = 0.0;
    go.f_reltol = 1.4901161193847656e-08;
    go.x_abstol = 0.0;
    go.x_reltol = 2.0 * kEps;
    go.min_iterations = 0;
    go.max_iterations = max_iterations;
    go.max_stalls = 2;
    go.norm = 0;
    go.g_tol = 1.4901161193847656e-08;
    go.kappa = 0.1;
    go.roundoff = 0;
    go.rate_test = 1;
    Opts o = to_opts(&go);
    Meth m;
    // columns of test/verification/standard_reference.csv: 0 "Newton Static LU",
    // 1 "Newton Backtracking LU", 2 "Newton Backtracking QR", 3 "Newton DogLeg LU",
    // 4 "Newton reuse 3 Backtracking LU"
    m.glob = column == 0 ? G_STATIC : column == 3 ? G_DOGLEG : G_BACKTRACKING;
    m.qr = column == 2;
    m.reuse = column == 4 ? 3 : 0;
    int n = -1;
    auto run = [&](auto prob) {
        using P = decltype(prob);
        double x[P::N];
        for (int k = 0; k < P::N; ++k) x[k] = x0[k];
        Solver<P> s(prob, m, o);
        Status r = s.solve(x);
        for (int k = 0; k < P::N; ++k) x_out[k] = x[k];
        to_status(r, st);
        *f_evals = s.f_evals;
        *dual_evals = s.dual_evals;
        n = P::N;
    };
    switch (number) {
    case 1: run(Standard<10, 1>{}); break;
    case 2: run(Standard<4, 2>{}); break;
    case 3: run(Standard<2, 3>{}); break;
    case 4: run(Standard<4, 4>{}); break;
    case 5: run(Standard<3, 5>{}); break;
    case 6: run(Standard<2, 6>{}); break;
    case 7: run(Standard<2, 7>{}); break;
    case 8: run(Standard<10, 8>{}); break;
    case 9: run(Standard<10, 9>{}); break;
    case 10: run(Standard<10, 10>{}); break;
    case 11: run(Standard<10, 11>{}); break;
    case 12: run(Standard<10, 12>{}); break;
    case 13: run(Standard<10, 13>{}); break;
    case 14: run(Standard<10, 14>{}); break;
    case 15: run(Standard<4, 15>{}); break;
    case 16: run(Standard<9, 16>{}); break;
    case 17: run(Standard<2, 17>{}); break;
    case 18: run(Standard<2, 18>{}); break;
    case 19: run(Standard<2, 19>{}); break;
    case 20: run(Standard<1, 20>{}); break;
    case 21: run(Standard<2, 21>{}); break;
    case 22: run(Standard<2, 22>{}); break;
    case 23: run(Standard<10, 23>{}); break;
    default: return -1;
    }
    return n;
}

// The residual of standard problem `number` at x (checks the restatement against the roots
// and the hand values of test/verification/standard.jl:55-79).
int oracle_standard_residual(int32_t number, const double* x, double* out) {
    int n = -1;
    auto ev = [&](auto prob) {
        using P = decltype(prob);
        prob.F(x, out);
        n = P::N;
    };
    switch (number) {
    case 1: ev(Standard<10, 1>{}); break;
    case 2: ev(Standard<4, 2>{}); break;
    case 3: ev(Standard<2, 3>{}); break;
    case 4: ev(Standard<4, 4>{}); break;
    case 5: ev(Standard<3, 5>{}); break;
    case 6: ev(Standard<2, 6>{}); break;
    case 7: ev(Standard<2, 7>{}); break;
    case 8: ev(Standard<10, 8>{}); break;
    case 9: ev(Standard<10, 9>{}); break;
    case 10: ev(Standard<10, 10>{}); break;
    case 11: ev(Standard<10, 11>{}); break;
    case 12: ev(Standard<10, 12>{}); break;
    case 13: ev(Standard<10, 13>{}); break;
    case 14: ev(Standard<10, 14>{}); break;
    case 15: ev(Standard<4, 15>{}); break;
    case 16: ev(Standard<9, 16>{}); break;
    case 17: ev(Standard<2, 17>{}); break;
    case 18: ev(Standard<2, 18>{}); break;
    case 19: ev(Standard<2, 19>{}); break;
    case 20: ev(Standard<1, 20>{}); break;
    case 21: ev(Standard<2, 21>{}); break;
    case 22: ev(Standard<2, 22>{}); break;
    case 23: ev(Standard<10, 23>{}); break;
    default: return -1;
    }
    return n;
}

// The Backtracking search along a line given by callbacks φ(α) and φ′(α), for the unit pins of
// test/globalization/linesearch.jl. Returns the code; α, φ and the evaluation count by pointer.
typedef double (*oracle_line_fn)(double alpha, void* ctx);
int oracle_backtracking(double c1, double p, int32_t maxiter, oracle_line_fn phi,
                        oracle_line_fn dphi, void* ctx, int32_t exact, double phi0, double alpha,
                        double* alpha_out, double* phi_out, int32_t* evals_out) {
    struct CbLine {
        oracle_line_fn phi, dphi;
        void* ctx;
        double merit(double a) { return phi(a, ctx); }
        double slope0() { return dphi(0.0, ctx); }
    } lf{phi, dphi, ctx};
    LSResult r = backtracking(c1, p, maxiter, lf, exact != 0, phi0, alpha);
    *alpha_out = r.alpha;
    *phi_out = r.phi;
    *evals_out = r.evals;
    return r.code;
}

double oracle_backtrack_step(double phi0, double d0, double a, double pa, double ap, double pp,
                             double p) {
    return backtrack_step(phi0, d0, a, pa, ap, pp, p);
}

double oracle_ldexp2(double x, int64_t e) { return ldexp2(x, (long)e); }
float oracle_ldexp2f(float x, int64_t e) { return ldexp2(x, (long)e); }
double oracle_rnorm(const double* a, int32_t n) { return rnorm(a, n); }
int32_t oracle_matrix_exponent(const double* a, int32_t len) { return matrix_exponent(a, len); }
int32_t oracle_rhs_exponent(const double* r, int32_t n, int32_t e) { return rhs_exponent(r, n, e); }

// The LU (qr = 0) or QR (qr = 1) factor and solve of an n x n column-major J (n in 1..8), in
// Float64 (f32 = 0) or Float32 (f32 = 1): d = J \ r through the reference's ldiv!!. Returns
// info; the exponent e of the factor by pointer.
int32_t oracle_factor_solve(const double* J, int32_t n, int32_t qr, int32_t f32, const double* r,
                            double* d, int32_t* e_out) {
    int32_t info = -1;
    auto go = [&](auto nn) {
        constexpr int N = decltype(nn)::value;
        if (f32) {
            Factor<N, float> f;
            f.factor(J, qr != 0);
            info = f.info();
            *e_out = f.e();
            if (info == 0) ldiv<N, float>(f, r, d);
        } else {
            Factor<N, double> f;
            f.factor(J, qr != 0);
            info = f.info();
            *e_out = f.e();
            if (info == 0) ldiv<N, double>(f, r, d);
        }
    };
    switch (n) {
    case 1: go(std::integral_constant<int, 1>{}); break;
    case 2: go(std::integral_constant<int, 2>{}); break;
    case 3: go(std::integral_constant<int, 3>{}); break;
    case 4: go(std::integral_constant<int, 4>{}); break;
    case 5: go(std::integral_constant<int, 5>{}); break;
    case 6: go(std::integral_constant<int, 6>{}); break;
    case 7: go(std::integral_constant<int, 7>{}); break;
    case 8: go(std::integral_constant<int, 8>{}); break;
    default: return -2;
    }
    return info;
}

// The Givens rotation (c, s, r) of the LM stacked solve.
void oracle_givens(double f, double g, double* c, double* s, double* r) { givens(f, g, *c, *s, *r); }

// The residual and the dual Jacobian (column-major m x n) of a batch family at one system, for
// tests of the device families.
int oracle_family_eval(const GsbProblem* prob, const double* x, const double* p, double* F,
                       double* J) {
    Meth m;
    Opts o{};
    auto ev = [&](auto pr) {
        using P = decltype(pr);
        Solver<P> s(pr, m, o);
        s.F(x, F);
        if (J) s.jacobian(x, J);
    };
    switch (prob->family) {
    case GSB_FAMILY_CUBIC_AFFINE:
        switch (prob->n) {
        case 3: ev(CubicAffine<3>{p}); return 0;
        case 8: ev(CubicAffine<8>{p}); return 0;
        default: return GSB_ERR_UNSUPPORTED;
        }
    case GSB_FAMILY_EXPSUM3_LSQ: ev(ExpSum3<64>{p, prob->shared}); return 0;
    case GSB_FAMILY_IRK3_HENON_HEILES: ev(IrkHenonHeiles{p, prob->shared}); return 0;
    default: return GSB_ERR_UNSUPPORTED;
    }
}

}  // extern "C"
