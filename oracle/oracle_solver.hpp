// ORACLE — test infrastructure only. The R1 solve loop `solve!!` of GeometricSolvers.jl with the
// Newton step (plain, mixed-precision with LU-IR refinement and promotion) and the
// Levenberg–Marquardt step (stacked Givens), the Static and Backtracking globalizations, and
// the stopping tests. Each function cites the reference file:line it restates.
#pragma once

#include <type_traits>

#include "oracle_core.hpp"
#include "oracle_dual.hpp"

namespace orc {

// Options{Float64}, src/base/options.jl:58-71.
struct Opts {
    double f_abstol, f_reltol, x_abstol, x_reltol;
    int min_iterations, max_iterations, max_stalls;
    bool maxnorm;
    double g_tol, kappa;
    bool roundoff, rate_test;
};

enum Glob : int { G_STATIC = 0, G_BACKTRACKING = 1, G_LM = 2, G_DOGLEG = 3 };

// The Newton method fields the batch path reads, src/nonlinear/newton.jl:138-250, with
// Backtracking (src/globalization/backtracking.jl:28-48), Static (static.jl:8-20),
// Refinement (src/nonlinear/refinement.jl:27-47) and LevenbergMarquardt
// (src/globalization/levenbergmarquardt.jl:48-98).
struct Meth {
    bool qr = false, f32 = false, refine = false;
    int refine_maxiter = 5;
    double refine_eta = 1.4901161193847656e-08;
    int glob = G_BACKTRACKING;
    double static_alpha = 1.0, bt_c1 = 1e-4, bt_p = 0.5;
    int bt_maxiter = 100;
    double mu0 = 1e-6, mu_min = 1e-15, mu_max = 1e12, mu_decrease = 1.0 / 3.0, mu_increase = 4.0,
           rho_accept = 0.0;
    int reuse = 0;            // Newton(reuse = k), k >= 1; 0: nothing
    double dl_radius = 0.0;   // DogLeg(radius); 0: nothing (the first step sets it)
};

// SolverStatus{Float64}, src/base/status.jl:101-117 (counts of calls are 0 for these methods).
struct Status {
    int code = SUCCESS, iterations = 0;
    double fnorm = 0, stepnorm = 0;
    int step_failures = 0;
    bool promoted = false, stationary = false;
    int rank = -1;
    double nullnorm = kNaN, gradratio = kNaN, rate = kNaN;
    bool contracted = false, reused = false;
};

// StepInfo{Float64}, src/base/status.jl:220-234.
struct StepInfo {
    int code;
    double fnorm, stepnorm;
    int failures;
    bool promoted, limited, shortened;
};

// NewtonDiagnostics, src/nonlinear/newton.jl:687-697.
struct Diag {
    int rank = -1;
    double nullnorm = kNaN, gradratio = kNaN, jnorm = 0.0;
};

// The value part of NewtonState that an R1 solve reads (src/nonlinear/newton.jl:715-734):
// the damping (LM rule state), the line-search anchor merit, the residual norm, the
// diagnostics, and the mixed-precision flags.
struct State {
    // FactorAge, src/nonlinear/newton.jl:621-625: the age of the held factor, whether the last
    // step stalled (or stepped along a reused factor at a rate >= 1), whether it stepped along a
    // factor an earlier step formed
    int age = 0;
    bool stalled = false, reused = false;
    // TrustRadius, newton.jl:637-640: DogLeg's radius (0 while unset)
    double radius = 0.0;
    double mu = kNaN;
    double merit = kNaN;  // NaN where the globalization carries `nothing`
    double fnorm = kNaN;
    Diag diag;
    bool promoted = false;
    int slow_steps = 0;
};

// record(status, info), src/base/status.jl:245-262.
inline Status record(const Status& s, const StepInfo& i) {
    Status r = s;
    r.rate = s.stepnorm > 0 ? i.stepnorm / s.stepnorm : kNaN;
    r.code = i.code;
    r.iterations = s.iterations + 1;
    r.fnorm = i.fnorm;
    r.stepnorm = i.stepnorm;
    r.step_failures = s.step_failures + i.failures;
    r.promoted = s.promoted || i.promoted;
    return r;
}

// closing_status, src/nonlinear/solver.jl:88-98 and 111-112.
inline Status closing(const Status& s, int code, bool stationary, bool contracted) {
    Status r = s;
    r.code = code;
    r.stationary = stationary;
    r.rank = -1;
    r.nullnorm = kNaN;
    r.gradratio = kNaN;
    r.contracted = contracted;
    r.reused = false;
    return r;
}

// discarded_step_status, src/nonlinear/solver.jl:103-109.
inline Status discarded(const Status& k, const Status& s) {
    Status r = k;
    r.code = SUCCESS;
    r.step_failures = s.step_failures;
    r.promoted = s.promoted;
    r.stationary = true;
    r.rank = -1;
    r.nullnorm = kNaN;
    r.gradratio = kNaN;
    r.contracted = false;
    r.reused = false;
    return r;
}

// The stopping tests, src/base/options.jl:267-307.
inline bool residual_converged(const Opts& o, const Status& s, double ftest, double ftest0) {
    if (!(s.iterations >= o.min_iterations)) return false;
    return ftest <= jmax(o.f_abstol, o.f_reltol * ftest0);
}
inline bool step_converged(const Opts& o, const Status& s, double xnorm) {
    if (!(s.iterations >= o.min_iterations)) return false;
    return s.iterations > 0 && s.stepnorm > 0 &&
           s.stepnorm <= jmax(o.x_abstol, o.x_reltol * xnorm);
}
inline bool rate_converged(const Opts& o, const Status& s, double theta_prev, double xnorm) {
    if (!o.rate_test) return false;
    if (!(s.iterations >= o.min_iterations)) return false;
    double th = jmax(s.rate, theta_prev);
    if (!(s.stepnorm > 0 && th < 1.0)) return false;
    return th / (1.0 - th) * s.stepnorm <= o.kappa * jmax(o.x_abstol, o.x_reltol * xnorm);
}
inline bool roundoff_stop(const Opts& o, const Status& s, double theta_prev) {
    if (!o.roundoff) return false;
    if (!(s.iterations >= o.min_iterations)) return false;
    return s.rate >= 1.0 && theta_prev < 1.0;
}

// ─── line search, src/globalization/linesearch.jl and backtracking.jl ──────────────────────

struct LSResult {
    double alpha, phi;
    int code, evals;
};

// roundoff(φ₀) = max(4 eps |φ₀|, 4 nextfloat(0)). linesearch.jl:214.
inline double ls_roundoff(double phi0) {
    return jmax(4.0 * kEps * std::fabs(phi0), 4.0 * std::numeric_limits<double>::denorm_min());
}
// smallest_step, linesearch.jl:223.
inline double smallest_step(double d0, double tau) {
    return jmax(tau / std::fabs(d0), kFloatmin);
}
// sufficient_decrease, linesearch.jl:234.
inline bool sufficient_decrease(double pa, double p0, double demand, double tau) {
    return pa - p0 <= jmin(0.0, demand + tau);
}
// floor_code and classify, linesearch.jl:243-250.
inline int floor_code(double pa, double p0, double tau) {
    return std::fabs(pa - p0) <= tau ? STALLED : LINESEARCH_FAILED;
}
inline int classify(double pa, double p0, double tau) {
    if (std::isfinite(pa) && pa - p0 < -tau) return SUCCESS;
    return floor_code(pa, p0, tau);
}

// backtrack_step, backtracking.jl:62-82.
inline double backtrack_step(double phi0, double d0, double a, double pa, double ap, double pp,
                             double p) {
    if (!std::isfinite(pa)) return 0.1 * a;
    double an = kNaN;
    double s = std::fabs(d0);
    double r1 = (pa - phi0) / s + a;
    if (!(ap > 0.0)) {
        if (r1 > 0.0) an = (a * a) / (2.0 * r1);
    } else if (std::isfinite(pp) && a != ap) {
        double q1 = r1 / (a * a);
        double q2 = ((pp - phi0) / s + ap) / (ap * ap);
        double A = (q1 - q2) / (a - ap);
        double B = (a * q2 - ap * q1) / (a - ap);
        double disc = B * B + 3.0 * A;
        if (disc >= 0.0) an = B > 0.0 ? 1.0 / (B + std::sqrt(disc)) : (-B + std::sqrt(disc)) / (3.0 * A);
    }
    if (!(std::isfinite(an) && an > 0.0)) an = p * a;
    return jmin(jmax(an, 0.1 * a), p * a);
}

// The Backtracking search along a line function `lf` with merit(α) and slope0(); the entry
// checks of `linesearch` (linesearch.jl:154-171) and the loop of `search`
// (backtracking.jl:96-132). `exact` selects ExactStep (φ′(0) = -2φ₀) over MeasuredSlope.
template <class LF>
inline LSResult backtracking(double c1, double p, int maxiter, LF& lf, bool exact, double phi0,
                             double alpha) {
    const double ceiling = std::numeric_limits<double>::infinity();
    alpha = jmin((alpha > 0.0 && std::isfinite(alpha)) ? alpha : 1.0, ceiling);
    double d0;
    int n;
    if (exact) {
        d0 = -2.0 * phi0;
        n = 0;
    } else {
        d0 = lf.slope0();
        n = 1;
    }
    if (!(std::isfinite(phi0) && std::isfinite(d0) && d0 < 0.0)) {
        int code = (std::isfinite(phi0) && std::isfinite(d0)) ? (d0 > 0.0 ? LINESEARCH_FAILED : STALLED)
                                                               : NONFINITE;
        return {alpha, kNaN, code, n};
    }
    double tau = ls_roundoff(phi0);
    alpha = jmin(jmax(alpha, smallest_step(d0, tau)), ceiling);
    // search
    double amin = smallest_step(d0, tau);
    double aa = alpha, pa = kNaN;
    double ap = kNaN, pp = kNaN;
    int frozen = 0, code = LINESEARCH_FAILED, trips = 0;
    bool done = false;
    const double sqrteps = 1.4901161193847656e-08;
    while (!done && trips < maxiter) {
        ++trips;
        aa = alpha;
        pa = lf.merit(alpha);
        ++n;
        frozen = (pa == phi0 && alpha <= sqrteps) ? frozen + 1 : 0;
        if (sufficient_decrease(pa, phi0, c1 * alpha * d0, tau)) {
            code = classify(pa, phi0, tau);
            done = true;
        } else if (frozen >= 2) {
            code = STALLED;
            done = true;
        } else if (alpha <= amin) {
            code = floor_code(pa, phi0, tau);
            done = true;
        } else {
            double an = std::isfinite(pa) ? backtrack_step(phi0, d0, alpha, pa, ap, pp, p)
                                          : jmin(0.1 * alpha, std::sqrt(alpha) * std::sqrt(amin));
            ap = alpha;
            pp = pa;
            alpha = jmax(an, amin);
        }
    }
    return {aa, pa, code, n};
}

// ─── the solver ─────────────────────────────────────────────────────────────────────────────

// A problem P gives N, M, `lsq`, `analytic_J`, a generic residual `F(x, out)` over double and
// Dual<K>, and `J(x, Jcm)` when `analytic_J`.
template <class P> struct Solver {
    static constexpr int N = P::N, M = P::M;
    const P& prob;
    const Meth& m;
    const Opts& o;
    long f_evals = 0, dual_evals = 0;
    Factor<N, double> held;  // the factor a step with reuse formed, for the steps after it

    Solver(const P& prob_, const Meth& m_, const Opts& o_) : prob(prob_), m(m_), o(o_) {}

    void F(const double* x, double* out) {
        ++f_evals;
        prob.F(x, out);
    }

    // jacobian!!: the problem's J, or one N-partial dual pass (src/ad/forwarddiff_static.jl:
    // 50-65), column-major M x N.
    void jacobian(const double* x, double* J) {
        if constexpr (P::analytic_J) {
            prob.J(x, J);
        } else {
            ++dual_evals;
            Dual<N> xd[N], rd[M];
            for (int j = 0; j < N; ++j) {
                xd[j].v = x[j];
                for (int k = 0; k < N; ++k) xd[j].p[k] = (k == j) ? 1.0 : 0.0;
            }
            prob.F(xd, rd);
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < M; ++i) J[i + j * M] = rd[i].p[j];
        }
    }

    // jvp!!: J(x) v from the problem's J, or one 1-partial dual pass (src/ad/jvp.jl:88-107).
    void jvp(const double* x, const double* v, double* out) {
        if constexpr (P::analytic_J) {
            double J[M * N];
            prob.J(x, J);
            matvec(J, v, out);
        } else {
            ++dual_evals;
            Dual<1> xd[N], rd[M];
            for (int j = 0; j < N; ++j) {
                xd[j].v = x[j];
                xd[j].p[0] = v[j];
            }
            prob.F(xd, rd);
            for (int i = 0; i < M; ++i) out[i] = rd[i].p[0];
        }
    }

    // SMatrix * SVector as a left fold over the columns.
    static void matvec(const double* J, const double* v, double* out) {
        for (int i = 0; i < M; ++i) {
            double s = J[i] * v[0];
            for (int k = 1; k < N; ++k) s = s + J[i + k * M] * v[k];
            out[i] = s;
        }
    }

    // grad_ratio_and_norm, src/nonlinear/newton.jl:1287-1298.
    static void grad_ratio_and_norm(const double* J, const double* Fx, double fnorm, double& gr,
                                    double& jnorm) {
        jnorm = rnorm(J, M * N);
        if (jnorm == 0.0 || fnorm == 0.0) {
            gr = 0.0;
            return;
        }
        double g[N];
        for (int j = 0; j < N; ++j) {
            double s = J[j * M] * Fx[0];
            for (int i = 1; i < M; ++i) s = s + J[i + j * M] * Fx[i];
            g[j] = s;
        }
        double gnorm = rnorm(g, N);
        if (std::isfinite(gnorm) || !(std::isfinite(jnorm) && std::isfinite(fnorm))) {
            gr = gnorm / jnorm / fnorm;
            return;
        }
        int e = jexponent(fnorm);
        double sc = std::ldexp(1.0, -e);
        double Fs[M];
        for (int i = 0; i < M; ++i) Fs[i] = Fx[i] * sc;
        for (int j = 0; j < N; ++j) {
            double s = J[j * M] * Fs[0];
            for (int i = 1; i < M; ++i) s = s + J[i + j * M] * Fs[i];
            g[j] = s;
        }
        gr = rnorm(g, N) / jnorm / std::ldexp(fnorm, -e);
    }

    // residual_norm, src/nonlinear/newton.jl:1274-1278. `has_merit` for a line search.
    double residual_norm(const State& st, const double* Fx) const {
        if (has_merit()) {
            if (std::isfinite(st.merit) && st.merit >= double(M) * kFloatmin)
                return std::sqrt(st.merit);
            return rnorm(Fx, M);
        }
        return std::isnan(st.fnorm) ? rnorm(Fx, M) : st.fnorm;
    }
    bool has_merit() const { return m.glob == G_BACKTRACKING; }

    // The line function along x + α d, src/globalization/linefunction.jl:17-52.
    struct Line {
        Solver* s;
        const double* x;
        const double* d;
        double xt[N], Ft[M];
        double merit(double a) {
            for (int i = 0; i < N; ++i) xt[i] = x[i] + a * d[i];
            s->F(xt, Ft);
            return norm2(Ft, M);
        }
        double slope0() {
            double x0[N], F0[M], Jv[M];
            for (int i = 0; i < N; ++i) x0[i] = x[i] + 0.0 * d[i];
            s->F(x0, F0);
            s->jvp(x0, d, Jv);
            return 2.0 * rdot(F0, Jv, M);
        }
    };

    // globalize_merit!! for a line search (linefunction.jl:159-199) and globalize!! for Static
    // (linefunction.jl:114-131). Updates x, Fx, info and the merit.
    void globalize(double* x, double* Fx, const double* d, bool exact, double& merit,
                   StepInfo& info) {
        if (m.glob == G_STATIC) {
            double s = m.static_alpha;
            double dn = rnorm(d, N);
            double stepnorm = std::fabs(s) * dn;
            if (!std::isfinite(stepnorm)) {
                info = {NONFINITE, rnorm(Fx, M), stepnorm, 0, false, false, false};
                return;
            }
            double xp[N], Fp[M];
            for (int i = 0; i < N; ++i) xp[i] = x[i] + s * d[i];
            F(xp, Fp);
            double fn = rnorm(Fp, M);
            if (!std::isfinite(fn)) {
                info = {NONFINITE, rnorm(Fx, M), stepnorm, 0, false, false, false};
                return;
            }
            std::memcpy(x, xp, sizeof(xp));
            std::memcpy(Fx, Fp, sizeof(Fp));
            info = {SUCCESS, fn, stepnorm, 0, false, false, false};
            return;
        }
        double phi0 = merit;
        double dn = rnorm(d, N);
        if (!std::isfinite(dn)) {
            info = {NONFINITE, rnorm(Fx, M), dn, 0, false, false, false};
            return;
        }
        Line lf{this, x, d, {}, {}};
        LSResult r = backtracking(m.bt_c1, m.bt_p, m.bt_maxiter, lf, exact, phi0, 1.0);
        if (r.code == SUCCESS) {
            for (int i = 0; i < N; ++i) x[i] = x[i] + r.alpha * d[i];
            std::memcpy(Fx, lf.Ft, sizeof(lf.Ft));
            info = {SUCCESS, std::sqrt(r.phi), r.alpha * dn, 0, false, false, r.alpha < 1.0};
            merit = r.phi;
        } else if (r.code == LINESEARCH_FAILED) {
            if (std::isfinite(r.phi) && r.phi < phi0) {
                for (int i = 0; i < N; ++i) x[i] = x[i] + r.alpha * d[i];
                std::memcpy(Fx, lf.Ft, sizeof(lf.Ft));
                info = {LINESEARCH_FAILED, std::sqrt(r.phi), r.alpha * dn, 1, false, false,
                        r.alpha < 1.0};
                merit = r.phi;
            } else {
                info = {LINESEARCH_FAILED, rnorm(Fx, M), 0.0, 1, false, false, false};
            }
        } else if (r.code == STALLED) {
            info = {STALLED, rnorm(Fx, M), 0.0, 0, false, false, false};
        } else {
            info = {NONFINITE, rnorm(Fx, M), 0.0, 0, false, false, false};
        }
    }

    // refine_passes!! with the held Jacobian, src/nonlinear/refinement.jl:211-244. Returns
    // `failed`.
    template <class TF>
    bool refine(double* d, const Factor<N, TF>& fac, const double* J, const double* Fx) {
        double fnorm = rnorm(Fx, M);
        if (fnorm == 0.0) return false;
        if (!std::isfinite(fnorm)) return true;
        double eta = jmax(m.refine_eta, 1.4901161193847656e-08);
        double Jv[N], r[N];
        matvec(J, d, Jv);
        for (int i = 0; i < N; ++i) r[i] = -Fx[i] + -Jv[i];
        double rprev = rnorm(r, N);
        if (!std::isfinite(rprev)) return true;
        if (rprev <= eta * fnorm) return false;
        for (int it = 1; it <= m.refine_maxiter; ++it) {
            double dd[N], dc[N];
            ldiv<N, TF>(fac, r, dd);
            for (int i = 0; i < N; ++i) dc[i] = d[i] + dd[i];
            matvec(J, dc, Jv);
            for (int i = 0; i < N; ++i) r[i] = -Fx[i] + -Jv[i];
            double rc = rnorm(r, N);
            if (!(rc < rprev)) return true;
            std::memcpy(d, dc, sizeof(dc));
            rprev = rc;
            if (rc <= eta * fnorm) return false;
        }
        return true;
    }

    // The plain Newton step (TF == T), src/nonlinear/newton.jl:1679-1688 with newton_factor
    // :1302-1311, newton_globalize :1396-1404 and newton_line :1410-1416.
    void step_plain(State& st, double* x, double* Fx, StepInfo& info) {
        double fnorm = residual_norm(st, Fx);
        double J[M * N];
        jacobian(x, J);
        Diag dg;
        grad_ratio_and_norm(J, Fx, fnorm, dg.gradratio, dg.jnorm);
        Factor<N, double> fac;
        fac.factor(J, m.qr);
        double merit = st.merit;
        if (fac.info() > 0) {
            info = {SINGULAR, rnorm(Fx, M), 0.0, 0, false, false, false};
        } else {
            double d[N];
            ldiv<N, double>(fac, Fx, d);
            for (int i = 0; i < N; ++i) d[i] = -d[i];
            if (m.refine) refine<double>(d, fac, J, Fx);
            bool exact = !m.refine;  // newton_stepkind, newton.jl:1244-1254
            globalize(x, Fx, d, exact, merit, info);
        }
        st.diag = dg;
        st.merit = merit;
        st.fnorm = info.fnorm;
    }

    // The mixed-precision step (TF = Float32), src/nonlinear/newton.jl:1692-1720 with
    // mixed_newton!! :1604-1666, promote_factor!! :1332-1339, linear_residual_ratio :1422-1430
    // and read_mixed_stall :1437-1451.
    void step_mixed(State& st, double* x, double* Fx, StepInfo& info) {
        double fnorm_old = residual_norm(st, Fx);
        const bool was_promoted = st.promoted;
        double J[M * N];
        jacobian(x, J);
        Diag dg;
        grad_ratio_and_norm(J, Fx, fnorm_old, dg.gradratio, dg.jnorm);
        double d[N];
        bool ok = true, exact = true;
        int failures = 0;
        double lin_rel = 0.0;
        bool md_promoted = st.promoted;
        if (st.promoted) {
            Factor<N, double> fac;
            fac.factor(J, m.qr);
            if (fac.info() > 0) {
                ok = false;
            } else {
                ldiv<N, double>(fac, Fx, d);
                for (int i = 0; i < N; ++i) d[i] = -d[i];
                if (m.refine) refine<double>(d, fac, J, Fx);
            }
        } else {
            Factor<N, float> fac;
            fac.factor(J, m.qr);
            bool ref_failed;
            if (fac.info() > 0) {
                ref_failed = true;
            } else {
                ldiv<N, float>(fac, Fx, d);
                for (int i = 0; i < N; ++i) d[i] = -d[i];
                ref_failed = m.refine ? refine<float>(d, fac, J, Fx) : false;
            }
            if (ref_failed || fac.info() > 0) {
                failures += 1;
                Factor<N, double> ft;
                ft.factor(J, m.qr);
                md_promoted = true;
                if (ft.info() > 0) {
                    ok = false;
                } else {
                    ldiv<N, double>(ft, Fx, d);
                    for (int i = 0; i < N; ++i) d[i] = -d[i];
                }
            } else if (!P::lsq) {
                if (fnorm_old == 0.0 || !std::isfinite(fnorm_old)) {
                    lin_rel = 0.0;
                } else {
                    double Jd[N], lin[N];
                    matvec(J, d, Jd);
                    for (int i = 0; i < N; ++i) lin[i] = Fx[i] + Jd[i];
                    lin_rel = rnorm(lin, N) / fnorm_old;
                }
            }
        }
        st.diag = dg;
        if (!ok) {
            st.promoted = md_promoted;
            info = {SINGULAR, rnorm(Fx, M), 0.0, failures, md_promoted, false, false};
            return;  // the state keeps its merit and norm (mixed_step!! returns md.state)
        }
        bool promoted_step = md_promoted && !was_promoted;
        bool exact_step = exact && md_promoted;  // newton_stepkind(.., in_working_T = promoted)
        double merit = st.merit;
        globalize(x, Fx, d, exact_step, merit, info);
        info.failures += failures;
        if (promoted_step) {
            info.promoted = true;
            st.promoted = true;
            st.slow_steps = 0;
        } else if (was_promoted) {
            // the state stays promoted with its slow-step count
        } else {
            const double eta_lin = 1e-4;  // max(sqrt(eps), 1e-4)
            if (info.fnorm > 0.5 * fnorm_old && lin_rel > eta_lin) {
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

    // ─── Levenberg–Marquardt, stacked QR path ──────────────────────────────────────────────

    // lm_qr_factor!, src/globalization/levenbergmarquardt.jl:359-421.
    static void lm_qr_factor(const double* J, const double* Fx, double* R0, double* c0) {
        for (int j = 0; j < N; ++j) {
            c0[j] = -Fx[j];
            for (int i = 0; i < N; ++i) R0[i + j * N] = J[i + j * M];
        }
        for (int j = 0; j < N; ++j)
            for (int i = j + 1; i < N; ++i) {
                double b = R0[i + j * N];
                if (b == 0.0) continue;
                double a = R0[j + j * N];
                double cs, sn, rv;
                givens(a, b, cs, sn, rv);
                R0[j + j * N] = rv;
                R0[i + j * N] = 0.0;
                for (int k = j + 1; k < N; ++k) {
                    double u = R0[j + k * N], v = R0[i + k * N];
                    R0[j + k * N] = cs * u + sn * v;
                    R0[i + k * N] = -sn * u + cs * v;
                }
                double ur = c0[j], vr = c0[i];
                c0[j] = cs * ur + sn * vr;
                c0[i] = -sn * ur + cs * vr;
            }
        for (int i = N; i < M; ++i) {
            double w[N];
            for (int k = 0; k < N; ++k) w[k] = J[i + k * M];
            double wr = -Fx[i];
            for (int k = 0; k < N; ++k) {
                double b = w[k];
                if (b == 0.0) continue;
                double a = R0[k + k * N];
                double cs, sn, rv;
                givens(a, b, cs, sn, rv);
                R0[k + k * N] = rv;
                w[k] = 0.0;
                for (int l = k + 1; l < N; ++l) {
                    double u = R0[k + l * N], v = w[l];
                    R0[k + l * N] = cs * u + sn * v;
                    w[l] = -sn * u + cs * v;
                }
                double ur = c0[k];
                c0[k] = cs * ur + sn * wr;
                wr = -sn * ur + cs * wr;
            }
        }
    }

    // lm_trial for the stacked workspace with D = I (scaling :none): lm_step_damping,
    // lm_damping_ok and lm_qr_solve!, levenbergmarquardt.jl:162-164, 425-482, 575-584.
    bool lm_trial(const double* R0, const double* c0, double mu, double* delta) const {
        double damp = mu < 4.0 * kEps ? 0.0 : mu;
        double sq = std::sqrt(damp);
        if (!std::isfinite(sq) || !std::isfinite(sq * 1.0)) {
            for (int i = 0; i < N; ++i) delta[i] = 0.0;
            return false;
        }
        double R[N * N], c[N], w[N];
        std::memcpy(R, R0, sizeof(R));
        std::memcpy(c, c0, sizeof(c));
        for (int j = 0; j < N; ++j) {
            for (int k = 0; k < N; ++k) w[k] = 0.0;
            w[j] = sq * 1.0;
            double wr = 0.0;
            for (int k = j; k < N; ++k) {
                double b = w[k];
                if (b == 0.0) continue;
                double a = R[k + k * N];
                double cs, sn, rv;
                givens(a, b, cs, sn, rv);
                R[k + k * N] = rv;
                w[k] = 0.0;
                for (int l = k + 1; l < N; ++l) {
                    double u = R[k + l * N], v = w[l];
                    R[k + l * N] = cs * u + sn * v;
                    w[l] = -sn * u + cs * v;
                }
                double ur = c[k];
                c[k] = cs * ur + sn * wr;
                wr = -sn * ur + cs * wr;
            }
        }
        for (int i = 0; i < N; ++i) delta[i] = 0.0;
        for (int i = N - 1; i >= 0; --i) {
            double s = c[i];
            for (int j = i + 1; j < N; ++j) s = s - R[i + j * N] * delta[j];
            double rii = R[i + i * N];
            if (rii == 0.0 || !std::isfinite(rii)) {
                for (int k = 0; k < N; ++k) delta[k] = 0.0;
                return false;
            }
            delta[i] = s / rii;
        }
        for (int i = 0; i < N; ++i)
            if (!std::isfinite(delta[i])) return false;
        return true;
    }

    // lm_newton_factor without an SVD factor: J, its diagnostics. newton.jl:1881-1892.
    void lm_factor(const double* x, const double* Fx, double fnorm, double* J, Diag& dg) {
        jacobian(x, J);
        dg = Diag();
        grad_ratio_and_norm(J, Fx, fnorm, dg.gradratio, dg.jnorm);
    }

    // The LevenbergMarquardt step, src/nonlinear/newton.jl:1897-1971.
    void step_lm(State& st, double* x, double* Fx, StepInfo& info) {
        double fnorm = rnorm(Fx, M);
        double mu = st.mu;
        if (!std::isfinite(mu)) {
            info = {NONFINITE, fnorm, 0.0, 0, false, false, false};
            return;
        }
        if (fnorm == 0.0) {
            info = {SUCCESS, 0.0, 0.0, 0, false, false, false};
            return;
        }
        double mu_min_eff = jmax(m.mu_min, 4.0 * kEps);
        double J[M * N];
        Diag dg;
        lm_factor(x, Fx, fnorm, J, dg);
        st.diag = dg;
        for (int i = 0; i < M * N; ++i)
            if (!std::isfinite(J[i])) {
                info = {NONFINITE, fnorm, 0.0, 0, false, false, false};
                return;
            }
        double R0[N * N], c0[N];
        lm_qr_factor(J, Fx, R0, c0);
        int failures = 0;
        while (true) {
            double delta[N];
            bool ok = lm_trial(R0, c0, mu, delta);
            if (ok) {
                double Jd[M];
                matvec(J, delta, Jd);
                double pred = -2.0 * rdot(Fx, Jd, M) - norm2(Jd, M);
                if (pred <= 0.0) {
                    double Fl[M];
                    for (int i = 0; i < M; ++i) Fl[i] = 1.0 * Fx[i] + 1.0 * Jd[i];
                    double fl = rnorm(Fl, M);
                    pred = (fnorm - fl) * (fnorm + fl);
                }
                double xp[N], Fp[M];
                for (int i = 0; i < N; ++i) xp[i] = x[i] + 1.0 * delta[i];
                F(xp, Fp);
                double fnp = rnorm(Fp, M);
                if (std::isfinite(fnp) && pred > 0.0) {
                    double ared = (fnorm - fnp) * (fnorm + fnp);
                    double rho = ared / pred;
                    if (rho > m.rho_accept) {
                        bool limited = mu > m.mu0;
                        double mu_next = jmax(mu * m.mu_decrease, mu_min_eff);
                        double stepnorm = rnorm(delta, N);
                        std::memcpy(x, xp, sizeof(xp));
                        std::memcpy(Fx, Fp, sizeof(Fp));
                        st.fnorm = fnp;
                        st.mu = mu_next;
                        info = {SUCCESS, fnp, stepnorm, failures, false, limited, false};
                        return;
                    }
                }
            }
            failures += 1;
            mu = jmax(mu * m.mu_increase, mu_min_eff);
            if (!std::isfinite(mu) || mu > m.mu_max) {
                st.mu = jmin(mu, kFloatmax);
                info = {STALLED, fnorm, 0.0, failures, false, false, false};
                return;
            }
        }
    }

    void step(State& st, double* x, double* Fx, StepInfo& info) {
        if (m.glob == G_LM) step_lm(st, x, Fx, info);
        else if (m.glob == G_DOGLEG) step_dogleg(st, x, Fx, info);
        else if (m.reuse > 0) step_reuse(st, x, Fx, info);
        else if (m.f32) step_mixed(st, x, Fx, info);
        else step_plain(st, x, Fx, info);
    }

    // newton_step!! with reuse = k (Float64 factor, no refinement), src/nonlinear/newton.jl:
    // 1783-1820: while the held factor is younger than k steps and the last step did not stall,
    // the step solves with it and searches along that direction with the measured slope; a
    // search that fails without a step is taken again, in the same step, from a fresh factor at
    // the same point. The rule state after the step follows reuse_result (:1811-1820).
    void step_reuse(State& st, double* x, double* Fx, StepInfo& info) {
        const int age_fresh = m.reuse == 1 ? 0 : 1;  // fresh_age, newton.jl:629
        if (!(st.age == 0 || st.stalled)) {
            const int age_next = st.age + 1 >= m.reuse ? 0 : st.age + 1;  // next_age, :632-633
            double d[N];
            ldiv_same<N>(held, Fx, d);
            for (int i = 0; i < N; ++i) d[i] = -d[i];
            double xr[N], Fr[M];
            std::memcpy(xr, x, sizeof(xr));
            std::memcpy(Fr, Fx, sizeof(Fr));
            double merit = st.merit;
            StepInfo ri;
            globalize(xr, Fr, d, false, merit, ri);  // newton_line with fresh = false
            if (!(ri.code == LINESEARCH_FAILED && ri.stepnorm == 0.0)) {
                std::memcpy(x, xr, sizeof(xr));
                std::memcpy(Fx, Fr, sizeof(Fr));
                info = ri;
                st.merit = merit;
                st.fnorm = info.fnorm;
                st.reused = true;
                st.age = ri.code == SINGULAR ? 0 : age_next;
                st.stalled = ri.code != SINGULAR && ri.code == STALLED;
                return;
            }
        }
        // a fresh factor (newton_factor, newton_globalize), kept for the steps after this one
        double fnorm = residual_norm(st, Fx);
        double J[M * N];
        jacobian(x, J);
        Diag dg;
        grad_ratio_and_norm(J, Fx, fnorm, dg.gradratio, dg.jnorm);
        held.factor(J, m.qr);
        double merit = st.merit;
        if (held.info() > 0) {
            info = {SINGULAR, rnorm(Fx, M), 0.0, 0, false, false, false};
        } else {
            double d[N];
            ldiv_same<N>(held, Fx, d);
            for (int i = 0; i < N; ++i) d[i] = -d[i];
            globalize(x, Fx, d, true, merit, info);
        }
        st.diag = dg;
        st.merit = merit;
        st.fnorm = info.fnorm;
        st.reused = false;
        st.age = info.code == SINGULAR ? 0 : age_fresh;
        st.stalled = info.code != SINGULAR && info.code == STALLED;
    }

    // newton_step!! with DogLeg, src/nonlinear/newton.jl:1725-1747: one Jacobian, one factor, the
    // Newton direction (none when the factor fails or its norm is zero or not finite), then the
    // trial loop of dogleg_step on the Jacobian.
    void step_dogleg(State& st, double* x, double* Fx, StepInfo& info) {
        double fnorm = residual_norm(st, Fx);
        double J[M * N];
        jacobian(x, J);
        Diag dg;
        grad_ratio_and_norm(J, Fx, fnorm, dg.gradratio, dg.jnorm);
        Factor<N, double> fac;
        fac.factor(J, m.qr);
        double d[N];
        bool newton = false;
        if (fac.info() == 0) {  // dogleg_direction, :1751-1756
            ldiv_same<N>(fac, Fx, d);
            for (int i = 0; i < N; ++i) d[i] = -d[i];
            const double nd = rnorm(d, N);
            newton = std::isfinite(nd) && nd != 0.0;
        }
        dogleg_step(x, Fx, J, d, newton, st.radius, info);
        st.diag = dg;
        st.fnorm = info.fnorm;
    }

    // dogleg_step, src/globalization/dogleg.jl:113-215 (Procedure 4.1 of Pawlowski, Simonis,
    // Walker and Shadid 2008): the Newton step inside the radius, else the Cauchy point cut to it,
    // else the point of norm delta on the segment between them; a trial is accepted when
    // pred = |F| - |F + J s| > 0 and ared = |F| - |F(x + s)| >= 1e-4 pred.
    void dogleg_step(double* x, double* Fx, const double* J, const double* sN, bool newton,
                     double& delta, StepInfo& info) {
        const double lo = 1e-6, hi = 1e10;
        const double fnorm = rnorm(Fx, M);
        if (fnorm == 0.0) {
            info = {SUCCESS, fnorm, 0.0, 0, false, false, false};
            return;
        }
        const double nN = newton ? rnorm(sN, N) : HUGE_VAL;
        const double inv_f = 1.0 / fnorm;
        double u[M], gt[N], gh[N], Jg[M];
        for (int i = 0; i < M; ++i) u[i] = inv_f * Fx[i];
        for (int j = 0; j < N; ++j) {  // J' u, a left fold down each column
            double t = J[j * M] * u[0];
            for (int i = 1; i < M; ++i) t = t + J[i + j * M] * u[i];
            gt[j] = t;
        }
        const double gnorm = rnorm(gt, N);
        const double inv_g = 1.0 / gnorm;
        for (int j = 0; j < N; ++j) gh[j] = inv_g * gt[j];
        matvec(J, gh, Jg);
        const double jnorm = rnorm(Jg, M);
        const bool cauchy = gnorm != 0.0 && std::isfinite(gnorm) && jnorm != 0.0 &&
                            std::isfinite(jnorm);
        const double nC = fnorm * ((gnorm / jnorm) / jnorm);
        if (delta == 0.0 && (newton || cauchy)) {
            const double n0 = newton ? nN : nC;
            delta = n0 < lo ? 2.0 * lo : jmin(jmax(n0, lo), hi);  // clamp, dogleg.jl:64
        }
        while (true) {
            double s[N];
            bool boundary;
            if (newton && nN <= delta) {
                std::memcpy(s, sN, sizeof(s));
                boundary = nN >= delta;
            } else if (!cauchy) {
                info = {STALLED, fnorm, 0.0, 0, false, false, false};
                return;
            } else if (!newton || nC >= delta) {
                const double a = -jmin(nC, delta);
                for (int j = 0; j < N; ++j) s[j] = a * gh[j];
                boundary = nC >= delta;
            } else {
                double a[N], b[N];
                const double ca = -(nC / delta);
                for (int j = 0; j < N; ++j) a[j] = ca * gh[j];
                for (int j = 0; j < N; ++j) b[j] = 1.0 * sN[j] + nC * gh[j];
                const double inv_b = 1.0 / rnorm(b, N);
                for (int j = 0; j < N; ++j) b[j] = inv_b * b[j];
                const double ab = rdot(a, b, N);
                const double c = 1.0 - norm2(a, N);
                const double ab2 = ab * ab;
                const double t = c / (ab + std::sqrt(ab2 + c));
                const double dt = delta * t;
                for (int j = 0; j < N; ++j) s[j] = delta * a[j] + dt * b[j];
                boundary = true;
            }
            double Js[M], Flin[M];
            matvec(J, s, Js);
            for (int i = 0; i < M; ++i) Flin[i] = 1.0 * Fx[i] + 1.0 * Js[i];
            const double pred = fnorm - rnorm(Flin, M);
            double xp[N], Fp[M];
            for (int j = 0; j < N; ++j) xp[j] = x[j] + 1.0 * s[j];
            F(xp, Fp);
            const double fnp = rnorm(Fp, M);
            const double ared = fnorm - fnp;
            if (pred > 0.0 && ared >= 1e-4 * pred) {
                const bool limited = !(newton && nN <= delta);
                const double rho = ared / pred;
                if (rho < 0.1) delta = nN < delta ? jmax(nN, lo) : jmax(0.25 * delta, lo);
                else if (rho > 0.75 && boundary) delta = jmin(4.0 * delta, hi);
                const double stepnorm = rnorm(s, N);
                std::memcpy(x, xp, sizeof(xp));
                std::memcpy(Fx, Fp, sizeof(Fp));
                info = {SUCCESS, fnp, stepnorm, 0, false, limited, false};
                return;
            }
            if (delta == lo) {
                info = {LINESEARCH_FAILED, fnorm, 0.0, 1, false, false, false};
                return;
            }
            delta = jmax(0.25 * delta, lo);
        }
    }

    // stationary_converged, src/nonlinear/solver.jl:148-158.
    bool stationary_converged(const State& st, const Status& s) const {
        if constexpr (!P::lsq) return false;
        if (!(s.iterations >= o.min_iterations)) return false;
        return st.diag.jnorm > 0.0 && s.fnorm > 0.0 && st.diag.gradratio <= o.g_tol;
    }

    // refresh_diagnostics!!, src/nonlinear/newton.jl:807-822 (LSQ only).
    void refresh(State& st, const double* x, const double* Fx) {
        if constexpr (P::lsq) {
            double J[M * N];
            Diag dg;
            lm_factor(x, Fx, rnorm(Fx, M), J, dg);
            st.diag = dg;
        }
    }

    // finish!! = newton_finish!!: the diagnostics of the last factorisation into the status.
    // src/nonlinear/newton.jl:1165-1184.
    // newton_finish!!, src/nonlinear/newton.jl:1169-1191: the diagnostics of the last
    // factorisation and, under reuse, whether the last step stepped along a reused factor.
    Status finish(const State& st, const Status& s) const {
        Status r = s;
        r.rank = st.diag.rank;
        r.nullnorm = st.diag.nullnorm;
        r.gradratio = st.diag.gradratio;
        r.reused = m.reuse > 0 && st.reused && s.iterations > 0;
        return r;
    }

    double ftest(const double* Fx, double fnorm) const {
        return o.maxnorm ? rmaxnorm(Fx, M) : fnorm;
    }

    // solve!!, src/nonlinear/solver.jl:277-378.
    Status solve(double* x) {
        double Fx[M];
        F(x, Fx);
        double fnorm0 = rnorm(Fx, M);
        State st;
        st.mu = m.mu0;                                      // reset_rule, newton.jl:678-680
        st.merit = has_merit() ? norm2(Fx, M) : kNaN;      // start_merit, linefunction.jl:85
        st.fnorm = fnorm0;
        st.promoted = false;
        st.slow_steps = 0;
        st.diag = Diag();
        st.age = 0;                 // reset_rule: FactorAge(0, false, false)
        st.stalled = false;
        st.reused = false;
        st.radius = m.dl_radius;    // reset_rule: TrustRadius(radius0, radius0)
        Status s0;
        s0.code = SUCCESS;
        s0.fnorm = fnorm0;
        if (!std::isfinite(fnorm0)) return finish(st, closing(s0, NONFINITE, false, false));
        Status status = s0;
        double ftest0 = ftest(Fx, fnorm0);
        if (residual_converged(o, status, ftest0, ftest0)) return finish(st, status);
        if (o.max_iterations == 0) return finish(st, closing(status, MAXITERS, false, false));
        int stalls = 0;
        double xk[N], Fk[M];
        while (true) {
            std::memcpy(xk, x, sizeof(xk));
            std::memcpy(Fk, Fx, sizeof(Fk));
            Status status_k = status;
            StepInfo info;
            step(st, x, Fx, info);
            status = record(status, info);
            // observe_rate!!, newton.jl:1205-1210: a step along a reused factor at a rate >= 1
            // refreshes the factor at the next step (a NaN rate refreshes nothing)
            if (m.reuse > 0 && st.reused && status.rate >= 1.0) st.stalled = true;
            State st_step = st;
            if (info.code == SINGULAR || info.code == NONFINITE || info.code == MAXITERS)
                return finish(st, status);
            if (info.code == LINESEARCH_FAILED && info.stepnorm == 0.0 &&
                !stationary_converged(st, status))
                return finish(st, status);
            if (residual_converged(o, status, ftest(Fx, status.fnorm), ftest0))
                return finish(st, closing(status, SUCCESS, false, false));
            bool refreshed = false;
            if (stationary_converged(st, status)) {
                refresh(st, x, Fx);
                refreshed = true;
                if (stationary_converged(st, status))
                    return finish(st, closing(status, SUCCESS, true, false));
                // keeps_step_start, solver.jl:183-189
                if (P::lsq && status_k.iterations >= 1 && status.fnorm >= status_k.fnorm &&
                    stationary_converged(st_step, status_k)) {
                    std::memcpy(x, xk, sizeof(xk));
                    std::memcpy(Fx, Fk, sizeof(Fk));
                    return finish(st_step, discarded(status_k, status));
                }
            }
            bool steptested = !(info.code == STALLED || info.limited);
            double xnorm = steptested ? rnorm(x, N) : kNaN;
            bool contracted = !info.shortened && rate_converged(o, status, status_k.rate, xnorm);
            if (contracted ||
                (steptested &&
                 (step_converged(o, status, xnorm) ||
                  (info.code == SUCCESS && info.stepnorm == 0.0 &&
                   status.iterations >= o.min_iterations) ||
                  roundoff_stop(o, status, status_k.rate)))) {
                if (!refreshed) refresh(st, x, Fx);
                if (stationary_converged(st, status))
                    return finish(st, closing(status, SUCCESS, true, false));
                if (contracted) return finish(st, closing(status, SUCCESS, false, true));
                return finish(st, closing(status, STALLED, false, false));
            }
            if (info.code == STALLED) {
                stalls += 1;
                if (stalls >= o.max_stalls) return finish(st, closing(status, STALLED, false, false));
            } else {
                stalls = 0;
            }
            if (status.iterations >= o.max_iterations)
                return finish(st, closing(status, MAXITERS, false, false));
        }
    }
};

}  // namespace orc
