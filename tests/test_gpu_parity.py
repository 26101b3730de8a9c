"""Parity of the device batch (libgsb, through the C-ABI) with the oracle, system by system.

The bar (the batch's own contract): identical status codes, identical iteration counts, and
per-system ‖x - x_ref‖∞ / ‖x_ref‖∞ ≤ 1e-10 for the default fused arithmetic; every status and
iterate bit for bit under the unfused arithmetic, which rounds like the CPU restatement.
"""

import numpy as np
import pytest

from workloads import cubic_affine_illcond, c0, c1, cubic_affine, cubic_affine_pivoting

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10
NAMES = ["SUCCESS", "STALLED", "MAXITERS", "SINGULAR", "NONFINITE", "LINESEARCH_FAILED"]


def _dev(a):
    import torch

    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def run_gpu(gsb, prob, method, X0, P, options, order=None, soa=False):
    import torch

    X = _dev(X0.T if soa else X0)
    Pd = _dev(P.T if soa else P)
    S = gsb.status_buffer(X0.shape[0])
    kw = {}
    if order is not None:
        kw["order"] = torch.tensor(order, dtype=torch.int64, device="cuda")
    gsb.solve_batch(gsb.SoA(X) if soa else X, S, prob,
                    method, gsb.PerSystem(gsb.SoA(Pd) if soa else Pd), options=options, **kw)
    x = X.cpu().numpy()
    return (x.T if soa else x), gsb.statuses(S)


def rel_err(x, xr):
    num = np.max(np.abs(x - xr), axis=1)
    den = np.max(np.abs(xr), axis=1)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(den > 0, num / den, num)


def check_parity(xg, sg, xo, so, bitwise, iterations=True):
    bad = np.flatnonzero(sg["code"] != so["code"])
    assert bad.size == 0, f"codes differ at {bad[:8]}: {sg['code'][bad[:8]]} vs {so['code'][bad[:8]]}"
    if iterations:
        bad = np.flatnonzero(sg["iterations"] != so["iterations"])
        assert bad.size == 0, f"iterations differ at {bad[:8]}"
        assert np.array_equal(sg["step_failures"], so["step_failures"])
        assert np.array_equal(sg["promoted"], so["promoted"])
    ok = so["code"] == 0
    assert np.all(rel_err(xg[ok], xo[ok]) <= REL_TOL)
    if bitwise:
        assert xg.tobytes() == xo.tobytes()
        assert sg.tobytes() == so.tobytes()


OPTS = dict(f_abstol=1e-12, f_reltol=0.0, max_iterations=50)


@pytest.mark.parametrize("arith", ["fused", "unfused"])
@pytest.mark.parametrize("cfg", ["c0", "c1"])
def test_plain_fp64_parity(gsb, oracle, cfg, arith):
    n = 3 if cfg == "c0" else 8
    X0, P = c0() if cfg == "c0" else c1(262144)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    m = gsb.Newton(globalization=gsb.Backtracking(), arithmetic=arith)
    opts = gsb.Options(**OPTS)
    xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    check_parity(xg, sg, xo, so, bitwise=(arith == "unfused"))
    assert np.all(so["code"] == 0)


def test_plain_fp64_full_c1(gsb, oracle):
    # the full configuration: 1,048,576 systems of n = 8
    X0, P = c1()
    prob = gsb.NonlinearProblem(gsb.CubicAffine(8))
    m = gsb.Newton(globalization=gsb.Backtracking())
    opts = gsb.Options(**OPTS)
    xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    check_parity(xg, sg, xo, so, bitwise=False)


@pytest.mark.parametrize("arith", ["fused", "unfused"])
def test_mixed_fp32_refinement_parity(gsb, oracle, arith):
    X0, P = c1(131072)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(8))
    m = gsb.Newton(linsolve=gsb.LUFactorization("float32"), refinement=gsb.Refinement(),
                   globalization=gsb.Backtracking(), arithmetic=arith)
    opts = gsb.Options(**OPTS)
    xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    # identical iterations are the contract of the plain FP64 path; the FP32 factor's rounding
    # under fused arithmetic may move a step, so the mixed form is held to its codes and error
    check_parity(xg, sg, xo, so, bitwise=(arith == "unfused"), iterations=(arith == "unfused"))
    # and the FP64-oracle error of the mixed form
    x64, s64 = oracle.solve_batch(prob, gsb.Newton(globalization=gsb.Backtracking()), X0.copy(), P,
                                  opts)
    assert np.array_equal(sg["code"], s64["code"])
    assert np.all(rel_err(xg, x64) <= REL_TOL)


@pytest.mark.parametrize("n", [4, 6, 8])
def test_mixed_promotion(gsb, oracle, n):
    # condition numbers 1e3..1e9: the Float32 factor needs its refinement passes and more than
    # half of the systems are promoted to the Float64 factor (from n = 6 on, the thread-local
    # one), with SUCCESS, MAXITERS, LINESEARCH_FAILED and STALLED among the outcomes
    X0, P = cubic_affine_illcond(n, 8192, 5)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    m = gsb.Newton(linsolve=gsb.LUFactorization("float32"), refinement=gsb.Refinement(),
                   globalization=gsb.Backtracking(), arithmetic="unfused")
    opts = gsb.Options(**OPTS)
    xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    assert so["promoted"].sum() > X0.shape[0] // 3
    assert len(np.unique(so["code"])) >= 3
    check_parity(xg, sg, xo, so, bitwise=True)


@pytest.mark.parametrize("n", [2, 4, 6])
@pytest.mark.parametrize("glob", ["static", "backtracking"])
def test_sizes_and_globalizations(gsb, oracle, n, glob):
    X0, P = cubic_affine(n, 20000, n + 1.0, 4)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    g = gsb.Static() if glob == "static" else gsb.Backtracking()
    for arith in ("fused", "unfused"):
        m = gsb.Newton(globalization=g, arithmetic=arith)
        opts = gsb.Options(**OPTS)
        xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
        xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
        check_parity(xg, sg, xo, so, bitwise=(arith == "unfused"))


@pytest.mark.parametrize("n", [2, 3, 4, 6, 8])
def test_pivoting(gsb, oracle, n):
    # rows of A in random order: the factor exchanges rows at nearly every step
    X0, P = cubic_affine_pivoting(n, 20000, n + 2.0, 6)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    for arith in ("fused", "unfused"):
        for m in (gsb.Newton(globalization=gsb.Backtracking(), arithmetic=arith),
                  gsb.Newton(linsolve=gsb.LUFactorization("float32"), refinement=gsb.Refinement(),
                             globalization=gsb.Backtracking(), arithmetic=arith)):
            opts = gsb.Options(**OPTS)
            xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
            xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
            mixed = m.linsolve.TF is not None
            check_parity(xg, sg, xo, so, bitwise=(arith == "unfused"),
                         iterations=(arith == "unfused" or not mixed))


@pytest.mark.parametrize("n,T", [(6, 2), (8, 2), (8, 4), (8, 8)])
@pytest.mark.parametrize("pivoting", [False, True])
def test_team_parity(gsb, oracle, n, T, pivoting):
    # T lanes per system: identical codes and iterations on the plain path, rel err <= 1e-10
    gen = cubic_affine_pivoting if pivoting else cubic_affine
    X0, P = gen(n, 40000, n - 1.0, 11)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    opts = gsb.Options(**OPTS)
    for mixed in (False, True):
        kw = dict(linsolve=gsb.LUFactorization("float32"), refinement=gsb.Refinement()) if mixed else {}
        m = gsb.Newton(globalization=gsb.Backtracking(), threads_per_system=T, **kw)
        xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
        xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
        check_parity(xg, sg, xo, so, bitwise=False, iterations=not mixed)
    for glob in (gsb.Static(),):
        m = gsb.Newton(globalization=glob, threads_per_system=T)
        xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
        xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
        check_parity(xg, sg, xo, so, bitwise=False)


def test_six_outcomes_and_count_form(gsb, oracle):
    codes = [1, 2, 3, 4, 5, 6, 1, 3]
    X0 = np.array([[2.5, 3.5]] * 8)
    P = np.array(codes, float)[:, None]
    prob = gsb.NonlinearProblem(gsb.Hetero6())
    m = gsb.Newton(globalization=gsb.Backtracking())
    opts = gsb.Options(max_iterations=3)
    xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
    assert [NAMES[c] for c in sg["code"]] == ["SUCCESS", "STALLED", "MAXITERS", "SINGULAR",
                                              "NONFINITE", "LINESEARCH_FAILED", "SUCCESS",
                                              "MAXITERS"]
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    assert sg.tobytes() == so.tobytes() and xg.tobytes() == xo.tobytes()
    X = _dev(X0)
    counts = gsb.solve_batch(X, prob, m, gsb.PerSystem(_dev(P)), max_iterations=3)
    assert counts == gsb.ReturnCodeCounts(2, 1, 2, 1, 1, 1)
    assert not gsb.isconverged(counts)
    assert X.cpu().numpy()[0].tolist() == xg[0].tolist()


def test_exact_root_singular_and_order(gsb, oracle):
    p = np.array([[2.125, 1.5], [1.25, 2.0], [1.5, 2.5], [1.75, 3.0]])
    x0 = np.array([[2.0, 1.0], [2.5, 1.5], [3.5, 2.5], [4.0, 3.0]])
    prob = gsb.NonlinearProblem(gsb.Coupled2())
    exact = gsb.Newton(arithmetic="unfused")
    xg, sg = run_gpu(gsb, prob, exact, x0, p, gsb.Options(max_iterations=150))
    assert xg[0].tolist() == [2.0, 1.0] and sg["iterations"][0] == 0 and sg["code"][0] == 0
    xo, so = oracle.solve_batch(prob, exact, x0.copy(), p, gsb.Options(max_iterations=150))
    assert sg.tobytes() == so.tobytes() and xg.tobytes() == xo.tobytes()
    xf, sf = run_gpu(gsb, prob, gsb.Newton(), x0, p, gsb.Options(max_iterations=150))
    check_parity(xf, sf, xo, so, bitwise=False)
    xgp, sgp = run_gpu(gsb, prob, exact, x0, p, gsb.Options(max_iterations=150),
                       order=[3, 1, 0, 2])
    assert sgp.tobytes() == sg.tobytes() and xgp.tobytes() == xg.tobytes()
    x0s = x0.copy()
    x0s[1] = [4.0, 4.0]
    _, ss = run_gpu(gsb, prob, gsb.Newton(), x0s, p, gsb.Options(max_iterations=60))
    assert [NAMES[c] for c in ss["code"]] == ["SUCCESS", "SINGULAR", "SUCCESS", "SUCCESS"]
    with pytest.raises(gsb.ArgumentError):
        run_gpu(gsb, prob, gsb.Newton(), x0, p, gsb.Options(), order=[0, 0, 1, 2])


def test_soa_layout_and_hostile_inputs(gsb, oracle):
    X0, P = cubic_affine(3, 1000, 4.0, 9)
    X0[0, 0] = np.nan
    X0[1, 1] = np.inf
    X0[2, 2] = 5e-324
    prob = gsb.NonlinearProblem(gsb.CubicAffine(3))
    m = gsb.Newton(globalization=gsb.Backtracking())
    opts = gsb.Options(**OPTS)
    xa, sa = run_gpu(gsb, prob, m, X0, P, opts)
    xs, ss = run_gpu(gsb, prob, m, X0, P, opts, soa=True)
    assert sa.tobytes() == ss.tobytes()
    assert np.array_equal(xa[3:], xs[3:])
    assert sa["code"].tolist()[:3] == [4, 4, 0]
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    check_parity(xa, sa, xo, so, bitwise=False)


def test_batch_summary(gsb, oracle):
    import torch

    X0, P = c0(5000)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(3))
    X = _dev(X0)
    S = gsb.status_buffer(5000)
    gsb.solve_batch(X, S, prob, gsb.Newton(globalization=gsb.Backtracking()),
                    gsb.PerSystem(_dev(P)), **OPTS)
    st = gsb.statuses(S)
    summ = gsb.batch_summary(S)
    assert summ.failure_count == int(np.count_nonzero(st["code"] != 0))
    assert summ.all_converged == (summ.failure_count == 0)
    assert summ.max_iterations == int(st["iterations"].max())
    assert summ.total_iterations == int(st["iterations"].sum())
    assert summ.fnorm == pytest.approx(np.sqrt(np.sum(st["fnorm"] ** 2)), rel=1e-12)
    assert gsb.batch_summary(gsb.status_buffer(0)) == gsb.BatchSummary(0.0, True, 0, 0, 0)
    del torch
