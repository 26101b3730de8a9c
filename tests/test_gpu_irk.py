"""The Gauss-3 stage systems of the Hénon–Heiles field (n = 12, the warp form) against the oracle:
bit-identical under unfused arithmetic, codes, iterations and 1e-10 under fused arithmetic."""

import numpy as np
import pytest

from test_gpu_parity import OPTS, check_parity, run_gpu
from workloads import c3

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("arith", ["unfused", "fused"])
def test_irk_parity(gsb, oracle, arith, mixed):
    X0, P = c3(8192)
    prob = gsb.NonlinearProblem(gsb.IrkHenonHeiles(0.1))
    kw = dict(linsolve=gsb.LUFactorization("float32"), refinement=gsb.Refinement()) if mixed else {}
    m = gsb.Newton(globalization=gsb.Backtracking(), arithmetic=arith, **kw)
    opts = gsb.Options(**OPTS)
    xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    check_parity(xg, sg, xo, so, bitwise=(arith == "unfused"),
                 iterations=(arith == "unfused" or not mixed))
    assert np.all(so["code"] == 0)


def test_irk_static_and_perturbed_starts(gsb, oracle):
    # starts away from zero (a step from the solution's neighbourhood) and the Static step
    X0, P = c3(4096)
    prob = gsb.NonlinearProblem(gsb.IrkHenonHeiles(0.1))
    opts = gsb.Options(**OPTS)
    g = np.random.default_rng(7)
    Xs = X0 + 0.02 * g.standard_normal(X0.shape)
    for glob in (gsb.Static(), gsb.Backtracking()):
        m = gsb.Newton(globalization=glob, arithmetic="unfused")
        xg, sg = run_gpu(gsb, prob, m, Xs, P, opts)
        xo, so = oracle.solve_batch(prob, m, Xs.copy(), P, opts)
        check_parity(xg, sg, xo, so, bitwise=True)
