"""The warp form (n = 12 ... 32, one team of 16 or 32 lanes per system) against the oracle.

Each team folds its distributed vectors in index order, so under unfused arithmetic the results
equal the oracle's bit for bit, as the one-thread kernels' do; under fused arithmetic codes and
iteration counts are equal and the solutions agree to 1e-10.
"""

import numpy as np
import pytest

from test_gpu_parity import OPTS, check_parity, run_gpu
from workloads import cubic_affine, cubic_affine_illcond, cubic_affine_pivoting

pytestmark = pytest.mark.gpu

SIZES = [12, 16, 24, 32]


@pytest.mark.parametrize("arith", ["unfused", "fused"])
@pytest.mark.parametrize("n", SIZES)
def test_warp_plain_parity(gsb, oracle, n, arith):
    X0, P = cubic_affine(n, 2048, n + 1.0, 4)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    m = gsb.Newton(globalization=gsb.Backtracking(), arithmetic=arith)
    opts = gsb.Options(**OPTS)
    xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    check_parity(xg, sg, xo, so, bitwise=(arith == "unfused"))
    assert np.all(so["code"] == 0)


@pytest.mark.parametrize("n", SIZES)
def test_warp_pivoting_and_static(gsb, oracle, n):
    # rows in random order: a row exchange in nearly every column; Static and Backtracking
    X0, P = cubic_affine_pivoting(n, 1024, n + 1.0, 4)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    opts = gsb.Options(**OPTS)
    for glob in (gsb.Static(), gsb.Backtracking()):
        m = gsb.Newton(globalization=glob, arithmetic="unfused")
        xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
        xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
        check_parity(xg, sg, xo, so, bitwise=True)


@pytest.mark.parametrize("n", SIZES)
def test_warp_mixed_parity(gsb, oracle, n):
    # the Float32 factor with refinement on well-conditioned systems, then ill-conditioned ones
    # where most systems are promoted to the Float64 factor
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    m = gsb.Newton(linsolve=gsb.LUFactorization("float32"), refinement=gsb.Refinement(),
                   globalization=gsb.Backtracking(), arithmetic="unfused")
    opts = gsb.Options(**OPTS)
    for X0, P in (cubic_affine(n, 1024, n + 1.0, 4), cubic_affine_illcond(n, 1024, 5)):
        xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
        xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
        check_parity(xg, sg, xo, so, bitwise=True)


def test_warp_soa_order(gsb, oracle):
    n = 16
    X0, P = cubic_affine(n, 999, n + 1.0, 4)  # not a multiple of the systems per CTA
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    m = gsb.Newton(globalization=gsb.Backtracking(), arithmetic="unfused")
    opts = gsb.Options(**OPTS)
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    xg, sg = run_gpu(gsb, prob, m, X0, P, opts, soa=True)
    check_parity(xg, sg, xo, so, bitwise=True)
    order = np.random.default_rng(1).permutation(X0.shape[0])
    xg, sg = run_gpu(gsb, prob, m, X0, P, opts, order=order)
    check_parity(xg, sg, xo, so, bitwise=True)
