"""The warp form (n = 12 ... 32, one team of 16 or 32 lanes per system) against the oracle.

Each team folds its distributed vectors in index order, so under unfused arithmetic the results
equal the oracle's bit for bit, as the one-thread kernels' do; under fused arithmetic codes and
iteration counts are equal and the solutions agree to 1e-10.
"""

import numpy as np
import pytest

from test_gpu_parity import OPTS, check_parity, run_gpu
from workloads import cubic_affine, cubic_affine_illcond, cubic_affine_pivoting, rng

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


def _hostile(n, nsys=768):
    """Cubic-affine systems that reach every branch of the factor: integer-valued A (ties in the
    pivot search, exact zeros), a zero row (singular at the first column), two equal rows
    (singular at a later column), rows scaled by 2^-600 and 2^+500 (the factor's exponent
    scaling), and starts with a NaN or an Inf entry."""
    g = rng(60 + n)
    A = np.round(g.normal(0.0, 1.5, (nsys, n, n)))
    A[:, np.arange(n), np.arange(n)] += np.where(g.random((nsys, n)) < 0.5, 0.0, n / 4)
    b = np.round(g.uniform(-2.0, 2.0, (nsys, n)))
    X0 = np.zeros((nsys, n))
    kind = np.arange(nsys) % 6
    rows = g.integers(0, n, (nsys, 2))
    for s in np.flatnonzero(kind == 1):
        A[s, rows[s, 0], :] = 0.0
    for s in np.flatnonzero(kind == 2):
        if rows[s, 0] != rows[s, 1]:
            A[s, rows[s, 1], :] = A[s, rows[s, 0], :]
    A[kind == 3] *= 2.0 ** -600
    b[kind == 3] *= 2.0 ** -600
    A[kind == 4] *= 2.0 ** 500
    X0[kind == 5, 0] = np.where(np.arange((kind == 5).sum()) % 2 == 0, np.nan, np.inf)
    P = np.concatenate([A.transpose(0, 2, 1).reshape(nsys, n * n), b], axis=1)
    return X0, np.ascontiguousarray(P)


def _same_statuses(sg, so):
    """Every status field bit for bit, except that a NaN equals any NaN: a residual norm made
    from an Inf start (Inf - Inf) is the device's NaN, whose sign bit differs from the x86 one
    the oracle's arithmetic makes."""
    for name in sg.dtype.names:
        a, b = sg[name], so[name]
        if a.dtype.kind == "f":
            same = (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))
            assert same.all(), f"{name} differs at {np.flatnonzero(~same)[:8]}"
        else:
            assert np.array_equal(a, b), f"{name} differs at {np.flatnonzero(a != b)[:8]}"


@pytest.mark.parametrize("n", SIZES)
def test_warp_ties_singular_and_scaling(gsb, oracle, n):
    X0, P = _hostile(n)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    opts = gsb.Options(**OPTS)
    for lin in (gsb.LUFactorization(), gsb.LUFactorization("float32")):
        m = gsb.Newton(linsolve=lin, globalization=gsb.Backtracking(), arithmetic="unfused")
        xg, sg = run_gpu(gsb, prob, m, X0, P, opts)
        xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
        assert xg.tobytes() == xo.tobytes()
        _same_statuses(sg, np.ascontiguousarray(so))
        # every kind of system is present: successes, singular factors, non-finite starts
        assert {0, 3, 4} <= set(np.unique(so["code"]).tolist())
