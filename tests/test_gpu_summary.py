"""The batch summary fused into the solve (gsb_solve_batch_summary) against batch_summary(S) of
the same statuses (src/nonlinear/batched.jl:63-89): the counts exactly, |F| to the rounding of
the accumulation order (the partial sums meet in atomics), on the one-thread, warp-form and
least-squares kernels, with NaN statuses and with fnorms whose squares underflow (rnorm's scaled
second pass)."""

import numpy as np
import pytest

from workloads import c2, cubic_affine

FN_TOL = 1e-12


def _both(gsb, prob, m, X0, P, opts):
    import torch

    X = torch.tensor(X0, device="cuda")
    S = gsb.status_buffer(X0.shape[0])
    _, fused = gsb.solve_batch_summary(X, S, prob, m, gsb.PerSystem(torch.tensor(P, device="cuda")),
                                       options=opts)
    return fused, gsb.batch_summary(S)


def _same(fused, ref):
    assert fused.failure_count == ref.failure_count
    assert fused.all_converged == ref.all_converged
    assert fused.max_iterations == ref.max_iterations
    assert fused.total_iterations == ref.total_iterations
    if np.isnan(ref.fnorm):
        assert np.isnan(fused.fnorm)
    else:
        assert abs(fused.fnorm - ref.fnorm) <= FN_TOL * abs(ref.fnorm), (fused.fnorm, ref.fnorm)


@pytest.mark.gpu
@pytest.mark.parametrize("n,nsys", [(8, 65536), (3, 10000), (16, 4096)])
def test_fused_summary_matches(gsb, n, nsys):
    X0, P = cubic_affine(n, nsys, n + 1.0, 70 + n)
    opts = gsb.Options(f_abstol=1e-12, f_reltol=0.0, max_iterations=3)  # some MAXITERS
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    m = gsb.Newton(globalization=gsb.Backtracking())
    fused, ref = _both(gsb, prob, m, X0, P, opts)
    _same(fused, ref)
    assert ref.total_iterations > 0


@pytest.mark.gpu
def test_fused_summary_nan_and_underflow(gsb):
    import torch

    prob = gsb.NonlinearProblem(gsb.Hetero6())
    X0 = np.array([[2.5, 3.5]] * 8)
    P = np.array([1, 2, 3, 4, 5, 6, 1, 3], float)[:, None]
    fused, ref = _both(gsb, prob, gsb.Newton(globalization=gsb.Backtracking()), X0, P,
                       gsb.Options(max_iterations=3))
    _same(fused, ref)
    assert np.isnan(fused.fnorm) and fused.failure_count == 6
    # residuals near 1e-170 at x0: converged at the start, their squares underflow
    X0, P = cubic_affine(4, 4096, 5.0, 77)
    P[:, 16:] *= 1e-170
    fused, ref = _both(gsb, gsb.NonlinearProblem(gsb.CubicAffine(4)),
                       gsb.Newton(globalization=gsb.Backtracking()), X0, P,
                       gsb.Options(f_abstol=1e-12, f_reltol=0.0))
    _same(fused, ref)
    assert 0.0 < fused.fnorm < 1e-160 and fused.total_iterations == 0


@pytest.mark.gpu
def test_fused_summary_least_squares(gsb):
    X0, Y, t = c2(2048)
    prob = gsb.LeastSquaresProblem(gsb.ExpSum3(t))
    m = gsb.Newton(linsolve=gsb.QRFactorization(), globalization=gsb.LevenbergMarquardt())
    fused, ref = _both(gsb, prob, m, X0, Y, gsb.Options(f_abstol=1e-12, f_reltol=0.0,
                                                        max_iterations=50))
    _same(fused, ref)
