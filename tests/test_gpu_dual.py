"""Families given by their residual alone: the device takes the Jacobian from one N-partial
forward-mode dual pass and the JVP from a 1-partial pass (src/ad/forwarddiff_static.jl:50-65,
src/ad/jvp.jl:96-107), as the oracle does with its Dual<K>.

- Wood's function with a per-system coupling weight, a family the device knows only by its
  residual: unfused, bit for bit the oracle's solve; fused, within the oracle's own one-ulp
  envelope.
- The cubic-affine family with the dual pass in place of its written-out Jacobian rule: the two
  device solves agree bit for bit, fused and unfused."""

import numpy as np
import pytest

from workloads import cubic_affine, rng


def _solve(gsb, prob, m, X0, P, opts):
    import torch

    X = torch.tensor(X0, device="cuda")
    S = gsb.status_buffer(X0.shape[0])
    gsb.solve_batch(X, S, prob, m, gsb.PerSystem(torch.tensor(P, device="cuda")), options=opts)
    return X.cpu().numpy(), S.cpu().numpy()


def _wood_batch(nsys=8192):
    g = rng(90)
    x0 = np.array([-3.0, -1.0, -3.0, -1.0]) * g.uniform(0.5, 1.5, (nsys, 4))
    w = g.uniform(15.0, 25.0, (nsys, 1))
    return x0, w


@pytest.mark.gpu
@pytest.mark.parametrize("glob", ["backtracking", "static"])
def test_wood_by_residual_alone(gsb, oracle, glob):
    X0, P = _wood_batch()
    prob = gsb.NonlinearProblem(gsb.Wood())
    g = gsb.Backtracking() if glob == "backtracking" else gsb.Static()
    opts = gsb.Options(f_abstol=1e-10, f_reltol=0.0, max_iterations=60)
    m = gsb.Newton(globalization=g, arithmetic="unfused")
    xg, sg = _solve(gsb, prob, m, X0, P, opts)
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    assert np.array_equal(xg.view(np.uint64), xo.view(np.uint64))
    assert np.array_equal(sg, np.ascontiguousarray(so).view(np.uint8).reshape(-1, 72))
    # the batch reaches more than one outcome and takes real steps
    assert (so["iterations"] > 3).mean() > 0.5
    # Fused: Wood's valley makes Newton's path from these starts sensitive to rounding (the
    # oracle's own run from x0 moved by one ulp changes some codes), so the fused batch is held
    # to that envelope, and to the oracle's root where both succeed with the same count.
    mf = gsb.Newton(globalization=g)
    xf, sf = _solve(gsb, prob, mf, X0, P, opts)
    sf = gsb.statuses(sf)
    _, s1 = oracle.solve_batch(prob, m, np.nextafter(X0, np.inf), P, opts)
    env = np.mean(s1["code"] != so["code"])
    assert np.mean(sf["code"] != so["code"]) <= max(3 * env, 0.005)
    both = (sf["code"] == 0) & (so["code"] == 0) & (sf["iterations"] == so["iterations"])
    assert both.sum() >= 0.9 * (so["code"] == 0).sum()
    err = np.max(np.abs(xf - xo), axis=1) / np.max(np.abs(xo), axis=1)
    assert float(err[both].max()) <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 3, 4])
@pytest.mark.parametrize("arith", ["fused", "unfused"])
def test_cubic_rule_equals_dual_pass(gsb, oracle, n, arith):
    X0, P = cubic_affine(n, 8192, n + 1.0, 91 + n)
    X0 = rng(95 + n).uniform(-2.0, 2.0, X0.shape)
    opts = gsb.Options(f_abstol=1e-12, f_reltol=0.0, max_iterations=50)
    m = gsb.Newton(globalization=gsb.Backtracking(), arithmetic=arith)
    xr, sr = _solve(gsb, gsb.NonlinearProblem(gsb.CubicAffine(n)), m, X0, P, opts)
    xd, sd = _solve(gsb, gsb.NonlinearProblem(gsb.CubicAffine(n, jacobian="dual")), m, X0, P, opts)
    assert np.array_equal(xr.view(np.uint64), xd.view(np.uint64))
    assert np.array_equal(sr, sd)
    if arith == "unfused":
        xo, so = oracle.solve_batch(gsb.NonlinearProblem(gsb.CubicAffine(n)), m, X0.copy(), P, opts)
        assert np.array_equal(xd.view(np.uint64), xo.view(np.uint64))
        assert np.array_equal(sd, np.ascontiguousarray(so).view(np.uint8).reshape(-1, 72))


def test_dual_family_checks(gsb):
    with pytest.raises(gsb.ArgumentError):
        gsb.CubicAffine(8, jacobian="dual")
    with pytest.raises(gsb.ArgumentError):
        gsb.CubicAffine(3, jacobian="symbolic")
    assert gsb.Wood().param_count == 1
