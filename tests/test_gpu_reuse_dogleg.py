"""Newton(reuse = k) and DogLeg in the batch (src/nonlinear/newton.jl:1725-1874,
src/globalization/dogleg.jl:113-215) against the oracle, whose two step rules reproduce the
reference's golden columns "Newton reuse 3 Backtracking LU" and "Newton DogLeg LU"
(tests/test_oracle_pins.py). Unfused arithmetic: the batch is the oracle's bit for bit (iterates
and all 72 status bytes, the `reused` flag included). Fused: the same codes and iteration
counts, iterates within 1e-10."""

import numpy as np
import pytest

from workloads import cubic_affine, cubic_affine_pivoting, rng

REL = 1e-10


def _batches():
    out = []
    for n in (2, 3, 4, 6, 8):
        X0, P = cubic_affine(n, 4096, n + 1.0, 40 + n)
        out.append((f"n{n}", n, X0, P))
        # far starts: the radius and the Cauchy point shape DogLeg's steps, and reused factors
        # are refreshed by stalls and rates >= 1
        g = rng(50 + n)
        out.append((f"n{n}-far", n, g.uniform(-6.0, 6.0, X0.shape), P))
    X0, P = cubic_affine_pivoting(8, 4096, 9.0, 61)
    out.append(("n8-pivoting", 8, rng(62).uniform(-3.0, 3.0, X0.shape), P))
    return out


BATCHES = _batches()


def _methods(gsb, arith):
    return {
        "reuse3": gsb.Newton(globalization=gsb.Backtracking(), reuse=3, arithmetic=arith),
        "reuse1": gsb.Newton(globalization=gsb.Backtracking(), reuse=1, arithmetic=arith),
        "dogleg": gsb.Newton(globalization=gsb.DogLeg(), arithmetic=arith),
        "dogleg-r": gsb.Newton(globalization=gsb.DogLeg(radius=0.05), arithmetic=arith),
    }


def _solve(gsb, n, m, X0, P, opts):
    import torch

    X = torch.tensor(X0, device="cuda")
    S = gsb.status_buffer(X0.shape[0])
    gsb.solve_batch(X, S, gsb.NonlinearProblem(gsb.CubicAffine(n)), m,
                    gsb.PerSystem(torch.tensor(P, device="cuda")), options=opts)
    return X.cpu().numpy(), S.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,X0,P", BATCHES, ids=[b[0] for b in BATCHES])
def test_unfused_bit_for_bit(gsb, oracle, name, n, X0, P):
    opts = gsb.Options(f_abstol=1e-12, f_reltol=0.0, max_iterations=50)
    for mname, m in _methods(gsb, "unfused").items():
        xg, sg = _solve(gsb, n, m, X0, P, opts)
        xo, so = oracle.solve_batch(gsb.NonlinearProblem(gsb.CubicAffine(n)), m, X0.copy(), P, opts)
        so_bytes = np.ascontiguousarray(so).view(np.uint8).reshape(-1, 72)
        assert np.array_equal(xg.view(np.uint64), xo.view(np.uint64)), mname
        assert np.array_equal(sg, so_bytes), mname
        if mname.startswith("reuse") and mname != "reuse1":
            # the batch exercises the rule: some systems end on a reused factor
            assert so["reused"].any() or name.endswith("far"), mname


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,X0,P", BATCHES, ids=[b[0] for b in BATCHES])
def test_fused_codes_iterations_and_roots(gsb, oracle, name, n, X0, P):
    opts = gsb.Options(f_abstol=1e-12, f_reltol=0.0, max_iterations=50)
    for mname, m in _methods(gsb, "fused").items():
        xg, sg = _solve(gsb, n, m, X0, P, opts)
        sg = gsb.statuses(sg)
        xo, so = oracle.solve_batch(gsb.NonlinearProblem(gsb.CubicAffine(n)), m, X0.copy(), P, opts)
        assert np.array_equal(sg["code"], so["code"]), mname
        assert np.array_equal(sg["iterations"], so["iterations"]), mname
        ok = so["code"] == 0
        err = np.max(np.abs(xg - xo), axis=1) / np.maximum(np.max(np.abs(xo), axis=1), 1e-300)
        assert float(err[ok].max(initial=0.0)) <= REL, (mname, float(err[ok].max(initial=0.0)))
        assert np.array_equal(sg["reused"], so["reused"]), mname


@pytest.mark.gpu
def test_six_outcomes_under_both_rules(gsb, oracle):
    """The reference's six-outcome batch (test/nonlinear/batched.jl:54-90) with reuse and DogLeg."""
    import torch

    codes = [1, 2, 3, 4, 5, 6, 1, 3]
    X0 = np.array([[2.5, 3.5]] * 8)
    P = np.array(codes, float)[:, None]
    prob = gsb.NonlinearProblem(gsb.Hetero6())
    opts = gsb.Options(max_iterations=3)
    for m in (gsb.Newton(globalization=gsb.Backtracking(), reuse=2, arithmetic="unfused"),
              gsb.Newton(globalization=gsb.DogLeg(), arithmetic="unfused")):
        X = torch.tensor(X0, device="cuda")
        S = gsb.status_buffer(8)
        gsb.solve_batch(X, S, prob, m, gsb.PerSystem(torch.tensor(P, device="cuda")), options=opts)
        xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
        assert np.array_equal(X.cpu().numpy().view(np.uint64), xo.view(np.uint64))
        assert np.array_equal(S.cpu().numpy(), np.ascontiguousarray(so).view(np.uint8).reshape(-1, 72))


def test_reuse_and_dogleg_checks(gsb):
    """The constructor checks of the reference (src/nonlinear/newton.jl, dogleg.jl:49-60)."""
    with pytest.raises(gsb.ArgumentError):
        gsb.Newton(globalization=gsb.DogLeg(), reuse=2)
    with pytest.raises(gsb.ArgumentError):
        gsb.Newton(globalization=gsb.Backtracking(), reuse=0)
    with pytest.raises(gsb.ArgumentError):
        gsb.DogLeg(radius=-1.0)
    assert gsb.DogLeg(radius=1e-9).radius == 1e-6 and gsb.DogLeg(radius=1e12).radius == 1e10
    m = gsb.Newton(globalization=gsb.Backtracking(), reuse=3).to_abi()
    assert m.reuse == 3 and m.globalization == gsb.abi.GSB_BACKTRACKING
    m = gsb.Newton(globalization=gsb.DogLeg(radius=0.5)).to_abi()
    assert m.globalization == gsb.abi.GSB_DOGLEG and m.dogleg_radius == 0.5 and m.reuse == 0
