"""The mixed form with Float32 line-search trials (``Newton(..., trial="float32")``), a departure
from the reference judged against the reference's plain Float64 solve: on well-conditioned
batches identical status codes and ‖x - x_ref‖∞ / ‖x_ref‖∞ ≤ 1e-10 per system; on
ill-conditioned ones the status contract and a bounded share of different outcomes."""

import numpy as np
import pytest

from test_gpu_parity import OPTS, rel_err, run_gpu
from workloads import cubic_affine, cubic_affine_illcond

REL_TOL = 1e-10


def _trial32(gsb, glob):
    return gsb.Newton(linsolve=gsb.LUFactorization("float32"), refinement=gsb.Refinement(),
                      globalization=glob, trial="float32")


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 3, 4, 6, 8])
def test_trial32_against_fp64_oracle(gsb, oracle, n):
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    opts = gsb.Options(**OPTS)
    X0, P = cubic_affine(n, 8192, n + 1.0, 4)
    for glob in (gsb.Backtracking(), gsb.Static()):
        xo, so = oracle.solve_batch(prob, gsb.Newton(globalization=glob), X0.copy(), P, opts)
        xg, sg = run_gpu(gsb, prob, _trial32(gsb, glob), X0, P, opts)
        same = sg["code"] == so["code"]
        ok = same & (so["code"] == 0)
        assert np.all(same), f"codes differ at {np.flatnonzero(~same)[:8]}"
        assert np.all(rel_err(xg[ok], xo[ok]) <= REL_TOL)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 4, 8])
def test_trial32_ill_conditioned(gsb, oracle, n):
    # Condition numbers 1e3 ... 1e9. Here the departure shows: the Float32 trials end
    # differently from the plain Float64 solve on 3.6 % (n = 2) to 16 % (n = 8) of the systems,
    # where the reference's own mixed form (Float64 trials) differs on 0.9 % to 5 %. What holds
    # is the status contract: every system reported SUCCESS meets the residual tolerance in
    # Float64, and the differences stay below a quarter of the batch.
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    opts = gsb.Options(**OPTS)
    X0, P = cubic_affine_illcond(n, 2048, 5)
    for glob in (gsb.Backtracking(), gsb.Static()):
        _, sp = oracle.solve_batch(prob, gsb.Newton(globalization=glob), X0.copy(), P, opts)
        _, sg = run_gpu(gsb, prob, _trial32(gsb, glob), X0, P, opts)
        assert np.mean(sg["code"] != sp["code"]) <= 0.25
        ok = sg["code"] == 0
        assert ok.mean() > 0.5
        assert np.all(sg["fnorm"][ok] <= OPTS["f_abstol"])


def test_trial32_checks(gsb):
    with pytest.raises(gsb.ArgumentError):
        gsb.Newton(trial="float32")  # a Float64 factor
    with pytest.raises(gsb.ArgumentError):
        gsb.Newton(linsolve=gsb.LUFactorization("float32"), trial="float32", reuse=2,
                   globalization=gsb.Backtracking())
    with pytest.raises(gsb.ArgumentError):
        gsb.Newton(linsolve=gsb.LUFactorization("float32"), trial="float16")
    m = _trial32(gsb, gsb.Backtracking())
    assert m.to_abi().trial_precision == 1 and gsb.Newton().to_abi().trial_precision == 0
