"""Ragged batches (systems of sizes 2 ... 32 in one call) against the oracle.

The oracle solves each size bucket as a batch of its own; the device call buckets the systems,
runs one persistent kernel per bucket and writes each system's iterate and status in place.
Under unfused arithmetic every system's result is bit-identical to the oracle's (the one-thread
kernels up to n = 8 and the warp form above are); under fused arithmetic codes and iteration
counts are equal and the solutions agree to 1e-10.
"""

import numpy as np
import pytest

from test_gpu_parity import OPTS, REL_TOL, rel_err
from workloads import C4_SIZES, c4

pytestmark = pytest.mark.gpu


def _dev(a, dtype=None):
    import torch

    return torch.tensor(np.ascontiguousarray(a), dtype=dtype or torch.float64, device="cuda")


def _oracle_by_bucket(gsb, oracle, method, opts, sizes, X0, P):
    """The oracle's solution and status of every system, one uniform batch per size."""
    n64 = sizes.astype(np.int64)
    x_off = np.cumsum(n64) - n64
    p_off = np.cumsum(n64 * n64 + n64) - (n64 * n64 + n64)
    X = X0.copy()
    S = np.zeros(sizes.size, dtype=gsb.SOLVER_STATUS_DTYPE)
    for n in C4_SIZES:
        sel = np.flatnonzero(sizes == n)
        if sel.size == 0:
            continue
        xi = x_off[sel][:, None] + np.arange(n)[None, :]
        pi = p_off[sel][:, None] + np.arange(n * n + n)[None, :]
        xo, so = oracle.solve_batch(gsb.NonlinearProblem(gsb.CubicAffine(n)), method,
                                    X0[xi].copy(), P[pi], opts)
        X[xi] = xo
        S[sel] = so
    return X, S


def _run(gsb, method, opts, sizes, X0, P, table=None, count_form=False):
    X = _dev(X0)
    S = None if count_form else gsb.status_buffer(sizes.size)
    out = gsb.solve_batch_uneven(X, S, _dev(sizes, dtype=__import__("torch").int32), _dev(P),
                                 method, table=table, options=opts)
    return X.cpu().numpy(), (out if count_form else gsb.statuses(S))


def _per_system_err(sizes, x, xo):
    n64 = sizes.astype(np.int64)
    x_off = np.cumsum(n64) - n64
    errs = np.empty(sizes.size)
    for n in C4_SIZES:
        sel = np.flatnonzero(sizes == n)
        if sel.size:
            xi = x_off[sel][:, None] + np.arange(n)[None, :]
            errs[sel] = rel_err(x[xi], xo[xi])
    return errs


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("arith", ["unfused", "fused"])
def test_uneven_parity(gsb, oracle, arith, mixed):
    sizes, X0, P = c4(6000)
    kw = dict(linsolve=gsb.LUFactorization("float32"), refinement=gsb.Refinement()) if mixed else {}
    m = gsb.Newton(globalization=gsb.Backtracking(), arithmetic=arith, **kw)
    opts = gsb.Options(**OPTS)
    xg, sg = _run(gsb, m, opts, sizes, X0, P)
    xo, so = _oracle_by_bucket(gsb, oracle, m, opts, sizes, X0, P)
    assert np.array_equal(sg["code"], so["code"])
    assert np.all(so["code"] == 0)
    if arith == "unfused":
        assert xg.tobytes() == xo.tobytes()
        assert sg.tobytes() == so.tobytes()
    else:
        assert np.all(_per_system_err(sizes, xg, xo) <= REL_TOL)
        if not mixed:
            assert np.array_equal(sg["iterations"], so["iterations"])


def test_uneven_tables_replay_and_count_form(gsb, oracle):
    sizes, X0, P = c4(3000)
    m = gsb.Newton(globalization=gsb.Backtracking(), arithmetic="unfused")
    opts = gsb.Options(**OPTS)
    xo, so = _oracle_by_bucket(gsb, oracle, m, opts, sizes, X0, P)
    # the 32-lane teams at n = 12 and 16, one CTA per SM everywhere: the same bits
    tab = [(0, 1)] * 9
    tab[5] = (32, 1)
    tab[6] = (32, 2)
    # the warp form's CTA size chosen per bucket: 32 lanes (two 16-lane systems) at n = 12, one
    # 32-lane system at n = 16 and 24, two at n = 32
    tab3 = [(0, 0, 0)] * 9
    tab3[5] = (16, 0, 2)
    tab3[6] = (32, 0, 1)
    tab3[7] = (32, 3, 1)
    tab3[8] = (32, 0, 2)
    # every bucket as one ordinary grid sized from its count, and a mix of the two forms
    tab_ord = [(0, -1, 0)] * 9
    tab_mix = list(tab3)
    tab_mix[0] = (0, -1, 0)
    tab_mix[4] = (0, -1, 0)
    tab_mix[8] = (32, -1, 2)
    for table in (None, tab, tab, tab3, tab_ord, tab_mix, tab_ord):
        # (the third call replays the graph of the second, the last that of tab_ord)
        xg, sg = _run(gsb, m, opts, sizes, X0, P, table=table)
        assert xg.tobytes() == xo.tobytes()
        assert sg.tobytes() == so.tobytes()
    counts = _run(gsb, m, opts, sizes, X0, P, count_form=True)[1]
    assert list(counts) == np.bincount(so["code"], minlength=6).tolist()


def test_uneven_fused_teams(gsb, oracle):
    # the multi-lane teams of n = 6 and 8 (fused arithmetic): codes, iterations and 1e-10
    sizes, X0, P = c4(3000)
    m = gsb.Newton(globalization=gsb.Backtracking())
    opts = gsb.Options(**OPTS)
    xo, so = _oracle_by_bucket(gsb, oracle, m, opts, sizes, X0, P)
    tab = [(0, 0)] * 9
    tab[3] = (2, 0)
    tab[4] = (4, 0)
    xg, sg = _run(gsb, m, opts, sizes, X0, P, table=tab)
    assert np.array_equal(sg["code"], so["code"])
    assert np.array_equal(sg["iterations"], so["iterations"])
    assert np.all(_per_system_err(sizes, xg, xo) <= REL_TOL)


def test_uneven_rejections(gsb):
    import torch

    sizes, X0, P = c4(64)
    m = gsb.Newton(globalization=gsb.Backtracking())
    bad = sizes.copy()
    bad[5] = 5  # not a bucket size
    Xd = _dev(X0)
    with pytest.raises(gsb.ArgumentError):
        gsb.solve_batch_uneven(Xd, None, torch.tensor(bad, device="cuda"), _dev(P), m)
    with pytest.raises(gsb.DimensionMismatch):
        gsb.solve_batch_uneven(Xd[:-1], None, torch.tensor(sizes, device="cuda"), _dev(P), m)
    # an unfused method has no multi-lane team at n = 8
    with pytest.raises(gsb.ArgumentError):
        gsb.solve_batch_uneven(Xd, None, torch.tensor(sizes, device="cuda"), _dev(P),
                               gsb.Newton(arithmetic="unfused"), table=[(0, 0)] * 4 + [(2, 0)] + [(0, 0)] * 4)


def test_uneven_cta_size_rejections(gsb):
    import torch

    sizes, X0, P = c4(64)
    m = gsb.Newton(globalization=gsb.Backtracking())
    args = (_dev(X0), None, torch.tensor(sizes, device="cuda"), _dev(P), m)
    for b, cfg in ((4, (1, 0, 2)),     # the one-thread form has a fixed CTA size
                   (8, (32, 0, 8)),    # 256 lanes: above the warp form's 128
                   (5, (16, 0, 1)),    # 16 lanes: not a whole warp
                   (3, (0, -2, 0))):   # CTAs per SM below -1
        tab = [(0, 0, 0)] * 9
        tab[b] = cfg
        with pytest.raises(gsb.ArgumentError):
            gsb.solve_batch_uneven(*args, table=tab)


def test_autotuner_table(gsb):
    m = gsb.Newton(globalization=gsb.Backtracking())
    table, timings = gsb.tune.autotune_uneven(m, sample=2048, reps=1, sizes=(8, 16))
    assert len(table) == 9 and all(len(t) == 3 for t in table)
    assert table[4][0] in (1, 2, 4, 8) and table[6][0] in (16, 32)
    assert table[4][2] == 0 and table[6][2] * table[6][0] in (32, 64, 128)
    assert set(timings) == {8, 16} and all(v > 0 for v in timings[8].values())
    # both CTA sizes and team sizes of n = 16 were timed
    assert {k.split("/")[2] for k in timings[16]} == {"s1", "s2", "s4", "s8"}
