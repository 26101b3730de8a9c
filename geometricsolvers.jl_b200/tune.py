"""The autotuner of the ragged batch (``solve_batch_uneven``): for each size bucket it times the
kernel configurations that libgsb has for that size under the given method, and keeps the
fastest. A configuration is

- the threads per system: one thread up to n = 8, or a team of 2, 4 or 8 lanes at n = 6 and 8
  under fused arithmetic; 16 or 32 lanes at n = 12 and 16; 32 lanes above;
- the systems per CTA of the warp form (n >= 12): CTAs of 32, 64 or 128 threads. Its systems
  keep their parameter blocks (and, in 16-lane teams, their factors) in shared memory and, in
  32-lane teams, their factor rows in registers, so the CTA size sets how finely the registers
  and the shared memory of an SM are divided (0: four systems of 32 lanes or eight of 16). The
  one-thread kernels work warp by warp and the team kernels of n = 6 and 8 hold one parameter
  row per system, so for them the CTA size is fixed;
- the resident CTAs per SM of the bucket's persistent launch (0: as many as fit), which sets how
  the bucket's kernel shares the GPU with the other buckets running beside it, or -1: no
  persistent kernel but one ordinary grid, sized from the bucket's count once the bucketing has
  run (the persistent form's work loop costs the large warp-form kernels registers and
  instruction-cache misses).

The timing batch of a size is synthetic and seeded: cubic-affine systems with A = (n+1) I +
0.5 N(0,1) and b ~ U(-1, 1)^n from x0 = 0 (the distribution of the ragged benchmark), unless the
caller passes its own generator. Tables are saved to and loaded from JSON; the package carries
the tables tuned on B200 (``tuned_uneven_b200.json``), which ``solve_batch_uneven`` takes when
it is given no table.
"""

from __future__ import annotations

import json
import os

from .abi import UNEVEN_SIZES

CANDIDATE_THREADS = {2: (1,), 3: (1,), 4: (1,), 6: (1, 2), 8: (1, 2, 4, 8), 12: (16, 32),
                     16: (16, 32), 24: (32,), 32: (32,)}
# persistent CTAs per SM (0: as many as fit), or -1: one ordinary grid sized from the count
CANDIDATE_CTAS = (-1, 0, 1, 2, 3, 4, 6, 8)
# systems per CTA of the warp form, by lanes per system (CTAs of 32 to 128 threads)
CANDIDATE_SPC = {16: (2, 4, 8), 32: (1, 2, 4)}

TUNED_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_uneven_b200.json")


def default_table():
    return [(0, 0, 0)] * len(UNEVEN_SIZES)


def form_key(method):
    """The key of a method's table: factor precision, refinement and arithmetic."""
    from . import abi

    m = method.to_abi()
    prec = "fp32" if m.factor_precision == abi.GSB_F32 else "fp64"
    ref = "refinement" if m.refinement == abi.GSB_REFINEMENT else "norefinement"
    arith = "unfused" if m.arithmetic == abi.GSB_UNFUSED else "fused"
    return f"{prec}_{ref}_{arith}"


def synthetic_bucket(n, count, seed=20261207, device="cuda"):
    """`count` systems of size n, packed: (X0, P) as flat float64 tensors on `device`."""
    import torch

    g = torch.Generator(device="cpu").manual_seed(seed + n)
    A = torch.randn(count, n, n, generator=g, dtype=torch.float64) * 0.5
    A += (n + 1.0) * torch.eye(n, dtype=torch.float64)
    b = torch.rand(count, n, generator=g, dtype=torch.float64) * 2.0 - 1.0
    P = torch.cat([A.transpose(1, 2).reshape(count, n * n), b], dim=1)
    return (torch.zeros(count * n, dtype=torch.float64, device=device),
            P.reshape(-1).contiguous().to(device))


def _time(solve, reps):
    import torch

    solve()  # builds the graph of this configuration
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        solve()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def candidates(n, fused):
    """Every (threads_per_system, ctas_per_sm, systems_per_cta) the library has for size n."""
    out = []
    for T in CANDIDATE_THREADS[n]:
        if T > 1 and n <= 8 and not fused:
            continue  # the multi-lane teams of small systems are fused-only
        for spc in (CANDIDATE_SPC[T] if n >= 12 else (0,)):
            for c in CANDIDATE_CTAS:
                out.append((T, c, spc))
    return out


def autotune_uneven(method, options=None, sample=16384, reps=3, generator=None, sizes=None,
                    verbose=False):
    """`sample` systems of size 32 per timing, proportionally more of the smaller sizes (up to
    262,144). Returns (table, timings): the table for ``solve_batch_uneven`` (nine
    (threads_per_system, ctas_per_sm, systems_per_cta) triples) and, per size, the milliseconds
    of every configuration tried."""
    import torch

    from .batch import solve_batch_uneven

    fused = getattr(method, "arithmetic", "fused") == "fused"
    table = default_table()
    timings = {}
    for b, n in enumerate(UNEVEN_SIZES):
        if sizes is not None and n not in sizes:
            continue
        # small systems take more samples, so that a timing is not a launch latency
        count = min(262144, sample * max(1, 32 // n))
        X0, P = (generator or synthetic_bucket)(n, count)
        X = torch.empty_like(X0)
        nv = torch.full((count,), n, dtype=torch.int32, device=X0.device)
        best, best_ms, tried = None, float("inf"), {}
        for cfg in candidates(n, fused):
            tab = list(table)
            tab[b] = cfg

            def solve(tab=tab):
                X.copy_(X0)
                solve_batch_uneven(X, None, nv, P, method, table=tab, options=options)

            ms = _time(solve, reps)
            tried["T{}/c{}/s{}".format(*cfg)] = ms
            if ms < best_ms:
                best, best_ms = cfg, ms
        table[b] = best
        timings[n] = tried
        if verbose:
            print(f"n={n}: {best} {best_ms:.3f} ms", flush=True)
    return table, timings


def save_table(path, table, timings=None, meta=None):
    """One table (a list of nine triples) as JSON."""
    with open(path, "w") as f:
        json.dump({"sizes": list(UNEVEN_SIZES), "table": [list(t) for t in table],
                   "timings_ms": timings or {}, "meta": meta or {}}, f, indent=1)


def _triples(rows):
    out = []
    for t in rows:
        t = tuple(int(v) for v in t)
        out.append(t + (0,) * (3 - len(t)))  # a pair from an older table: default CTA size
    return out


def load_table(path):
    with open(path) as f:
        d = json.load(f)
    if d.get("sizes") != list(UNEVEN_SIZES):
        raise ValueError("the table was written for another set of sizes")
    return _triples(d["table"])


def save_tables(path, tables, timings=None, meta=None):
    """Tables of several methods, keyed by ``form_key``, as JSON."""
    with open(path, "w") as f:
        json.dump({"sizes": list(UNEVEN_SIZES),
                   "tables": {k: [list(t) for t in v] for k, v in tables.items()},
                   "timings_ms": timings or {}, "meta": meta or {}}, f, indent=1)


_tuned = {}


def tuned_table(method, path=TUNED_PATH):
    """The committed table of `method`'s form, or None when the file has none for it."""
    if path not in _tuned:
        try:
            with open(path) as f:
                d = json.load(f)
        except FileNotFoundError:
            d = {}
        if d and d.get("sizes") != list(UNEVEN_SIZES):
            raise ValueError(f"{path} was written for another set of sizes")
        _tuned[path] = {k: _triples(v) for k, v in d.get("tables", {}).items()}
    return _tuned[path].get(form_key(method))


def main(argv=None):
    """Tune the ragged batch's forms on this GPU and write the package's table file:
    ``python -c "import gsb200.tune as t; t.main()" [--out PATH] [--sample N] [--reps R]``.
    The forms are the plain Float64 LU step and the Float32 LU step with refinement (both with
    Backtracking) under fused arithmetic, and the plain step under unfused arithmetic."""
    import argparse

    import torch

    from .api import Backtracking, LUFactorization, Newton, Options, Refinement

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=TUNED_PATH)
    ap.add_argument("--sample", type=int, default=16384)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args(argv)
    opts = Options(f_abstol=1e-12, f_reltol=0.0, max_iterations=50)
    forms = [Newton(globalization=Backtracking()),
             Newton(linsolve=LUFactorization("float32"), refinement=Refinement(),
                    globalization=Backtracking()),
             Newton(globalization=Backtracking(), arithmetic="unfused")]
    tables, timings = {}, {}
    for m in forms:
        key = form_key(m)
        tables[key], timings[key] = autotune_uneven(m, options=opts, sample=args.sample,
                                                    reps=args.reps, verbose=True)
    meta = {"gpu": torch.cuda.get_device_name(), "sample": args.sample, "reps": args.reps,
            "options": "f_abstol=1e-12, f_reltol=0, max_iterations=50",
            "workload": "cubic-affine, A = (n+1)I + 0.5 N(0,1), b ~ U(-1,1)^n, x0 = 0"}
    save_tables(args.out, tables, timings, meta)
    _tuned.pop(args.out, None)
    print(f"wrote {args.out}")
