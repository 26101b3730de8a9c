"""The autotuner of the ragged batch (``solve_batch_uneven``): for each size bucket it times the
kernel configurations that libgsb has for that size under the given method, and keeps the
fastest. A configuration is the threads per system (one thread up to n = 8, or a team of 2, 4
or 8 lanes at n = 6 and 8 under fused arithmetic; 16 or 32 lanes at n = 12 and 16; 32 lanes
above) and the resident CTAs per SM of the bucket's persistent launch (0: as many as fit),
which sets how the bucket's kernel shares the GPU with the other buckets running beside it.

The timing batch of a size is synthetic and seeded: cubic-affine systems with A = (n+1) I +
0.5 N(0,1) and b ~ U(-1, 1)^n from x0 = 0 (the distribution of the ragged benchmark), unless the
caller passes its own generator. The table can be saved to and loaded from a JSON file.
"""

from __future__ import annotations

import json

from .abi import UNEVEN_SIZES

CANDIDATE_THREADS = {2: (1,), 3: (1,), 4: (1,), 6: (1, 2), 8: (1, 2, 4, 8), 12: (16, 32),
                     16: (16, 32), 24: (32,), 32: (32,)}
CANDIDATE_CTAS = (0, 1, 2, 3, 4, 6, 8)


def default_table():
    return [(0, 0)] * len(UNEVEN_SIZES)


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


def autotune_uneven(method, options=None, sample=16384, reps=3, generator=None, sizes=None,
                    verbose=False):
    """`sample` systems of size 32 per timing, proportionally more of the smaller sizes (up to
    262,144). Returns (table, timings): the table for ``solve_batch_uneven`` (nine (threads_per_system,
    ctas_per_sm) pairs) and, per size, the milliseconds of every configuration tried."""
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
        for T in CANDIDATE_THREADS[n]:
            if T > 1 and n <= 8 and not fused:
                continue  # the multi-lane teams of small systems are fused-only
            for c in CANDIDATE_CTAS:
                tab = list(table)
                tab[b] = (T, c)

                def solve(tab=tab):
                    X.copy_(X0)
                    solve_batch_uneven(X, None, nv, P, method, table=tab, options=options)

                ms = _time(solve, reps)
                tried[f"T{T}/c{c}"] = ms
                if ms < best_ms:
                    best, best_ms = (T, c), ms
        table[b] = best
        timings[n] = tried
        if verbose:
            print(f"n={n}: {best} {best_ms:.3f} ms", flush=True)
    return table, timings


def save_table(path, table, timings=None, meta=None):
    with open(path, "w") as f:
        json.dump({"sizes": list(UNEVEN_SIZES), "table": [list(t) for t in table],
                   "timings_ms": timings or {}, "meta": meta or {}}, f, indent=1)


def load_table(path):
    with open(path) as f:
        d = json.load(f)
    if d.get("sizes") != list(UNEVEN_SIZES):
        raise ValueError("the table was written for another set of sizes")
    return [tuple(t) for t in d["table"]]
