"""Benchmark of the batch solver: systems solved per second at per-system relative error ≤ 1e-10
with matching status codes, the chosen form against plain FP64, on the n = 8 cubic-affine batch
of 1,048,576 systems (F(x) = A x + 0.1 x.^3 - b, A = 6I + 0.5 N(0,1), b ~ U(-1,1)^8, x0 = 0,
f_abstol = 1e-12, f_reltol = 0, max_iterations = 50, Newton + LU + Backtracking).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A step solves one batch in place (the start iterates are copied into the working buffer, a
device-to-device copy inside the step). The inputs (604 MB of parameters) exceed the 126 MB L2,
so no flush is needed between steps. One JSON line is printed by rank 0.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

N_UNKNOWNS = 8
NSYS = 1 << 20
METRIC = "systems solved/s at rel err ≤1e-10, chosen form vs plain FP64, one B200"
REL_TOL = 1e-10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="gsb200", choices=["gsb200", "reference"])
    ap.add_argument("--nsys", type=int, default=NSYS)
    ap.add_argument("--profile", choices=["plain", "mixed", "lm", "irk", "mlp", "predict", "shared"],
                    default=None,
                    help="run `--warmup` + `--steps` solves of one form only (for ncu captures): "
                         "the cubic-affine batch of size --n, or the exponential-sum fit (lm)")
    ap.add_argument("--workload", choices=["c1", "c0", "c2", "c3", "c4"], default="c1",
                    help="c1 (default): the n = 8 batch of the headline metric; c0: n = 3, "
                         "65,536 systems; c2: the exponential-sum least-squares fit; c3: the "
                         "Gauss-3 stage systems with the learned warm start; c4: the "
                         "ragged batch of sizes 2..32 (one GPU)")
    ap.add_argument("--launch-check", action="store_true",
                    help="start the ranks as for a run and take the job's collectives (barrier, "
                         "maximum and sum over ranks) over gloo on the CPU, rank 0 printing the "
                         "world size: the multi-rank launcher without a GPU")
    ap.add_argument("--n", type=int, default=N_UNKNOWNS,
                    help="cubic-affine size of a --profile run (A = 6I + ... at n = 8, else (n+1)I)")
    return ap.parse_args()


def options(gsb):
    return gsb.Options(f_abstol=1e-12, f_reltol=0.0, max_iterations=50)


def methods(gsb):
    plain = gsb.Newton(globalization=gsb.Backtracking())
    mixed = gsb.Newton(linsolve=gsb.LUFactorization("float32"), refinement=gsb.Refinement(),
                       globalization=gsb.Backtracking())
    return plain, mixed


def workload(rank, nsys):
    """Rank `rank`'s shard of the n = 8 batch: its own counter stream of the seeded generator,
    so shards are disjoint draws and every run draws the same ones."""
    from workloads import cubic_affine

    return cubic_affine(N_UNKNOWNS, nsys, 6.0, 1, stream=rank)


class Ranks:
    """The job's ranks as the bench uses them: a barrier, and the maximum (timings) and sum
    (solved counts) of one value over ranks. Every rank calls each in the same order; with one
    rank they are the identity. `dev` is where the reduction tensors live (the rank's GPU under
    NCCL, the CPU under gloo)."""

    def __init__(self, world, dev=None):
        self.world = world
        self.dev = dev

    def _reduce(self, v, op):
        if self.world == 1:
            return v
        import torch
        import torch.distributed as dist

        t = torch.tensor([v], dtype=torch.float64, device=self.dev)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist

            dist.barrier()

    def max(self, v):
        import torch.distributed as dist

        return self._reduce(v, dist.ReduceOp.MAX if self.world > 1 else None)

    def sum(self, v):
        import torch.distributed as dist

        return self._reduce(v, dist.ReduceOp.SUM if self.world > 1 else None)


# ─── roofline model ──────────────────────────────────────────────────────────────────────────


def flops_per_system(n, iterations, f_evals):
    """Floating-point operations of the plain FP64 Newton + LU + Backtracking step on the
    cubic-affine family (a fused multiply-add counts 2, a division or square root 1), from the
    oracle's per-system counts: f_evals residual evaluations (each with its merit) and
    `iterations` steps (Jacobian, gradient ratio, pivoted LU, solve, step norms)."""
    f_eval = 2 * n * n + 6 * n                       # rows, cubic terms, norm2
    lu = n * (n - 1) // 2 + (n - 1) * n * (2 * n - 1) // 3
    per_step = (6 * n                                  # forward-mode diagonal of J
                + 4 * n * n + 2 * n + 4                # ‖J‖_F, Jᵀ F, their norms and ratio
                + lu                                   # pivoted LU
                + 2 * n * n - n                        # forward and back substitution
                + 4 * n + 2 + 10)                      # ‖d‖, ‖x‖, the stopping tests
    trials = np.maximum(f_evals - 1, 0)
    return f_evals * f_eval + iterations * per_step + trials * 2 * n


def bytes_per_system(n):
    return 8 * n + 8 * (n * n + n) + 8 * n + 72


def measured_peaks():
    """The HBM copy bandwidth of MEASURED_PEAKS.json (measured on this pool's B200s), else the
    pool's earlier measurement of 6650 GB/s, with a label that says which."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6650 GB/s (MEASURED_PEAKS.json absent)"


def fp_peaks():
    lib = ctypes.CDLL(os.path.join(ROOT, "geometricsolvers.jl_b200", "peak", "libgsbpeak.so"))
    lib.gsb_peak_fma.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    out = {}
    for name, fp64 in (("fp64", 1), ("fp32", 0)):
        best = 0.0
        for _ in range(3):
            t = ctypes.c_double()
            if lib.gsb_peak_fma(fp64, 4000, ctypes.byref(t)) == 0:
                best = max(best, t.value)
        out[name] = best
    return out


# DRAM bytes per launch of the plain n = 8 kernel (dram__bytes_read.sum + dram__bytes_write.sum)
# from one ncu capture of 262,144 systems, scaled by 4 to the 1,048,576-system launch (traffic grows
# with the systems): the capture and its command are in profiles/newton_cubic8_fp64.md. A figure
# of a capture, not of this run: the line labels it so.
TRAFFIC_PER_LAUNCH = 189.75e6 * 4
TRAFFIC_SOURCE = "ncu capture (profiles/newton_cubic8_fp64.md), 262,144 systems scaled x4"


# ─── clocks ──────────────────────────────────────────────────────────────────────────────────


class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="gsb_clocks_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait(timeout=10)
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                f = [v.strip() for v in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax.append(float(f[2]))
                except ValueError:
                    continue
                for name, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
        os.remove(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# ─── the reference arm: the oracle (the CPU restatement) on the host cores ─────────────────


def run_reference(args, rank, world):
    if rank != 0:
        return
    import gsb200 as G
    from oracle import oracle_py as O

    nt = O.max_threads()
    X0, P = workload(0, args.nsys)
    prob = G.NonlinearProblem(G.CubicAffine(N_UNKNOWNS))
    plain, _ = methods(G)
    opts = options(G)
    sample = min(args.nsys, 262144)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        O.solve_batch(prob, plain, X0[:sample].copy(), P[:sample], opts, nthreads=nt)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    med = statistics.median(times)
    value = sample / med
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "systems/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": med * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Philox)",
        "config": {"workload": f"cubic-affine n=8, {args.nsys} systems, Newton+LU+Backtracking FP64",
                   "sample_systems": sample},
        "cpu_baseline": {"value": value, "unit": "systems/s", "cores": nt, "kind": "port",
                         "sample": f"{sample} of the {args.nsys} systems per step, plain FP64"},
        "e2e": {"value": value, "unit": "systems/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ─── our arm ─────────────────────────────────────────────────────────────────────────────────


def rel_err(x, xr):
    num = np.max(np.abs(x - xr), axis=1)
    den = np.max(np.abs(xr), axis=1)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(den > 0, num / den, num)


def free_port():
    import socket

    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def launch_ranks(args):
    """`--gpus N` without a launcher around this process: start N ranks of the same command under
    torch.distributed.run (one per GPU, rendezvous on 127.0.0.1) and return their exit code.
    NCCL's initialisation log (the communicator and its rank count) goes to stderr, so stdout
    keeps the one JSON line of rank 0."""
    env = dict(os.environ)
    env.setdefault("NCCL_DEBUG", "INFO")
    env.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
    env.setdefault("NCCL_DEBUG_FILE", "/dev/stderr")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
           f"--master-port={free_port()}", os.path.abspath(__file__), *sys.argv[1:]]
    proc = subprocess.Popen(cmd, env=env, start_new_session=True)
    try:
        return proc.wait(timeout=1800)
    except subprocess.TimeoutExpired:
        os.killpg(proc.pid, 9)  # the launcher's own process group: its ranks
        proc.wait()
        return 124


def launch_check(rank, world):
    import datetime

    import torch
    import torch.distributed as dist

    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        ranks = Ranks(world, torch.device("cpu"))
        ranks.barrier()
        slowest = ranks.max(float(rank))
        count = ranks.sum(1.0)
        ranks.barrier()
        if rank == 0:
            print(json.dumps({"launch_check": True, "n_gpus": world, "max_rank": slowest,
                              "ranks_counted": count}), flush=True)
    finally:
        if world > 1:
            dist.destroy_process_group()


def main():
    args = parse()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(launch_ranks(args))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        sys.exit(f"bench.py: --gpus {args.gpus} but the launcher started {world} ranks")
    if args.launch_check:
        launch_check(rank, world)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1 and (args.profile or args.workload != "c1"):
        sys.exit("bench.py: --profile and --workload c0/c2/c3/c4 run on one GPU")
    if args.profile:
        run_profile(args)
        return
    if args.workload != "c1":
        run_workload(args)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    ranks = Ranks(world, dev)
    barrier, max_over_ranks, sum_over_ranks = ranks.barrier, ranks.max, ranks.sum

    import gsb200 as G
    from oracle import oracle_py as O

    nsys = args.nsys
    X0_h, P_h = workload(rank, nsys)
    prob = G.NonlinearProblem(G.CubicAffine(N_UNKNOWNS))
    plain, mixed = methods(G)
    opts = options(G)
    X0 = torch.tensor(X0_h, device=dev)
    P = torch.tensor(P_h, device=dev)
    X = torch.empty_like(X0)
    S = G.status_buffer(nsys, device=dev)
    ps = G.PerSystem(P)
    stream = torch.cuda.current_stream(dev)

    # correctness of each form against the oracle (untimed): the count of systems solved
    nt = max(1, O.max_threads() // max(1, world))
    xo, so = O.solve_batch(prob, plain, X0_h.copy(), P_h, opts, nthreads=nt)
    solved = {}
    fp64_err = {}
    # the mixed form with its line-search trials in Float32 too (a labelled departure)
    trial32 = G.Newton(linsolve=G.LUFactorization("float32"), refinement=G.Refinement(),
                       globalization=G.Backtracking(), trial="float32")
    for name, m in (("plain_fp64", plain), ("fp32_lu_refinement", mixed),
                    ("fp32_lu_refinement_fp32_trials", trial32)):
        X.copy_(X0)
        G.solve_batch(X, S, prob, m, ps, options=opts)
        st = G.statuses(S)
        x = X.cpu().numpy()
        err = rel_err(x, xo)
        ok = (st["code"] == so["code"]) & (err <= REL_TOL)
        solved[name] = int(np.count_nonzero(ok))
        fp64_err[name] = float(np.max(err))
        if name == "plain_fp64":
            iters_match = bool(np.array_equal(st["iterations"], so["iterations"]))
    flops = float(np.sum(flops_per_system(N_UNKNOWNS, so["iterations"].astype(np.int64),
                                          so["iterations"].astype(np.int64) * 0 + 1 +
                                          _trials(so))))

    def timed(m, steps, warmup):
        for _ in range(warmup):
            X.copy_(X0)
            G.solve_batch(X, S, prob, m, ps, options=opts)
        barrier()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            X.copy_(X0)
            G.solve_batch(X, S, prob, m, ps, options=opts)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / steps)

    # kernel-only time of one launch (no copy), for the roofline
    def kernel_ms(m, reps=8):
        """The kernel alone: `reps` launches through the C-ABI queued back to back on the stream
        (each on its own copy of the start iterates, made beforehand), between two events, so
        that no host work sits between the launches; the mean per launch."""
        lib = G.load_library()
        from gsb200 import batch as B

        Xs = [X0.clone() for _ in range(reps)]
        gm, go = B._abi_of(m), B._abi_of(opts)
        gp = prob.to_abi(None)
        st = ctypes.c_void_p(stream.cuda_stream)
        torch.cuda.synchronize(dev)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for Xr in Xs:
            rc = lib.gsb_solve_batch(ctypes.byref(gp), ctypes.byref(gm), ctypes.byref(go),
                                     Xr.data_ptr(), 0, S.data_ptr(), 0, P.data_ptr(), 0, None, 0,
                                     nsys, st, None)
            assert rc == 0, rc
        b.record(stream)
        torch.cuda.synchronize(dev)
        assert lib.gsb_synchronize(st) == 0
        return a.elapsed_time(b) / reps

    with Clocks(local) as clk:
        ms_plain = timed(plain, args.steps, args.warmup)
        ms_mixed = timed(mixed, args.steps, args.warmup)
        ms_trial32 = timed(trial32, args.steps, args.warmup)
    clocks = clk.summary()
    chosen_name = "fp32_lu_refinement" if solved["fp32_lu_refinement"] / ms_mixed >= \
        solved["plain_fp64"] / ms_plain else "plain_fp64"
    chosen_m = mixed if chosen_name == "fp32_lu_refinement" else plain
    ms_chosen = ms_mixed if chosen_name == "fp32_lu_refinement" else ms_plain
    total_solved = sum_over_ranks(solved[chosen_name])
    value = total_solved / (ms_chosen * 1e-3)
    plain_value = sum_over_ranks(solved["plain_fp64"]) / (ms_plain * 1e-3)

    # end to end through the public API: the batch in pinned host memory, solved by the
    # pipelined host-buffer call (copies in both directions overlapping the chunk solves); the
    # call returns when every result is in host memory, so each step is timed by the host clock
    x_pin = torch.from_numpy(X0_h).pin_memory()
    p_pin = torch.from_numpy(P_h).pin_memory()
    x_io = torch.empty_like(x_pin).pin_memory()
    s_out = torch.empty((nsys, 72), dtype=torch.uint8).pin_memory()
    pse = G.PerSystem(p_pin)

    def e2e_step():
        G.solve_batch_host(x_io, s_out, prob, chosen_m, pse, options=opts)

    for _ in range(max(1, args.warmup // 4)):
        x_io.copy_(x_pin)
        e2e_step()
    barrier()
    e2e_steps = max(3, args.steps // 10)
    t_e2e = []
    for _ in range(e2e_steps):
        x_io.copy_(x_pin)  # the start iterates again (host side, outside the timed call)
        t0 = time.perf_counter()
        e2e_step()
        t_e2e.append(time.perf_counter() - t0)
    ms_e2e = max_over_ranks(statistics.median(t_e2e) * 1e3)
    e2e_value = total_solved / (ms_e2e * 1e-3)
    h2d = X0_h.nbytes + P_h.nbytes
    d2h = X0_h.nbytes + nsys * 72

    # roofline of the plain FP64 kernel
    hbm_peak, hbm_src = measured_peaks()
    peaks = fp_peaks()
    kms = kernel_ms(plain)
    bytes_total = bytes_per_system(N_UNKNOWNS) * nsys
    t_bytes = bytes_total / (hbm_peak * 1e9)
    t_flops = flops / (peaks["fp64"] * 1e12)
    achieved_gbs = bytes_total / (kms * 1e-3) / 1e9
    achieved_tf = flops / (kms * 1e-3) / 1e12
    traffic = TRAFFIC_PER_LAUNCH if nsys == NSYS else None
    if t_bytes >= t_flops:
        roof = {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved_gbs / hbm_peak, "traffic": traffic,
                "traffic_source": TRAFFIC_SOURCE,
                "peak_source": hbm_src}
    else:
        roof = {"bound": "fp64", "achieved": achieved_tf, "peak": peaks["fp64"],
                "unit": "TFLOP/s", "frac": achieved_tf / peaks["fp64"], "traffic": traffic,
                "peak_source": "measured (FP64 FMA probe, libgsbpeak)"}
    roof["kernel"] = "newton_kernel<CubicAffine<8>, fused, FP64>"
    roof["kernel_ms"] = kms
    roof["fp64_frac"] = achieved_tf / peaks["fp64"] if peaks["fp64"] else None
    roof["hbm_frac"] = achieved_gbs / hbm_peak
    roof["flops_per_launch"] = flops
    roof["bytes_per_launch"] = bytes_total
    roof["fp64_peak_tflops"] = peaks["fp64"]
    roof["fp32_peak_tflops"] = peaks["fp32"]

    # CPU baseline: the oracle on the host cores, on a bounded sample of the same batch
    cpu = None
    if rank == 0 and world == 1:
        ntall = O.max_threads()
        sample = 262144
        reps, t_tot = 0, 0.0
        while t_tot < 10.0 and reps < 40:
            t0 = time.perf_counter()
            O.solve_batch(prob, plain, X0_h[:sample].copy(), P_h[:sample], opts, nthreads=ntall)
            t_tot += time.perf_counter() - t0
            reps += 1
        # one host thread on a smaller sample of the same batch
        s1 = 32768
        t0 = time.perf_counter()
        O.solve_batch(prob, plain, X0_h[:s1].copy(), P_h[:s1], opts, nthreads=1)
        t1 = time.perf_counter() - t0
        cpu = {"value": sample * reps / t_tot, "unit": "systems/s", "cores": ntall, "kind": "port",
               "sample": f"{reps} x {sample} of the {nsys} systems, plain FP64, "
                         f"{ntall} threads, {t_tot:.1f} s",
               "value_1_thread": s1 / t1,
               "sample_1_thread": f"{s1} of the {nsys} systems, plain FP64, 1 thread, {t1:.2f} s"}

    line = {
        "metric": METRIC, "value": value, "unit": "systems/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_chosen,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Philox; reference configuration's shapes and distributions)",
        "config": {
            "workload": "cubic-affine F = A x + 0.1 x.^3 - b, n=8, 1,048,576 systems per GPU, "
                        "Newton + LU + Backtracking, f_abstol 1e-12, max_iterations 50",
            "chosen_form": chosen_name, "global_batch": int(nsys * world),
            "parallelism": f"independent shards x{world} (no collective in the solve)",
            "l2": "inputs (604 MB parameters) exceed the 126 MB L2; no flush",
        },
        "forms": {
            "plain_fp64": {"systems_per_s": plain_value, "ms_per_step": ms_plain,
                           "solved": solved["plain_fp64"], "fp64_oracle_max_rel_err": fp64_err["plain_fp64"],
                           "iterations_match_oracle": iters_match},
            "fp32_lu_refinement": {"systems_per_s": sum_over_ranks(solved["fp32_lu_refinement"]) / (ms_mixed * 1e-3),
                                   "ms_per_step": ms_mixed, "solved": solved["fp32_lu_refinement"],
                                   "fp64_oracle_max_rel_err": fp64_err["fp32_lu_refinement"]},
            "fp32_lu_refinement_fp32_trials": {
                "systems_per_s": sum_over_ranks(solved["fp32_lu_refinement_fp32_trials"]) /
                                 (ms_trial32 * 1e-3),
                "ms_per_step": ms_trial32, "solved": solved["fp32_lu_refinement_fp32_trials"],
                "fp64_oracle_max_rel_err": fp64_err["fp32_lu_refinement_fp32_trials"],
                "departure": "trial increments alpha d in Float32, measured slope from the held "
                             "residual (Float32 fold); residuals, norms and tests Float64"},
            "chosen_over_plain": value / plain_value,
        },
        "e2e": {"value": e2e_value, "unit": "systems/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e,
                "api": "gsb_solve_batch_host (pinned host X, P, S; chunks of 262,144 systems)",
                "timer": "host clock around the blocking call, median of the steps"},
        "gpu_launches": args.steps,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_profile(args):
    """Solves of one form on args.nsys systems, for an ncu capture of the batch kernel."""
    import torch

    import gsb200 as G

    if args.profile == "predict":
        # the warm-start network's prediction for args.nsys states (untrained weights)
        from workloads import c3_states

        net = G.MlpWarmStart(G.IrkHenonHeiles(0.1), seed=0)
        st_h = c3_states(args.nsys, stream=1)
        net.set_normalisation(st_h, net.stage_guess(st_h))
        S_ = torch.tensor(st_h, device="cuda")
        ms = _events_ms(lambda: net.predict(S_), args.steps, args.warmup,
                        torch.cuda.current_stream())
        print(json.dumps({"profile": "predict", "nsys": args.nsys, "ms_per_step": ms,
                          "err": int(net.err.item())}))
        return
    if args.profile == "mlp":
        # gradient steps of the warm-start network on args.nsys states (random targets)
        from workloads import c3_states

        net = G.MlpWarmStart(G.IrkHenonHeiles(0.1), seed=0)
        st_h = c3_states(args.nsys, stream=1)
        net.set_normalisation(st_h, net.stage_guess(st_h))
        S_ = torch.tensor(st_h, device="cuda")
        T_ = torch.randn(args.nsys, 12, dtype=torch.float32, device="cuda")
        for _ in range(args.warmup + args.steps):
            net.gradient(S_, T_)
        torch.cuda.synchronize()
        print(json.dumps({"profile": "mlp", "nsys": args.nsys, "err": int(net.err.item())}))
        return
    if args.profile == "irk":
        from workloads import c3

        X0_h, P_h = c3(args.nsys)
        prob = G.NonlinearProblem(G.IrkHenonHeiles(0.1))
        m = G.Newton(globalization=G.Backtracking())
    elif args.profile == "lm":
        from workloads import c2

        X0_h, P_h, t = c2(args.nsys)
        prob = G.LeastSquaresProblem(G.ExpSum3(t))
        m = G.Newton(linsolve=G.QRFactorization(), globalization=G.LevenbergMarquardt())
    else:
        from workloads import cubic_affine

        n = args.n
        X0_h, P_h = (workload(0, args.nsys) if n == N_UNKNOWNS
                     else cubic_affine(n, args.nsys, n + 1.0, 4))
        prob = G.NonlinearProblem(G.CubicAffine(n))
        plain, mixed = methods(G)
        m = mixed if args.profile == "mixed" else plain
    X0 = torch.tensor(X0_h, device="cuda")
    P = G.PerSystem(torch.tensor(P_h, device="cuda"))
    if args.profile == "shared":
        # BatchParams: the first system's A shared by the batch, every system's own b
        n = X0_h.shape[1]
        A = torch.tensor(P_h[0, :n * n].reshape(n, n).T.copy(), device="cuda")
        P = G.BatchParams(A, torch.tensor(P_h[:, n * n:].copy(), device="cuda"))
    X = torch.empty_like(X0)
    S = G.status_buffer(args.nsys)
    stream = torch.cuda.current_stream()

    def step():
        X.copy_(X0)
        G.solve_batch(X, S, prob, m, P, options=options(G))

    ms = _events_ms(step, args.steps, args.warmup, stream)
    st = G.statuses(S)
    print(json.dumps({"profile": args.profile, "nsys": args.nsys, "ms_per_step": ms,
                      "systems_per_s": args.nsys / (ms * 1e-3),
                      "codes": np.bincount(st["code"], minlength=6).tolist()}))


# ─── the other configurations, one GPU: c0 (n = 3), c2 (least squares), c4 (ragged) ─────────


def lm_flops_per_system(m, n, iterations, failures):
    """Operations of the Levenberg–Marquardt solve of the exponential-sum fit (an `exp` counts
    one), from the oracle's per-system counts: one Jacobian pass per step (rows by the dual
    rules, J'F, ‖J‖, the stacked Givens reduction) and one trial per step or rejected trial (the
    damped triangle, back substitution, the predicted reduction, a residual evaluation)."""
    row_f = 9 + 3                                     # residual row with its three exps
    rot = 6 * n + 6 * n * (n - 1) // 2 + 6 * n         # one row rotated into the triangle
    jpass = m * (row_f + 6 + 4 * n) + (m - n) * rot + n * rot
    trial = n * rot // 2 + n * n + 4 * n + m * (row_f + 2)
    return iterations * jpass + (iterations + failures) * trial


def _events_ms(fn, steps, warmup, stream):
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _cpu_sample(solve_sample, sample, label):
    """Time the oracle on `sample` systems until about 10 s have passed."""
    from oracle import oracle_py as O

    nt = O.max_threads()
    reps, t_tot = 0, 0.0
    while t_tot < 10.0 and reps < 40:
        t0 = time.perf_counter()
        solve_sample(nt)
        t_tot += time.perf_counter() - t0
        reps += 1
    return {"value": sample * reps / t_tot, "unit": "systems/s", "cores": nt, "kind": "port",
            "sample": f"{reps} x {sample} systems of {label}, {nt} threads, {t_tot:.1f} s"}


def _roof(bytes_total, flops, kms, peaks, hbm_peak, hbm_src, kernel):
    t_bytes = bytes_total / (hbm_peak * 1e9)
    t_flops = flops / (peaks["fp64"] * 1e12)
    gbs = bytes_total / (kms * 1e-3) / 1e9
    tf = flops / (kms * 1e-3) / 1e12
    if t_bytes >= t_flops:
        r = {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
             "frac": gbs / hbm_peak, "peak_source": hbm_src}
    else:
        r = {"bound": "fp64", "achieved": tf, "peak": peaks["fp64"], "unit": "TFLOP/s",
             "frac": tf / peaks["fp64"], "peak_source": "measured (FP64 FMA probe, libgsbpeak)"}
    r.update(traffic=None, kernel=kernel, kernel_ms=kms, fp64_frac=tf / peaks["fp64"],
             hbm_frac=gbs / hbm_peak, flops_per_launch=flops, bytes_per_launch=bytes_total)
    return r


def run_c3(args, opts, hbm_peak, hbm_src, peaks):
    """The stage systems: plain Newton from Z = 0 against the learned warm start (the network
    trained first, on 2,097,152 plain-solver solutions of a disjoint draw; its training time is
    reported, not timed in the step)."""
    import torch

    import gsb200 as G
    from oracle import oracle_py as O
    from workloads import c3, c3_states

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    nsys = args.nsys if args.nsys != NSYS else 262144
    fam = G.IrkHenonHeiles(0.1)
    prob = G.NonlinearProblem(fam)
    plain = G.Newton(globalization=G.Backtracking())
    ntr = 2097152
    tr = c3_states(ntr, stream=1)
    Ztr = torch.zeros(ntr, 12, dtype=torch.float64, device=dev)
    G.solve_batch(Ztr, G.status_buffer(ntr), prob, plain,
                  G.PerSystem(torch.tensor(tr, device=dev)), options=opts)
    net = G.MlpWarmStart(fam, seed=0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = net.train(tr, Ztr.cpu().numpy(), epochs=80, batch=8192, lr=5e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    X0_h, P_h = c3(nsys)
    X0 = torch.tensor(X0_h, device=dev)
    P = torch.tensor(P_h, device=dev)
    ps = G.PerSystem(P)
    X = torch.empty_like(X0)
    S = G.status_buffer(nsys)

    def step_plain():
        X.copy_(X0)
        G.solve_batch(X, S, prob, plain, ps, options=opts)

    Xw = torch.empty_like(X0)
    acc_last = {}

    def step_warm():
        Z, acc = net.warm_start(P, X0)
        Xw.copy_(Z)
        G.solve_batch(Xw, S, prob, plain, ps, options=opts)
        acc_last["acc"] = acc

    xo, so = O.solve_batch(prob, plain, X0_h.copy(), P_h, opts)
    forms = {}
    with Clocks(0) as clk:
        for name, step, xbuf in (("plain_fp64", step_plain, X), ("mlp_warm_start", step_warm, Xw)):
            ms = _events_ms(step, args.steps, args.warmup, stream)
            step()
            st = G.statuses(S)
            err = rel_err(xbuf.cpu().numpy(), xo)
            ok = (st["code"] == so["code"]) & (err <= REL_TOL)
            forms[name] = {"systems_per_s": float(np.sum(ok)) / (ms * 1e-3), "ms_per_step": ms,
                           "solved": int(np.sum(ok)), "mean_iterations": float(st["iterations"].mean()),
                           "fp64_oracle_max_rel_err": float(err.max())}
        # where the warm step's time goes: the network's prediction, the accept-if-better gate
        # and the Newton solve from the chosen starts
        Z0 = net.predict(P)
        Zs, _ = net.select(P, Z0, X0)

        def solve_from_warm():
            Xw.copy_(Zs)
            G.solve_batch(Xw, S, prob, plain, ps, options=opts)

        forms["mlp_warm_start"]["phases_ms"] = {
            "predict": _events_ms(lambda: net.predict(P), args.steps, args.warmup, stream),
            "select": _events_ms(lambda: net.select(P, Z0, X0), args.steps, args.warmup, stream),
            "solve": _events_ms(solve_from_warm, args.steps, args.warmup, stream)}
    clocks = clk.summary()
    forms["mlp_warm_start"]["fallback_rate"] = 1.0 - float(acc_last["acc"].float().mean().item())
    forms["mlp_warm_start"]["training"] = {"samples": ntr, "epochs": 80, "batch": 8192,
                                           "seconds": t_train, "loss_first": hist[0],
                                           "loss_last": hist[-1]}
    chosen = max(("plain_fp64", "mlp_warm_start"), key=lambda k: forms[k]["systems_per_s"])
    forms["chosen_over_plain"] = forms[chosen]["systems_per_s"] / forms["plain_fp64"]["systems_per_s"]
    value = forms[chosen]["systems_per_s"]
    ms = forms[chosen]["ms_per_step"]
    kms = forms["plain_fp64"]["ms_per_step"] - _events_ms(lambda: X.copy_(X0), 20, 2, stream)
    flops = float(np.sum(flops_per_system(12, so["iterations"].astype(np.int64),
                                          1 + _trials(so))))
    bytes_total = (32 + 96 + 96 + 72) * nsys
    x_pin = torch.from_numpy(X0_h).pin_memory()
    p_pin = torch.from_numpy(P_h).pin_memory()
    x_out = torch.empty_like(x_pin).pin_memory()
    s_out = torch.empty((nsys, 72), dtype=torch.uint8).pin_memory()
    Pe, Xe = torch.empty_like(P), torch.empty_like(X0)

    def e2e():
        Pe.copy_(p_pin, non_blocking=True)
        Xe.copy_(x_pin, non_blocking=True)
        if chosen == "mlp_warm_start":
            Z, _ = net.warm_start(Pe, Xe)
            Xe.copy_(Z)
        G.solve_batch(Xe, S, prob, plain, G.PerSystem(Pe), options=opts)
        x_out.copy_(Xe, non_blocking=True)
        s_out.copy_(S, non_blocking=True)

    ms_e2e = _events_ms(e2e, max(1, args.steps // 2), 1, stream)
    sample = min(nsys, 65536)
    cpu = _cpu_sample(lambda nt: O.solve_batch(prob, plain, X0_h[:sample].copy(), P_h[:sample],
                                               opts, nthreads=nt), sample, "c3, plain from Z = 0")
    line = {
        "metric": METRIC, "value": value, "unit": "systems/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded; the configuration's shapes and distributions)",
        "config": {"workload": f"Gauss-3 stage systems of the Hénon–Heiles field, h = 0.1, n = 12, "
                               f"{nsys} systems, Newton + LU + Backtracking; learned warm start "
                               "(4-128-128-12 MLP, BF16 tcgen05) with the accept-if-better gate",
                   "chosen_form": chosen, "global_batch": nsys, "parallelism": "one GPU",
                   "l2": "inputs fit in L2; a step rewrites X from X0"},
        "forms": forms,
        "e2e": {"value": value * ms / ms_e2e, "unit": "systems/s",
                "h2d_bytes_per_step": int(X0_h.nbytes + P_h.nbytes),
                "d2h_bytes_per_step": int(X0_h.nbytes + nsys * 72), "ms_per_step": ms_e2e},
        "gpu_launches": args.steps * (3 if chosen == "mlp_warm_start" else 1),
        "roofline": _roof(bytes_total, flops, kms, peaks, hbm_peak, hbm_src,
                          "warp_kernel<WarpIrk, 16, fused, FP64>"),
        "cpu_baseline": cpu,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def run_workload(args):
    import torch

    import gsb200 as G
    from oracle import oracle_py as O

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    opts = options(G)
    hbm_peak, hbm_src = measured_peaks()
    peaks = fp_peaks()
    forms = {}

    if args.workload == "c3":
        return run_c3(args, opts, hbm_peak, hbm_src, peaks)
    if args.workload in ("c0", "c2"):
        if args.workload == "c0":
            from workloads import c0

            nsys = args.nsys if args.nsys != NSYS else 65536
            X0_h, P_h = c0(nsys)
            prob = G.NonlinearProblem(G.CubicAffine(3))
            method = G.Newton(globalization=G.Backtracking())
            workload = (f"cubic-affine n=3, {nsys} systems, A = 4I + 0.5 N(0,1), Newton + LU + "
                        "Backtracking FP64, f_abstol 1e-12, max_iterations 50")
            kernel = "newton_kernel<CubicAffine<3>, fused, FP64>"
        else:
            from workloads import c2

            nsys = args.nsys if args.nsys != NSYS else 524288
            X0_h, P_h, t = c2(nsys)
            prob = G.LeastSquaresProblem(G.ExpSum3(t))
            method = G.Newton(linsolve=G.QRFactorization(), globalization=G.LevenbergMarquardt())
            workload = (f"exponential-sum least squares m=64 n=6, {nsys} systems, "
                        "LevenbergMarquardt (stacked QR), FP64, max_iterations 50")
            kernel = "lm_kernel<ExpSum3<64>, fused>"
        X0 = torch.tensor(X0_h, device=dev)
        P = torch.tensor(P_h, device=dev)
        X = torch.empty_like(X0)
        S = G.status_buffer(nsys)
        ps = G.PerSystem(P)

        def step():
            X.copy_(X0)
            G.solve_batch(X, S, prob, method, ps, options=opts)

        # correctness against the oracle (untimed), on the whole batch for c0 and on a sample
        # of 65,536 systems for c2 (codes equal and |F| within the fit's 1e-10 envelope)
        step()
        st = G.statuses(S)
        x = X.cpu().numpy()
        ns = nsys if args.workload == "c0" else min(nsys, 65536)
        xo, so = O.solve_batch(prob, method, X0_h[:ns].copy(), P_h[:ns], opts)
        if args.workload == "c0":
            ok = (st["code"][:ns] == so["code"]) & (rel_err(x[:ns], xo) <= REL_TOL)
            flops = float(np.sum(flops_per_system(3, so["iterations"].astype(np.int64),
                                                  1 + _trials(so))))
            bytes_total = bytes_per_system(3) * nsys
        else:
            # solved: the oracle's code and the iterate within 1e-10 of the oracle's
            ok = (st["code"][:ns] == so["code"]) & (rel_err(x[:ns], xo) <= REL_TOL)
            flops = float(np.mean(lm_flops_per_system(
                64, 6, st["iterations"].astype(np.int64), st["step_failures"].astype(np.int64))))
            flops *= nsys
            bytes_total = (512 + 48 + 48 + 72) * nsys
        solved_frac = float(np.mean(ok))
        with Clocks(0) as clk:
            ms = _events_ms(step, args.steps, args.warmup, stream)
            if args.workload == "c2":
                # the other forms of the fit: FP64 with unfused arithmetic (the oracle's rounding,
                # bit for bit) and the FP32 stacked factor with FP64 refinement
                others = {
                    "fp64_unfused": G.Newton(linsolve=G.QRFactorization(),
                                             globalization=G.LevenbergMarquardt(),
                                             arithmetic="unfused"),
                    "fp32_qr_refinement": G.Newton(linsolve=G.QRFactorization("float32"),
                                                   globalization=G.LevenbergMarquardt()),
                }
                for fname, mo in others.items():
                    def step_o(mo=mo):
                        X.copy_(X0)
                        G.solve_batch(X, S, prob, mo, ps, options=opts)

                    ms_o = _events_ms(step_o, args.steps, args.warmup, stream)
                    step_o()
                    st_o = G.statuses(S)
                    x_o = X.cpu().numpy()
                    ok_o = (st_o["code"][:ns] == so["code"]) & (rel_err(x_o[:ns], xo) <= REL_TOL)
                    forms[fname] = {
                        "systems_per_s": float(np.mean(ok_o)) * nsys / (ms_o * 1e-3),
                        "ms_per_step": ms_o, "solved_fraction": float(np.mean(ok_o)),
                        "oracle_checked_systems": ns, "method": mo}
        clocks = clk.summary()
        # the end-to-end leg runs the form with the most systems solved per second
        chosen_m = method
        best = solved_frac * nsys / (ms * 1e-3)
        for f in forms.values():
            if f["systems_per_s"] > best:
                best, chosen_m = f["systems_per_s"], f["method"]
        value = solved_frac * nsys / (ms * 1e-3)
        # the solve alone: the step minus the copy of the start iterates
        kms = ms - _events_ms(lambda: X.copy_(X0), 20, 2, stream)
        # end to end: pinned host inputs in, solutions and statuses out, every step
        x_pin = torch.from_numpy(X0_h).pin_memory()
        p_pin = torch.from_numpy(P_h).pin_memory()
        x_out = torch.empty_like(x_pin).pin_memory()
        s_out = torch.empty((nsys, 72), dtype=torch.uint8).pin_memory()
        Xe, Pe = torch.empty_like(X0), torch.empty_like(P)

        def e2e():
            Xe.copy_(x_pin, non_blocking=True)
            Pe.copy_(p_pin, non_blocking=True)
            G.solve_batch(Xe, S, prob, chosen_m, G.PerSystem(Pe), options=opts)
            x_out.copy_(Xe, non_blocking=True)
            s_out.copy_(S, non_blocking=True)

        ms_e2e = _events_ms(e2e, max(1, args.steps // 2), 1, stream)
        h2d, d2h = X0_h.nbytes + P_h.nbytes, X0_h.nbytes + nsys * 72
        sample = min(nsys, 65536 if args.workload == "c0" else 8192)
        cpu = _cpu_sample(lambda nt: O.solve_batch(prob, method, X0_h[:sample].copy(),
                                                   P_h[:sample], opts, nthreads=nt),
                          sample, args.workload)
        forms["fp64"] = {"systems_per_s": value, "ms_per_step": ms, "solved_fraction": solved_frac,
                         "oracle_checked_systems": ns}
        launches = args.steps
        chosen = "fp64"
        for fname in ("fp64_unfused", "fp32_qr_refinement"):
            if fname in forms and forms[fname]["systems_per_s"] > forms[chosen]["systems_per_s"]:
                chosen = fname
        if chosen != "fp64":
            value = forms[chosen]["systems_per_s"]
            ms = forms[chosen]["ms_per_step"]
        for f in forms.values():
            f.pop("method", None)
        if args.workload == "c2":
            forms["chosen"] = chosen
            forms["chosen_over_plain"] = value / forms["fp64"]["systems_per_s"]
    else:
        from workloads import c4

        nsys = args.nsys if args.nsys != NSYS else 4194304
        sizes_h, X0_h, P_h = c4(nsys)
        sizes = torch.tensor(sizes_h, dtype=torch.int32, device=dev)
        X0 = torch.tensor(X0_h, device=dev)
        P = torch.tensor(P_h, device=dev)
        X = torch.empty_like(X0)
        S = G.status_buffer(nsys)
        x_off, p_off = G.ragged_offsets(sizes)
        plain, mixed = methods(G)
        # the oracle, bucket by bucket (untimed)
        n64 = sizes_h.astype(np.int64)
        xo_all = np.empty_like(X0_h)
        so_all = np.zeros(nsys, dtype=G.SOLVER_STATUS_DTYPE)
        xoff_h, poff_h = x_off.cpu().numpy(), p_off.cpu().numpy()
        flops = 0.0
        for n in (2, 3, 4, 6, 8, 12, 16, 24, 32):
            sel = np.flatnonzero(sizes_h == n)
            xi = xoff_h[sel][:, None] + np.arange(n)[None, :]
            pi = poff_h[sel][:, None] + np.arange(n * n + n)[None, :]
            xo, so = O.solve_batch(G.NonlinearProblem(G.CubicAffine(n)), plain, X0_h[xi].copy(),
                                   P_h[pi], opts)
            xo_all[xi] = xo
            so_all[sel] = so
            flops += float(np.sum(flops_per_system(n, so["iterations"].astype(np.int64),
                                                   1 + _trials(so))))
        bytes_total = float(np.sum(8 * n64 + 8 * (n64 * n64 + n64) + 8 * n64 + 72 + 4 + 16))
        # the tables tuned on B200 that the package carries; a form without one is tuned here
        tables, table_source = {}, {}
        for name, m in (("plain_fp64", plain), ("fp32_lu_refinement", mixed)):
            tables[name] = G.tune.tuned_table(m)
            table_source[name] = "committed"
            if tables[name] is None:
                tables[name], _ = G.tune.autotune_uneven(m, options=opts, sample=16384, reps=2)
                table_source[name] = "tuned in this run"

        def solver(m, table):
            def step():
                X.copy_(X0)
                G.solve_batch_uneven(X, S, sizes, P, m, x_off=x_off, p_off=p_off, table=table,
                                     options=opts)
            return step

        with Clocks(0) as clk:
            for name, m in (("plain_fp64", plain), ("fp32_lu_refinement", mixed)):
                step = solver(m, tables[name])
                ms = _events_ms(step, args.steps, args.warmup, stream)
                step()
                st = G.statuses(S)
                x = X.cpu().numpy()
                ok = st["code"] == so_all["code"]
                err = np.zeros(nsys)
                for n in (2, 3, 4, 6, 8, 12, 16, 24, 32):
                    sel = np.flatnonzero(sizes_h == n)
                    xi = xoff_h[sel][:, None] + np.arange(n)[None, :]
                    err[sel] = rel_err(x[xi], xo_all[xi])
                ok &= err <= REL_TOL
                forms[name] = {"systems_per_s": float(np.sum(ok)) / (ms * 1e-3), "ms_per_step": ms,
                               "solved": int(np.sum(ok)), "fp64_oracle_max_rel_err": float(err.max()),
                               "table": [list(t) for t in tables[name]],
                               "table_source": table_source[name]}
            # the baseline of the comparison: plain FP64 with one ordinary launch per size
            # bucket (each bucket a uniform batch of its own, laid out beforehand; no graph, no
            # persistent kernels, each call waiting for its kernel as solve_batch! does)
            buckets = []
            for n in (2, 3, 4, 6, 8, 12, 16, 24, 32):
                sel = np.flatnonzero(sizes_h == n)
                if sel.size == 0:
                    continue
                xi = xoff_h[sel][:, None] + np.arange(n)[None, :]
                pi = poff_h[sel][:, None] + np.arange(n * n + n)[None, :]
                x0n = torch.tensor(X0_h[xi], device=dev)
                buckets.append((n, sel, xi, x0n, torch.empty_like(x0n),
                                torch.tensor(P_h[pi], device=dev), G.status_buffer(sel.size),
                                G.NonlinearProblem(G.CubicAffine(n))))

            def per_bucket():
                for n, sel, xi, x0n, xn, pn, sn, pb in buckets:
                    xn.copy_(x0n)
                    G.solve_batch(xn, sn, pb, plain, G.PerSystem(pn), options=opts)

            ms_b = _events_ms(per_bucket, args.steps, args.warmup, stream)
            per_bucket()
            okb = np.zeros(nsys, dtype=bool)
            errb = np.zeros(nsys)
            for n, sel, xi, x0n, xn, pn, sn, pb in buckets:
                stb = G.statuses(sn)
                errb[sel] = rel_err(xn.cpu().numpy(), xo_all[xi])
                okb[sel] = (stb["code"] == so_all["code"][sel]) & (errb[sel] <= REL_TOL)
            forms["plain_fp64_per_bucket_launches"] = {
                "systems_per_s": float(np.sum(okb)) / (ms_b * 1e-3), "ms_per_step": ms_b,
                "solved": int(np.sum(okb)), "fp64_oracle_max_rel_err": float(errb.max()),
                "launches": len(buckets),
                "layout": "each bucket laid out as a uniform batch beforehand (not timed)"}
            del buckets
            # what laying a mixed batch out by size costs a caller at the least: one read and
            # one write of its parameter blocks and start iterates (a plain device copy)
            P2, X2 = torch.empty_like(P), torch.empty_like(X0)

            def layout_copy():
                P2.copy_(P)
                X2.copy_(X0)

            ms_lay = _events_ms(layout_copy, args.steps, args.warmup, stream)
            del P2, X2
            forms["plain_fp64_per_bucket_launches"]["layout_copy_ms"] = ms_lay
            forms["plain_fp64_per_bucket_launches"]["systems_per_s_with_layout_copy"] = \
                float(np.sum(okb)) / ((ms_b + ms_lay) * 1e-3)
        clocks = clk.summary()
        chosen = max(("plain_fp64", "fp32_lu_refinement"), key=lambda k: forms[k]["systems_per_s"])
        value = forms[chosen]["systems_per_s"]
        ms = forms[chosen]["ms_per_step"]
        forms["chosen_over_plain"] = value / forms["plain_fp64"]["systems_per_s"]
        forms["chosen_over_per_bucket_launches"] = (
            value / forms["plain_fp64_per_bucket_launches"]["systems_per_s"])
        m_ch = mixed if chosen == "fp32_lu_refinement" else plain
        kms = ms - _events_ms(lambda: X.copy_(X0), 20, 2, stream)
        kernel = "bucketing + 9 persistent bucket kernels (one CUDA graph)"
        x_pin = torch.from_numpy(X0_h).pin_memory()
        p_pin = torch.from_numpy(P_h).pin_memory()
        n_pin = torch.from_numpy(sizes_h).pin_memory()
        x_out = torch.empty_like(x_pin).pin_memory()
        s_out = torch.empty((nsys, 72), dtype=torch.uint8).pin_memory()
        Xe, Pe = torch.empty_like(X0), torch.empty_like(P)
        ne = torch.empty_like(sizes)

        def e2e():
            Xe.copy_(x_pin, non_blocking=True)
            Pe.copy_(p_pin, non_blocking=True)
            ne.copy_(n_pin, non_blocking=True)
            G.solve_batch_uneven(Xe, S, ne, Pe, m_ch, table=tables[chosen], options=opts)
            x_out.copy_(Xe, non_blocking=True)
            s_out.copy_(S, non_blocking=True)

        ms_e2e = _events_ms(e2e, max(1, args.steps // 2), 1, stream)
        h2d, d2h = X0_h.nbytes + P_h.nbytes + sizes_h.nbytes, X0_h.nbytes + nsys * 72
        sample = 131072

        def cpu_solve(nt):
            for n in (2, 3, 4, 6, 8, 12, 16, 24, 32):
                sel = np.flatnonzero(sizes_h[:sample] == n)
                xi = xoff_h[sel][:, None] + np.arange(n)[None, :]
                pi = poff_h[sel][:, None] + np.arange(n * n + n)[None, :]
                O.solve_batch(G.NonlinearProblem(G.CubicAffine(n)), plain, X0_h[xi].copy(),
                              P_h[pi], opts, nthreads=nt)

        cpu = _cpu_sample(cpu_solve, sample, "the ragged batch, plain FP64")
        workload = (f"ragged cubic-affine batch, {nsys} systems, n in {{2,...,32}} with P(n) ∝ 1/n, "
                    "A = (n+1)I + 0.5 N(0,1), Newton + LU + Backtracking, autotuned persistent "
                    "bucket kernels in one CUDA graph")
        launches = args.steps * 13
    line = {
        "metric": METRIC, "value": value, "unit": "systems/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded; the configuration's shapes and distributions)",
        "config": {"workload": workload, "chosen_form": chosen, "global_batch": nsys,
                   "parallelism": "one GPU",
                   "l2": f"inputs of {bytes_total / 1e6:.0f} MB per step exceed the 126 MB L2"
                   if bytes_total > 126e6 else "inputs fit in L2; a step rewrites X from X0"},
        "forms": forms,
        "e2e": {"value": value * ms / ms_e2e, "unit": "systems/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e},
        "gpu_launches": launches,
        "roofline": _roof(bytes_total, flops, kms, peaks, hbm_peak, hbm_src, kernel),
        "cpu_baseline": cpu,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def _trials(so):
    """Line-search trials per system are not in the status; the flop model takes one trial per
    step (the accepted full step of a converging Newton iteration)."""
    return so["iterations"].astype(np.int64)


if __name__ == "__main__":
    main()
