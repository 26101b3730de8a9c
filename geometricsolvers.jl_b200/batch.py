"""solve_batch and batch_summary over device tensors, through libgsb's C-ABI.

solve_batch(X, S, prob, method, p=None; order, options, **kwargs) -> S      batched.jl:257-287
solve_batch(X, prob, method, p=None; ...) -> ReturnCodeCounts               batched.jl:289-307
solve_batch_uneven(X, S, sizes, P, method; ...) -> S   systems of different sizes in one call
solve_batch_host(X, S, prob, method, p; chunk, ...) -> S   a batch in host memory, pipelined
Like the reference's `_launch!` (src/nonlinear/batched.jl:183-195) every call waits for its
kernel before it returns. Host checks raise before any launch, with the reference's messages.
"""

from __future__ import annotations

import contextlib
import ctypes

import numpy as np

from . import abi
from .api import (
    ArgumentError,
    BatchParams,
    BatchSummary,
    DimensionMismatch,
    NonlinearProblem,
    Options,
    PerSystem,
    ReturnCodeCounts,
    SoA,
    _raise_for,
)


def _tensor(x):
    return x.data if isinstance(x, SoA) else x


def _check_device_f64(t, what):
    import torch

    if not isinstance(t, torch.Tensor):
        raise ArgumentError(f"{what} must be a torch tensor on a CUDA device")
    if not t.is_cuda:
        raise ArgumentError(f"{what} must be on a CUDA device (the batch solver has no host path)")
    if t.dtype != torch.float64:
        raise ArgumentError(f"{what} must be float64")
    if not t.is_contiguous():
        raise ArgumentError(f"{what} must be contiguous")


_abi_cache = {}


def _abi_of(obj):
    """The C-ABI struct of a (frozen, hashable) Newton or Options, built once per distinct
    value: the library only reads it."""
    try:
        return _abi_cache[obj]
    except KeyError:
        if len(_abi_cache) > 256:
            _abi_cache.clear()
        v = _abi_cache[obj] = obj.to_abi()
        return v
    except TypeError:  # not hashable
        return obj.to_abi()


def _resolve_options(options, kwargs):
    """resolve_options, src/nonlinear/solver.jl:391-398: the keywords or an Options, never both."""
    if options is None:
        return Options(**kwargs)
    if kwargs:
        raise ArgumentError("pass either `options` or keyword arguments, not both")
    if not isinstance(options, Options):
        raise ArgumentError("options must be an Options")
    return options


def _is_perm(order, n):
    import torch

    o = order.detach().to("cpu", torch.int64)
    if o.numel() != n:
        return False
    seen = torch.zeros(n, dtype=torch.bool)
    if n == 0:
        return True
    if int(o.min()) < 0 or int(o.max()) >= n:
        return False
    seen[o] = True
    return bool(seen.all())


def _shared_matrix(fam, A, device):
    """The shared matrix of a CubicAffine BatchParams, column-major, as a float64 tensor on the
    device of the batch."""
    import torch

    if fam.family != abi.Family.CUBIC_AFFINE:
        raise ArgumentError("BatchParams takes a CubicAffine family (a shared A, per-system b)")
    if isinstance(A, torch.Tensor):
        if A.device != device:
            raise ArgumentError("the shared matrix must be on the device of X")
        At = A.to(torch.float64)
    else:
        At = torch.as_tensor(np.asarray(A, dtype=np.float64), device=device)
    if tuple(At.shape) != (fam.n, fam.n):
        raise DimensionMismatch(f"the shared matrix must be ({fam.n}, {fam.n}), got {tuple(At.shape)}")
    return At.t().contiguous().reshape(-1)  # column-major: A[i, k] at i + k n


def solve_batch(X, S, prob=None, method=None, p=None, *, order=None, options=None, stream=None,
                _summary=None, **kwargs):
    """Solve every system of X in place (see the module docstring). X is an (nsys, n) float64
    CUDA tensor (Vector{SVector}: one row per system) or SoA of an (n, nsys) tensor; S is a
    (nsys, 72) uint8 tensor of statuses (``status_buffer``). `order` is a permutation of
    0..nsys-1 (an int64 tensor on the device or host)."""
    import torch

    counts_form = isinstance(S, NonlinearProblem)
    if counts_form:  # solve_batch(X, prob, method, p)
        S, prob, method, p = None, S, prob, method
    if not isinstance(prob, NonlinearProblem):
        raise ArgumentError("prob must be a NonlinearProblem or a LeastSquaresProblem")
    fam = prob.family
    Xt = _tensor(X)
    x_layout = abi.GSB_SOA if isinstance(X, SoA) else abi.GSB_AOS
    _check_device_f64(Xt, "X")
    if x_layout == abi.GSB_AOS:
        if Xt.dim() != 2 or Xt.shape[1] != fam.n:
            raise DimensionMismatch(f"X must be (nsys, {fam.n}), got {tuple(Xt.shape)}")
        nsys = Xt.shape[0]
    else:
        if Xt.dim() != 2 or Xt.shape[0] != fam.n:
            raise DimensionMismatch(f"SoA X must be ({fam.n}, nsys), got {tuple(Xt.shape)}")
        nsys = Xt.shape[1]
    # parameters: PerSystem blocks, or BatchParams (a shared A and per-system b) for CubicAffine
    shared_A = None
    if isinstance(p, BatchParams):
        shared_A = _shared_matrix(fam, p.shared, Xt.device)
        p = PerSystem(p.per_system)
    if not isinstance(p, PerSystem):
        raise ArgumentError("p must be a PerSystem of per-system parameter blocks or a BatchParams")
    Pt = _tensor(p.data)
    p_layout = abi.GSB_SOA if isinstance(p.data, SoA) else abi.GSB_AOS
    _check_device_f64(Pt, "PerSystem data")
    npar = fam.n if shared_A is not None else fam.param_count
    plen = Pt.shape[0] if p_layout == abi.GSB_AOS else (Pt.shape[1] if Pt.dim() == 2 else -1)
    if Pt.dim() != 2 or plen != nsys:
        raise DimensionMismatch(
            f"PerSystem parameter length {plen} does not match batch length {nsys}")
    if (Pt.shape[1] if p_layout == abi.GSB_AOS else Pt.shape[0]) != npar:
        raise DimensionMismatch(f"each system takes {npar} parameters")
    if Pt.get_device() != Xt.get_device():
        raise ArgumentError("PerSystem data must be on the device of X")
    order_t = None
    if order is not None:
        order_t = torch.as_tensor(order)
        if order_t.numel() != nsys:
            raise DimensionMismatch(f"order length {order_t.numel()} does not match batch length {nsys}")
        if not _is_perm(order_t, nsys):
            raise ArgumentError(f"order is not a permutation of 0:{nsys - 1}")
        order_t = order_t.to(device=Xt.device, dtype=torch.int64).contiguous()
    opt = _resolve_options(options, kwargs)
    if counts_form:
        S_buf = torch.empty(nsys, dtype=torch.uint8, device=Xt.device)
        s_kind = abi.GSB_CODES
    else:
        if not (isinstance(S, torch.Tensor) and S.dtype == torch.uint8 and S.is_cuda):
            raise ArgumentError("S must be a (nsys, 72) uint8 CUDA tensor (status_buffer)")
        if S.numel() != nsys * 72:
            raise DimensionMismatch(
                f"status vector length {S.numel() // 72} does not match batch length {nsys}")
        if S.get_device() != Xt.get_device():
            raise ArgumentError(
                f"status vector backend {S.device} does not match batch backend {Xt.device}")
        S_buf = S
        s_kind = abi.GSB_STATUS64
    gm = _abi_of(method)
    if nsys == 0:
        return ReturnCodeCounts(0, 0, 0, 0, 0, 0) if counts_form else S
    lib = abi.load_library()
    sh = prob.shared_device(Xt.device)
    gp = prob.to_abi(None if sh is None else sh.data_ptr())
    if shared_A is not None:
        gp.shared, gp.shared_len = shared_A.data_ptr(), shared_A.numel()
    go = _abi_of(opt)
    if stream is None:
        stream = torch.cuda.current_stream(Xt.device)
    tally = abi.GsbTally() if counts_form else None
    # the launch goes to the device of X; a context switch only when it is not the current one
    on_dev = torch.cuda.current_device() == Xt.device.index
    with contextlib.nullcontext() if on_dev else torch.cuda.device(Xt.device):
        st = ctypes.c_void_p(stream.cuda_stream)
        if _summary is not None:
            rc = lib.gsb_solve_batch_summary(
                ctypes.byref(gp), ctypes.byref(gm), ctypes.byref(go), Xt.data_ptr(), x_layout,
                S_buf.data_ptr(), Pt.data_ptr(), p_layout,
                None if order_t is None else order_t.data_ptr(), 0, nsys, st,
                ctypes.byref(_summary))
        else:
            rc = lib.gsb_solve_batch(
                ctypes.byref(gp), ctypes.byref(gm), ctypes.byref(go), Xt.data_ptr(), x_layout,
                S_buf.data_ptr(), s_kind, Pt.data_ptr(), p_layout,
                None if order_t is None else order_t.data_ptr(), 0, nsys, st,
                ctypes.byref(tally) if counts_form else None,
            )
        _raise_for(rc, lib)
        _raise_for(lib.gsb_synchronize(st), lib)
    if counts_form:
        return ReturnCodeCounts(*[int(c) for c in tally.counts])
    return S


def solve_batch_summary(X, S, prob, method, p=None, *, order=None, options=None, stream=None,
                        **kwargs):
    """solve_batch(X, S, prob, method, p; ...) followed by batch_summary(S), with the summary
    reduced by the solve's kernel as it closes the statuses (gsb_solve_batch_summary). Returns
    (S, BatchSummary)."""
    if isinstance(S, NonlinearProblem):
        raise ArgumentError("solve_batch_summary takes a status vector S")
    if nsys_of(X) == 0:
        solve_batch(X, S, prob, method, p, order=order, options=options, stream=stream, **kwargs)
        return S, BatchSummary(0.0, True, 0, 0, 0)
    out = abi.GsbSummary()
    solve_batch(X, S, prob, method, p, order=order, options=options, stream=stream,
                _summary=out, **kwargs)
    return S, BatchSummary(out.fnorm, bool(out.all_converged), int(out.failure_count),
                           int(out.max_iterations), int(out.total_iterations))


def nsys_of(X):
    t = _tensor(X)
    return t.shape[1] if isinstance(X, SoA) else t.shape[0]


def batch_summary(S, stream=None) -> BatchSummary:
    """batch_summary(S), src/nonlinear/batched.jl:80-89, reduced on the device."""
    import torch

    nsys = S.numel() // 72
    if nsys == 0:
        return BatchSummary(0.0, True, 0, 0, 0)
    lib = abi.load_library()
    if stream is None:
        stream = torch.cuda.current_stream(S.device)
    out = abi.GsbSummary()
    with torch.cuda.device(S.device):
        _raise_for(lib.gsb_batch_summary(S.data_ptr(), nsys, ctypes.c_void_p(stream.cuda_stream),
                                         ctypes.byref(out)), lib)
    return BatchSummary(out.fnorm, bool(out.all_converged), int(out.failure_count),
                        int(out.max_iterations), int(out.total_iterations))


_ragged_cache = {}


def ragged_offsets(sizes):
    """The offsets (in doubles) of each system's iterate and cubic-affine parameter block in the
    packed X and P of a ragged batch: exclusive prefix sums of n and n^2 + n."""
    import torch

    n = sizes.to(torch.int64)
    x_off = torch.cumsum(n, 0) - n
    pl = n * n + n
    p_off = torch.cumsum(pl, 0) - pl
    return x_off.contiguous(), p_off.contiguous()


def solve_batch_uneven(X, S, sizes, P, method, *, x_off=None, p_off=None, table=None,
                       options=None, stream=None, **kwargs):
    """Solve a ragged batch of cubic-affine systems in place: system s has sizes[s] unknowns
    (from {2, 3, 4, 6, 8, 12, 16, 24, 32}); its iterate is X[x_off[s] : x_off[s] + n] of the
    packed float64 vector X and its parameter block (A column-major, then b) is P[p_off[s] :
    p_off[s] + n^2 + n]. S is a (nsys, 72) uint8 status tensor, or None for the count form (the
    six return-code counts are returned). `table` is a list of nine (threads_per_system,
    ctas_per_sm, systems_per_cta) triples (or pairs, systems_per_cta 0), one per size (see
    ``tune.autotune_uneven``); None takes the table tuned on B200 for the method's form, which
    the package carries, or the library's defaults where it has none.
    The offsets default to the back-to-back packing of ``ragged_offsets``."""
    import torch

    _check_device_f64(X, "X")
    _check_device_f64(P, "P")
    if X.dim() != 1 or P.dim() != 1:
        raise DimensionMismatch("X and P of a ragged batch are packed 1-D vectors")
    if not (isinstance(sizes, torch.Tensor) and sizes.dim() == 1):
        raise ArgumentError("sizes must be a 1-D integer tensor")
    nsys = sizes.numel()
    n_dev = sizes.to(device=X.device, dtype=torch.int32).contiguous()
    if x_off is None or p_off is None:
        # The sizes and offsets go into buffers kept per batch length and device, rewritten on
        # every call, so that repeated calls pass the same pointers and replay one graph.
        key = (nsys, str(X.device))
        if _ragged_cache.get("key") != key:
            _ragged_cache.clear()
            _ragged_cache.update(key=key,
                                 n=torch.empty(nsys, dtype=torch.int32, device=X.device),
                                 x=torch.empty(nsys, dtype=torch.int64, device=X.device),
                                 p=torch.empty(nsys, dtype=torch.int64, device=X.device))
        _ragged_cache["n"].copy_(n_dev)
        xo, po = ragged_offsets(n_dev)
        _ragged_cache["x"].copy_(xo)
        _ragged_cache["p"].copy_(po)
        n_dev = _ragged_cache["n"]
        x_off = _ragged_cache["x"] if x_off is None else x_off
        p_off = _ragged_cache["p"] if p_off is None else p_off
    x_off = torch.as_tensor(x_off).to(device=X.device, dtype=torch.int64).contiguous()
    p_off = torch.as_tensor(p_off).to(device=X.device, dtype=torch.int64).contiguous()
    if x_off.numel() != nsys or p_off.numel() != nsys:
        raise DimensionMismatch("x_off and p_off must have one entry per system")
    if nsys:
        n64 = n_dev.to(torch.int64)
        if int((x_off + n64).max()) > X.numel() or int(x_off.min()) < 0:
            raise DimensionMismatch("an iterate reaches outside X")
        if int((p_off + n64 * n64 + n64).max()) > P.numel() or int(p_off.min()) < 0:
            raise DimensionMismatch("a parameter block reaches outside P")
    opt = _resolve_options(options, kwargs)
    counts_form = S is None
    if counts_form:
        S_buf = torch.empty(nsys, dtype=torch.uint8, device=X.device)
        s_kind = abi.GSB_CODES
    else:
        if not (isinstance(S, torch.Tensor) and S.dtype == torch.uint8 and S.is_cuda):
            raise ArgumentError("S must be a (nsys, 72) uint8 CUDA tensor (status_buffer)")
        if S.numel() != nsys * 72:
            raise DimensionMismatch(
                f"status vector length {S.numel() // 72} does not match batch length {nsys}")
        S_buf = S
        s_kind = abi.GSB_STATUS64
    if table is None:
        from .tune import tuned_table

        table = tuned_table(method)  # the committed table of the method's form, if any
    tab = None
    if table is not None:
        if len(table) != abi.GSB_UNEVEN_BUCKETS:
            raise ArgumentError(f"table takes {abi.GSB_UNEVEN_BUCKETS} entries")
        rows = []
        for t in table:
            t = tuple(int(v) for v in t)
            if len(t) not in (2, 3):
                raise ArgumentError("a table entry is (threads_per_system, ctas_per_sm"
                                    "[, systems_per_cta])")
            rows.append(abi.GsbBucketConfig(*(t + (0,) * (3 - len(t)))))
        tab = (abi.GsbBucketConfig * abi.GSB_UNEVEN_BUCKETS)(*rows)
    gm, go = method.to_abi(), opt.to_abi()
    if nsys == 0:
        return ReturnCodeCounts(0, 0, 0, 0, 0, 0) if counts_form else S
    lib = abi.load_library()
    if stream is None:
        stream = torch.cuda.current_stream(X.device)
    tally = abi.GsbTally()
    with torch.cuda.device(X.device):
        rc = lib.gsb_solve_batch_uneven(
            ctypes.byref(gm), ctypes.byref(go), X.data_ptr(), S_buf.data_ptr(), s_kind,
            P.data_ptr(), n_dev.data_ptr(), x_off.data_ptr(), p_off.data_ptr(), nsys,
            None if tab is None else ctypes.cast(tab, ctypes.c_void_p),
            ctypes.c_void_p(stream.cuda_stream), ctypes.byref(tally))
        _raise_for(rc, lib)
    if counts_form:
        return ReturnCodeCounts(*[int(c) for c in tally.counts])
    return S


def solve_batch_host(X, S, prob, method, p, *, chunk=0, options=None, device=None, **kwargs):
    """Solve a batch whose X ((nsys, n) float64), S ((nsys, 72) uint8 statuses, or None for
    the count form) and PerSystem parameters live in host memory (pin them with
    ``tensor.pin_memory()`` for overlapping copies): the batch streams through the device in
    chunks, the copies in both directions overlapping the solves. Returns S or the counts."""
    import torch

    if not isinstance(prob, NonlinearProblem):
        raise ArgumentError("prob must be a NonlinearProblem or a LeastSquaresProblem")
    fam = prob.family
    for t, what in ((X, "X"),):
        if not (isinstance(t, torch.Tensor) and t.device.type == "cpu" and t.dtype == torch.float64
                and t.is_contiguous()):
            raise ArgumentError(f"{what} must be a contiguous float64 host tensor")
    if X.dim() != 2 or X.shape[1] != fam.n:
        raise DimensionMismatch(f"X must be (nsys, {fam.n}), got {tuple(X.shape)}")
    nsys = X.shape[0]
    device = torch.device(device or "cuda")
    shared_A = None
    if isinstance(p, BatchParams):  # the shared A goes to the device once, b streams per chunk
        A = p.shared.cpu() if isinstance(p.shared, torch.Tensor) else p.shared
        shared_A = _shared_matrix(fam, A, torch.device("cpu")).to(device)
        p = PerSystem(p.per_system)
    if not isinstance(p, PerSystem):
        raise ArgumentError("p must be a PerSystem of per-system parameter blocks or a BatchParams")
    Pt = p.data
    if not (isinstance(Pt, torch.Tensor) and Pt.device.type == "cpu" and Pt.dtype == torch.float64
            and Pt.is_contiguous() and Pt.dim() == 2):
        raise ArgumentError("PerSystem data must be a contiguous (nsys, np) float64 host tensor")
    if Pt.shape[0] != nsys:
        raise DimensionMismatch(f"PerSystem parameter length {Pt.shape[0]} does not match batch length {nsys}")
    npar = fam.n if shared_A is not None else fam.param_count
    if Pt.shape[1] != npar:
        raise DimensionMismatch(f"each system takes {npar} parameters")
    opt = _resolve_options(options, kwargs)
    counts_form = S is None
    if counts_form:
        S_buf = torch.empty(nsys, dtype=torch.uint8)
        s_kind = abi.GSB_CODES
    else:
        if not (isinstance(S, torch.Tensor) and S.dtype == torch.uint8 and S.device.type == "cpu"):
            raise ArgumentError("S must be a (nsys, 72) uint8 host tensor")
        if S.numel() != nsys * 72:
            raise DimensionMismatch(f"status vector length {S.numel() // 72} does not match batch length {nsys}")
        S_buf, s_kind = S, abi.GSB_STATUS64
    gm, go = method.to_abi(), opt.to_abi()
    if nsys == 0:
        return ReturnCodeCounts(0, 0, 0, 0, 0, 0) if counts_form else S
    lib = abi.load_library()
    sh = prob.shared_device(device)
    gp = prob.to_abi(None if sh is None else sh.data_ptr())
    if shared_A is not None:
        gp.shared, gp.shared_len = shared_A.data_ptr(), shared_A.numel()
    tally = abi.GsbTally()
    with torch.cuda.device(device):
        _raise_for(lib.gsb_solve_batch_host(
            ctypes.byref(gp), ctypes.byref(gm), ctypes.byref(go), X.data_ptr(), S_buf.data_ptr(),
            s_kind, Pt.data_ptr(), nsys, int(chunk), ctypes.byref(tally)), lib)
    if counts_form:
        return ReturnCodeCounts(*[int(c) for c in tally.counts])
    return S
