"""Builds libgsb.so (the CUDA kernels and the C-ABI) in this directory, for sm_100a.

Each csrc/*.cu is compiled to an object in parallel (the kernel instantiations are spread over
several translation units), then the objects are linked into one shared library. An object newer
than its source and every header is reused.

python geometricsolvers.jl_b200/build.py [--verbose]
"""

from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libgsb.so")
PEAK_SRC = os.path.join(HERE, "peak", "gsb_peak.cu")
PEAK_OUT = os.path.join(HERE, "peak", "libgsbpeak.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    hs.append(os.path.join(HERE, "..", "include", "gsb.h"))
    return hs


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    files = [os.path.join(CSRC, s) for s in sources()] + _headers()
    return all(os.path.getmtime(f) <= t for f in files)


def _fresh(src: str, obj: str) -> bool:
    """An object is kept when it is newer than its source and every header."""
    if not os.path.exists(obj):
        return False
    t = os.path.getmtime(obj)
    return all(os.path.getmtime(f) <= t for f in [os.path.join(CSRC, src), *_headers()])


def _compile(src: str, verbose: bool, force: bool = True):
    nvcc = os.environ.get("NVCC", "nvcc")
    obj = os.path.join(OBJ, src[:-3] + ".o")
    if not force and not verbose and _fresh(src, obj):
        return src, obj, subprocess.CompletedProcess([], 0, "", "")
    cmd = [nvcc, *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    return src, obj, proc


def build_peak(force: bool = False) -> str:
    """libgsbpeak.so: the FMA-throughput probe that bench.py reads its FP64/FP32 peaks from."""
    if not force and os.path.exists(PEAK_OUT) and os.path.getmtime(PEAK_OUT) >= os.path.getmtime(PEAK_SRC):
        return PEAK_OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, "-O3", "-std=c++17", "--shared", "-Xcompiler", "-fPIC", PEAK_SRC,
           "-o", PEAK_OUT]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("nvcc failed to build libgsbpeak.so")
    return PEAK_OUT


def build(verbose: bool = False, force: bool = False, jobs: int = 0) -> str:
    build_peak(force)
    if not force and up_to_date():
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    jobs = jobs or max(1, min(len(sources()), os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as pool:
        results = list(pool.map(lambda s: _compile(s, verbose, force), sources()))
    failed = [r for r in results if r[2].returncode != 0]
    for src, _, proc in results:
        if verbose or proc.returncode != 0:
            sys.stderr.write(f"== {src}\n{proc.stdout}{proc.stderr}")
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(r[0] for r in failed))
    nvcc = os.environ.get("NVCC", "nvcc")
    link = [nvcc, *ARCH, "--shared", "-o", OUT + ".tmp", *[r[1] for r in results]]
    proc = subprocess.run(link, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("nvcc failed to link libgsb.so")
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
