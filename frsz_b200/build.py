"""Build libfrsz2_b200.so in-tree for sm_100a (nvcc, no JIT cache).

The shared library sits next to this file so it travels with the repository
snapshot; ``python -m frsz_b200.build`` rebuilds it when a source is newer.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfrsz2_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]

# translation units of the library (headers are tracked for staleness only);
# compiled in parallel, then linked
SOURCES = ["frsz2_capi.cu", "frsz2_fast_f32.cu", "frsz2_fast_f64.cu", "frsz2_fast_small_f32.cu",
           "frsz2_fast_small_f64.cu", "frsz2_batch.cu", "frsz2_batch_f32.cu",
           "frsz2_batch_f64.cu", "frsz2_batch_static.cu", "frsz2_krylov.cu",
           "frsz2_serve.cu", "frsz1_legacy.cu", "frsz2_blockwise_f32.cu", "frsz2_blockwise_f64.cu",
           "frsz2_fast_mis_f32.cu", "frsz2_fast_mis_f64.cu",
           "frsz2_blockvec_f32.cu", "frsz2_blockvec_f64.cu", "frsz2_chunked_f32.cu", "frsz2_chunked_f64.cu",
           "frsz2_fast_gen_f32.cu", "frsz2_fast_gen_f64.cu"] + \
          [f"frsz2_bwc_{t}_e{e}.cu" for t in ("f64", "f32") for e in (3, 5, 6, 7, 12)]
OBJDIR = os.path.join(HERE, "_build")


def _sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def _deps():
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "frsz2_b200.h"))
    return deps


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in _deps() if os.path.exists(d))


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _obj(src: str) -> str:
    return os.path.join(OBJDIR, os.path.basename(src).replace(".cu", ".o"))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the stale objects (a source or any header newer than its
    object), at most one nvcc per host core, then link."""
    if not force and not stale():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include")]
    flags = [f for f in NVCC_FLAGS if f != "-shared"]
    headers = [d for d in _deps() if not d.endswith(".cu") and os.path.exists(d)]
    newest_header = max(os.path.getmtime(h) for h in headers)
    todo, objs = [], []
    for src in _sources():
        obj = _obj(src)
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), newest_header):
            todo.append((src, obj))
    # heaviest first (the fp64 instance files), so the longest compiles start early
    todo.sort(key=lambda so: -os.path.getsize(so[0]) - (10_000 if "f64" in so[0] else 0))
    running = []
    jobs = max(1, os.cpu_count() or 1)

    def reap(block: bool):
        for p, cmd in list(running):
            if block or p.poll() is not None:
                if p.wait() != 0:
                    raise subprocess.CalledProcessError(p.returncode, cmd)
                running.remove((p, cmd))
                if not block:
                    return

    for src, obj in todo:
        while len(running) >= jobs:
            reap(False)
            if len(running) >= jobs:
                import time

                time.sleep(0.2)
        cmd = [nvcc(), *ARCH, *flags, *inc, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        running.append((subprocess.Popen(cmd), cmd))
    while running:
        reap(True)
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", tmp, *objs], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
