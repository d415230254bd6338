"""Build recipe for libkate_b200.so (sm_100a) and the CPU checkers.

``python -m kate_b200.build`` compiles every source in ``kate_b200/csrc`` with
nvcc for ``sm_100a`` into ``kate_b200/libkate_b200.so`` (objects go to
``kate_b200/_build``). Sources are rebuilt only when they, a header, or the
flags changed.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libkate_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
CUFLAGS = ARCH + ["-lineinfo", "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers_digest():
    h = hashlib.sha256()
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in sorted(os.listdir(d)):
            p = os.path.join(d, f)
            if os.path.isfile(p) and f.endswith((".h", ".hpp", ".cuh")):
                h.update(open(p, "rb").read())
    return h.hexdigest()


def _compile(src: str, hdr: str, verbose: bool) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    flags = COMMON + (CUFLAGS if src.endswith(".cu") else [])
    if src.endswith(".cpp"):
        flags = flags + ["-x", "cu"] + ARCH  # one toolchain for all sources
    key = hashlib.sha256((open(path, "rb").read().hex() + hdr + " ".join(flags)).encode()).hexdigest()
    stamp = obj + ".key"
    if os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == key:
        return obj
    cmd = [NVCC, *flags, "-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    with open(stamp, "w") as f:
        f.write(key)
    return obj


def build(verbose: bool = False) -> str:
    """Compiles the library; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    hdr = _headers_digest()
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: _compile(s, hdr, verbose), _sources()))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcuda", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def build_oracle(with_ref: bool = True, verbose: bool = False) -> None:
    """Compiles oracle/libkate_oracle.so and, when the reference headers are
    present (the tree in KATE_REF_DIR, default the reference checkout this
    build was written against), oracle/_ref/libkate_ref.so and
    oracle/_ref/libkate_ref_gpu.so (test and measurement infrastructure)."""
    targets = ["oracle"]
    ref_dir = os.environ.get("KATE_REF_DIR", "/root/reference")
    if with_ref and os.path.exists(os.path.join(ref_dir, "Kate.hpp")):
        targets += ["ref", "refgpu", f"REF={ref_dir}"]
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), *targets], capture_output=True, text=True)
    if verbose:
        print(r.stdout, r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")


if __name__ == "__main__":
    print(build(verbose=True))
    build_oracle(verbose=True)
