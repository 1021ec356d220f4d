"""Build the in-tree CUDA library ``coqui_b200/_lib/libcoqui_b200.so`` for sm_100a.

Each ``csrc/*.cu`` is compiled with nvcc (in parallel) and linked against the CUDA runtime
alone (every product and factorisation is the library's own kernel).
Objects are cached by content hash under ``coqui_b200/_build`` so rebuilds are incremental.

    python -m coqui_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libcoqui_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr"]
LIBS: list = []


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_digest():
    h = hashlib.sha256()
    for d in (CSRC, os.path.join(HERE, "..", "include")):
        for f in sorted(os.listdir(d)):
            if f.endswith((".cuh", ".h")):
                with open(os.path.join(d, f), "rb") as fh:
                    h.update(f.encode() + fh.read())
    return h.hexdigest()


def _compile(src, hdr_digest, force):
    path = os.path.join(CSRC, src)
    with open(path, "rb") as fh:
        digest = hashlib.sha256(fh.read() + hdr_digest.encode() + " ".join(ARCH + FLAGS).encode()).hexdigest()[:16]
    obj = os.path.join(BUILD, f"{src[:-3]}.{digest}.o")
    if os.path.exists(obj) and not force:
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, "-I", os.path.join(HERE, "..", "include"), "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hd = _headers_digest()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, hd, force), srcs))
    key = hashlib.sha256("".join(objs).encode()).hexdigest()[:16]
    stamp = os.path.join(BUILD, "lib.stamp")
    if os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read() == key and not force:
        return LIB
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, *LIBS]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    with open(stamp, "w") as fh:
        fh.write(key)
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
