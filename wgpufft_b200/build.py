"""Builds libwgpufft_b200.so in-tree: every csrc/*.cu compiled for sm_100a by
nvcc (in parallel), linked with the static CUDA runtime."""
from __future__ import annotations

import concurrent.futures
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwgpufft_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
                 "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu") or f.endswith(".cpp"))


_INCLUDE = re.compile(r'^\s*#\s*include\s*"([^"]+)"', re.M)
_DIRS = (CSRC, os.path.join(HERE, "..", "include"))


def _deps_mtime(path: str, seen=None) -> float:
    """Newest modification time of a source and the local headers it
    includes, recursively."""
    seen = set() if seen is None else seen
    if path in seen:
        return 0.0
    seen.add(path)
    m = os.path.getmtime(path)
    with open(path, encoding="utf-8") as f:
        text = f.read()
    for name in _INCLUDE.findall(text):
        for d in (os.path.dirname(path),) + _DIRS:
            cand = os.path.join(d, name)
            if os.path.exists(cand):
                m = max(m, _deps_mtime(cand, seen))
                break
    return m


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if os.path.exists(obj) and os.path.getmtime(obj) >= _deps_mtime(path):
        return obj
    cmd = [NVCC] + CFLAGS + ["-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-cudart=static", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
