"""Builds libpfsf.so (C ABI + CUDA sm_100a kernels) in-tree.

    python pfsf-core_b200/build.py [--force]

CUDA sources are compiled by nvcc for sm_100a only, host C++ by g++; the
shared library is linked by nvcc with the static CUDA runtime so it loads
without a CUDA toolkit on the library path.  Output: pfsf-core_b200/lib/libpfsf.so
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(HERE, "lib", "libpfsf.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.path.dirname(os.path.dirname(os.path.realpath(NVCC)))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "-I" + INCLUDE, "-I" + CSRC, "-DPFSF_EXPORT"]
# host primitives keep the reference's rounding: no FMA contraction
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-ffp-contract=off", "-Wall", "-I" + INCLUDE, "-I" + CSRC,
             "-I" + os.path.join(CUDA_HOME, "include"), "-DPFSF_EXPORT"]
# per-file extra flags: the reference-schedule kernels round every product
# and sum as written (no FMA contraction) so they track the FP32 restatement.
EXTRA = {"compat_kernels.cu": ["-fmad=false"]}


def sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith(".cu") or f.endswith(".cpp"):
            out.append(f)
    return out


_INCLUDE_RE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def dep_mtime(path, seen=None):
    """Newest mtime of a source and of every project header it includes
    (directly or through other project headers)."""
    seen = set() if seen is None else seen
    if path in seen:
        return 0.0
    seen.add(path)
    m = os.path.getmtime(path)
    with open(path, errors="replace") as f:
        text = f.read()
    for inc in _INCLUDE_RE.findall(text):
        for d in (os.path.dirname(path), CSRC, INCLUDE):
            cand = os.path.join(d, inc)
            if os.path.exists(cand):
                m = max(m, dep_mtime(cand, seen))
                break
    return m


def compile_one(src, force):
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJ, src + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) > dep_mtime(path):
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + ARCH + NVCC_FLAGS + EXTRA.get(src, []) + ["-c", path, "-o", obj]
    else:
        cmd = ["g++"] + CXX_FLAGS + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return obj, None


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: compile_one(s, force), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("libpfsf build failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("libpfsf link failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    try:
        build(a.force, verbose=True)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
