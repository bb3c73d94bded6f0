"""Build the sm_100a shared library ``libcgs_b200.so`` in-tree.

Each ``csrc/*.cu`` is compiled by nvcc for ``sm_100a`` (one object per translation
unit, in parallel) and linked into ``cugridsearch_b200/libcgs_b200.so`` with the CUDA
runtime linked statically, so the library loads with nothing but the driver.

Usage: ``python -m cugridsearch_b200.build [--verbose] [--force]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcgs_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no implicit multiply-add contraction.  Every fused operation in the kernels is an
# explicit fmaf(), so a grid point's arithmetic is the same in every kernel instantiation and
# results do not depend on the tuning choice.
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-fmad=false", "-Xcompiler", "-fPIC,-O2",
           "-I", CSRC, "-I", INCLUDE]
# Translation units built with nvcc's default contraction instead: the image steps around a
# search (warp, overlay, filter, quantisation) follow the reference's device build of them.
DEFAULT_FMAD = {"cgs_image.cu"}


def _flags(src: str) -> list[str]:
    if os.path.basename(src) in DEFAULT_FMAD:
        return [f for f in NVFLAGS if f != "-fmad=false"]
    return NVFLAGS


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


_INCLUDE_RE = re.compile(r'^\s*#\s*include\s*"([^"]+)"', re.M)


def _deps(src: str) -> list[str]:
    """The file and every project header it includes, transitively (quoted includes
    resolved against the including file's folder, csrc/ and include/)."""
    seen: list[str] = []
    todo = [os.path.abspath(src)]
    while todo:
        f = todo.pop()
        if f in seen:
            continue
        seen.append(f)
        with open(f) as fh:
            text = fh.read()
        for name in _INCLUDE_RE.findall(text):
            for base in (os.path.dirname(f), CSRC, INCLUDE):
                cand = os.path.abspath(os.path.join(base, name))
                if os.path.exists(cand):
                    todo.append(cand)
                    break
    return sorted(seen)


def _stamp(src: str, extra: list[str]) -> str:
    h = hashlib.sha256()
    for f in _deps(src):
        with open(f, "rb") as fh:
            h.update(fh.read())
    # flags with the checkout's own folders made relative, so a copy of the tree at another path
    # (built objects travel with it) keeps its stamps
    root = os.path.dirname(HERE)
    flags = [os.path.relpath(f, root) if os.path.isabs(f) and f.startswith(root) else f
             for f in _flags(src) + ARCH + extra]
    h.update(" ".join(flags).encode())
    return h.hexdigest()[:16]


def _compile(src: str, verbose: bool, extra: list[str], force: bool) -> str:
    base = os.path.splitext(os.path.basename(src))[0]
    obj = os.path.join(OBJ, base + ".o")
    stamp_file = obj + ".stamp"
    stamp = _stamp(src, extra)
    if not force and os.path.exists(obj) and os.path.exists(stamp_file):
        with open(stamp_file) as fh:
            if fh.read().strip() == stamp:
                return obj
    cmd = [nvcc(), *_flags(src), *ARCH, *extra, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)
    with open(stamp_file, "w") as fh:
        fh.write(stamp)
    return obj


def build(verbose: bool = False, force: bool = False, extra: list[str] | None = None) -> str:
    extra = extra or []
    os.makedirs(OBJ, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, extra, force), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill reports")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force))
