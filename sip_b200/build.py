"""Build libasdsip_fft.so in-tree with nvcc for sm_100a.

    python -m sip_b200.build          # incremental
    python -m sip_b200.build --clean  # rebuild everything

Objects go to sip_b200/_build/, the shared library to sip_b200/libasdsip_fft.so
(both git-ignored).  Every .cu is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; host .cpp files go
through nvcc as well so one toolchain builds the library.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import re
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libasdsip_fft.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
CU_FLAGS = ARCH + ["-lineinfo", "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(src: str, seen: set[str] | None = None) -> set[str]:
    """The file and every project header it includes, transitively."""
    seen = set() if seen is None else seen
    if src in seen or not os.path.exists(src):
        return seen
    seen.add(src)
    with open(src, encoding="utf-8", errors="replace") as f:
        text = f.read()
    for inc in _INCLUDE.findall(text):
        for base in (os.path.dirname(src), CSRC, os.path.join(ROOT, "include")):
            path = os.path.normpath(os.path.join(base, inc))
            if os.path.exists(path):
                _deps(path, seen)
                break
    return seen


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(t < os.path.getmtime(d) for d in _deps(src))


def _compile(src: str, obj: str, verbose: bool) -> tuple[str, str]:
    cmd = [NVCC] + COMMON
    if src.endswith(".cu"):
        cmd += CU_FLAGS
    else:
        cmd += ARCH + ["-x", "c++"]
    cmd += ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    return src, r.stderr


def build(clean: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    """Compile every source under csrc/ and link libasdsip_fft.so; returns its path."""
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    objs, todo = [], []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, src):
            todo.append((src, obj))
    # device-heavy translation units first, so that the longest compiles start at once
    todo.sort(key=lambda so: (not so[0].endswith(".cu"), -os.path.getsize(so[0]) if "row_inst_32" not in so[0] else -1e9))
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
            for src, warn in ex.map(lambda so: _compile(so[0], so[1], verbose), todo):
                if warn.strip() and verbose:
                    print(f"{os.path.basename(src)}:\n{warn}", file=sys.stderr)
    if todo or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args()
    print(build(clean=args.clean, verbose=args.verbose))


if __name__ == "__main__":
    main()
