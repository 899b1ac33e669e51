"""Builds the FastFss drop-in library for B200 (sm_100a) in-tree.

    python -m fastfunctionsecretsharing_b200.build [--verbose-ptxas] [-j N]

Every ``csrc/*.cu`` / ``csrc/*.cpp`` is compiled by nvcc into ``_build/`` and linked into
``lib/libFastFss.so`` (CUDA runtime linked statically, so the library does not depend on
which libcudart the host process loaded). The exported symbols are the ``FastFss_*`` C ABI
declared under ``include/FastFss``.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libFastFss.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "--default-stream", "per-thread", "-Xcompiler", "-fPIC,-fvisibility=hidden",
          "-DFAST_FSS_BUILD", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    hs += glob.glob(os.path.join(INCLUDE, "FastFss", "**", "*.h"), recursive=True)
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, verbose_ptxas: bool) -> tuple[str, str]:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    cmd = [nvcc(), *ARCH, *COMMON, "-lineinfo", "-c", src, "-o", obj]
    if verbose_ptxas and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose_ptxas: bool = False, jobs: int = 0, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sources()
    hdr = _headers_mtime()
    todo = []
    for s in srcs:
        obj = os.path.join(BUILD, os.path.basename(s) + ".o")
        if force or verbose_ptxas or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(s), hdr):
            todo.append(s)
    logs = []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
            for obj, log in ex.map(lambda s: _compile(s, verbose_ptxas), todo):
                logs.append(log)
    objs = [os.path.join(BUILD, os.path.basename(s) + ".o") for s in srcs]
    if todo or not os.path.exists(LIB):
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    if verbose_ptxas:
        sys.stderr.write("".join(logs))
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=0)
    a = ap.parse_args()
    print(build(verbose_ptxas=a.verbose_ptxas, jobs=a.j, force=a.force))


if __name__ == "__main__":
    main()
