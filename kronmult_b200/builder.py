"""Build libkronmult_b200.so (sm_100a) in-tree.

    python -m kronmult_b200.builder          # or kronmult_b200.build.build()

Every CUDA source under kronmult_b200/csrc is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo`` into
kronmult_b200/lib/obj/ and linked (static CUDA runtime) into
kronmult_b200/lib/libkronmult_b200.so.  Sources are rebuilt only when they
or a header changed.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIBNAME = "libkronmult_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def cflags():
    return ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                   "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
                   "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, obj: str) -> str:
    cmd = [nvcc()] + cflags() + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hm = _headers_mtime()
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(OBJDIR, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hm):
            todo.append((s, o))
    jobs = jobs or min(len(todo) or 1, os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for (s, o), log in zip(todo, ex.map(lambda so: _compile(*so), todo)):
            if verbose and log.strip():
                print(f"[{os.path.basename(s)}] {log.strip()}", file=sys.stderr)
    lib = os.path.join(LIBDIR, LIBNAME)
    if todo or not os.path.exists(lib):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", lib] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
