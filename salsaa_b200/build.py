"""Compiles libsalsaa_gpu.so in place with nvcc for sm_100a.

Usage: python -m salsaa_b200.build   (or salsaa_b200.build.build())
The library is written next to this file and loaded by salsaa_b200/__init__.py.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsalsaa_gpu.so")
SOURCES = ["ntt.cu", "kernels.cu", "prover.cu", "hexl_compat.cu", "no_alloc.cu", "server.cu", "ck_umma.cu", "dense.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "salsaa_gpu.h")]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force=False, verbose=False, extra=()):
    """Compiles every source (in parallel, one nvcc per file) and links the library."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    objs, cmds = [], []
    for src in SOURCES:
        obj = os.path.join(CSRC, src.replace(".cu", ".o"))
        cmds.append([NVCC, *ARCH, *FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)

    def run(cmd):
        return subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        results = list(ex.map(run, cmds))
    for cmd, r in zip(cmds, results):
        if verbose:
            print(" ".join(cmd))
            sys.stdout.write(r.stdout)
            sys.stdout.write(r.stderr)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise subprocess.CalledProcessError(r.returncode, cmd)
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)
