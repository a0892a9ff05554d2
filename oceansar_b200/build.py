"""Build the sm_100a shared library ``oceansar_b200/_lib/liboceansar_b200.so``.

``python -m oceansar_b200.build`` (or ``__graft_entry__.build()``) compiles every ``.cu``
file under ``oceansar_b200/csrc`` with nvcc for ``sm_100a`` only and links them into one
shared library exporting the C ABI declared in ``include/oceansar_b200.h``.  Objects are
rebuilt when a source or header is newer than the library.  nvcc cross-compiles, so no GPU
is needed to build.
"""
import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "_lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "liboceansar_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xptxas", "-O3", "-I", INCLUDE, "-I", CSRC]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build oceansar_b200")


def _newest_dep():
    deps = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(d) for d in deps), default=0.0)


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    dep_t = _newest_dep()
    objs = []
    cmds = []
    for src in srcs:
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= dep_t):
            continue
        cmds.append([nvcc()] + ARCH + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) +
                    ["-c", src, "-o", obj])
    # one nvcc per translation unit, run side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd))
        for f in [ex.submit(subprocess.check_call, cmd) for cmd in cmds]:
            f.result()
    rebuilt = bool(cmds)
    if rebuilt or force or not os.path.exists(LIB) or \
            any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
