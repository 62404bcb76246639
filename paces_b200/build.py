"""Build libpaces_b200.so (sm_100a) in-tree with nvcc.

    python -m paces_b200.build [--force]

Each .cu file under paces_b200/csrc is compiled to an object under paces_b200/_build
(in parallel), then linked into paces_b200/libpaces_b200.so with a static CUDA runtime,
so the library works next to PyTorch's own runtime.
"""

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpaces_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-O3"]


def nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libpaces_b200")
    return cand


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers():
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    out.append(os.path.join(os.path.dirname(HERE), "include", "paces_b200.h"))
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, extra):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if _stale(obj, [src] + headers()):
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + extra + ["-c", src, "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr}")
        if res.stderr.strip() and "-Xptxas" in " ".join(extra):
            sys.stderr.write(res.stderr)
    return obj


def build(force=False, verbose_ptxas=False):
    """Compile every kernel source for sm_100a and link the shared library; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    if not force and not _stale(LIB, srcs + headers()):
        return LIB
    if force:
        for f in os.listdir(BUILD):
            if f.endswith(".o"):
                os.remove(os.path.join(BUILD, f))
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), srcs))
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv))
