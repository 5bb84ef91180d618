"""Build recipe of libkami_b200.so: every kami_b200/csrc/*.cu compiled by nvcc
for sm_100a (in parallel, incrementally) and linked into one shared library
in the package directory, so the library travels with the source tree.

Usage:  python -m kami_b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libkami_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INCLUDE,
                     "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.inc")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _compile(src: str, force: bool, hdr_mtime: float) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj):
        m = os.path.getmtime(obj)
        if m >= os.path.getmtime(src) and m >= hdr_mtime:
            return obj
    cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if "spill" in r.stderr and "0 bytes spill" not in r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hdr_mtime), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + ".tmp"
        cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
        if verbose:
            print(f"linked {LIB}")
    return LIB


OPS_SRC = os.path.join(HERE, "torch_ops", "kami_torch_ops.cpp")
OPS_LIB = os.path.join(HERE, "libkami_torch_ops.so")


def build_torch_ops(force: bool = False, verbose: bool = False) -> str:
    """torch.ops.kami (the differentiable batched GEMM as a C++ torch operator,
    kami_b200/torch_ops/) linked against libkami_b200.so and libtorch."""
    import torch
    tdir = os.path.dirname(torch.__file__)
    srcs = [OPS_SRC, os.path.join(INCLUDE, "kami.h")]
    if not force and os.path.exists(OPS_LIB) and os.path.getmtime(OPS_LIB) >= max(os.path.getmtime(x) for x in srcs) \
            and os.path.getmtime(OPS_LIB) >= os.path.getmtime(LIB):
        return OPS_LIB
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    tmp = OPS_LIB + ".tmp"
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           "-I", os.path.join(tdir, "include"), "-I", os.path.join(tdir, "include", "torch", "csrc", "api", "include"),
           "-I", os.path.join(cuda_home, "include"), "-I", INCLUDE, OPS_SRC, "-o", tmp,
           "-L", os.path.join(tdir, "lib"), "-ltorch", "-ltorch_cpu", "-lc10", "-lc10_cuda",
           "-L", HERE, "-l:libkami_b200.so", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.join(tdir, "lib")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"torch operator build failed:\n{r.stderr[-3000:]}")
    os.replace(tmp, OPS_LIB)
    if verbose:
        print(f"linked {OPS_LIB}")
    return OPS_LIB


CMP_DIR = os.path.join(HERE, "cmp")
CMP_LIB = os.path.join(HERE, "libkami_cmp.so")


def cutlass_include():
    """The CUTLASS / CuTe header tree shipped in this image (flashinfer's copy),
    or $KAMI_CUTLASS_ROOT; None when absent."""
    roots = [os.environ.get("KAMI_CUTLASS_ROOT")]
    try:
        import importlib.util
        spec = importlib.util.find_spec("flashinfer")
        if spec and spec.origin:
            roots.append(os.path.join(os.path.dirname(spec.origin), "data", "cutlass"))
    except Exception:
        pass
    for r in roots:
        if r and os.path.exists(os.path.join(r, "include", "cute", "arch", "mma_sm100_umma.hpp")):
            return r
    return None


def build_comparators(force: bool = False, verbose: bool = False):
    """Comparator library (not the product): CUTLASS's own sm_100a batched GEMM
    (kami_b200/cmp/*.cu) for the benchmark's side-by-side lines.  Skipped,
    returning None, when the CUTLASS headers are absent or it fails to build."""
    srcs = sorted(glob.glob(os.path.join(CMP_DIR, "*.cu")))
    root = cutlass_include()
    if not srcs or root is None:
        return None
    newest = max(os.path.getmtime(x) for x in srcs)
    if not force and os.path.exists(CMP_LIB) and os.path.getmtime(CMP_LIB) >= newest:
        return CMP_LIB
    tmp = CMP_LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-DNDEBUG",
                             "-diag-suppress", "20012", "-I", os.path.join(root, "include"),
                             "-I", os.path.join(root, "tools", "util", "include"), "-shared", "-o", tmp] + srcs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(f"comparator build skipped:\n{r.stderr[-2000:]}\n")
        return None
    os.replace(tmp, CMP_LIB)
    if verbose:
        print(f"linked {CMP_LIB}")
    return CMP_LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--comparators", action="store_true", help="also build the CUTLASS comparator library")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j, verbose=True))
    print(build_torch_ops(force=a.force, verbose=True))
    if a.comparators:
        print(build_comparators(force=a.force, verbose=True))
