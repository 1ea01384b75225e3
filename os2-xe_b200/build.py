"""Builds liboz2.so (the product: CUDA kernels for sm_100a + the C ABI) in-tree.

    python os2-xe_b200/build.py [--jobs N] [--verbose-ptxas]

Objects go to os2-xe_b200/_build/, the library to os2-xe_b200/oz2/liboz2.so, next to the
Python binding that loads it. nvcc cross-compiles, so no GPU is needed to build.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "oz2", "liboz2.so")
SOURCES = ["oz2_plan.cpp", "oz2_split.cu", "oz2_gemm.cu", "oz2_crt.cu", "oz2_api.cu", "oz2_noalloc.cu", "oz2_adaptive.cu",
           "oz2_mlp.cu", "oz2_certify.cu"]
NVCC = os.environ.get("OZ2_NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX,
         "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(HERE, "csrc")]


def _compile(src, verbose_ptxas):
    path = os.path.join(HERE, "csrc", src)
    obj = os.path.join(BUILD, src + ".o")
    deps = [path] + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))
                     if f.endswith((".cuh", ".hpp"))] + [os.path.join(ROOT, "include", "oz2", "oz2.h")]
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj, ""
    cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else []) + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(jobs=8, verbose_ptxas=False, quiet=True):
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES))
    objs = [o for o, _ in results]
    if verbose_ptxas:
        for _, log in results:
            sys.stderr.write(log)
    if not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", HOST_CXX, "-Xlinker", "--no-undefined", "-o", OUT] + objs + ["-lcuda", "-lcublas"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if not quiet:
        print(OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    build(a.jobs, a.verbose_ptxas, quiet=False)
