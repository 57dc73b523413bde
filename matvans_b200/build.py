"""Build libmatvans.so in-tree for sm_100a (B200).

    python -m matvans_b200.build [--verbose-ptxas]

CUDA sources are compiled by nvcc with ``-gencode arch=compute_100a,code=sm_100a``,
host sources by g++; objects are cached under matvans_b200/_build/ by mtime and
linked into matvans_b200/libmatvans.so (cudart linked statically, so the
library does not depend on the CUDA runtime version torch ships).
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmatvans.so")
INCLUDE = os.path.join(ROOT, "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def sources():
    out = []
    for fn in sorted(os.listdir(CSRC)):
        if fn.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, fn))
    return out


def headers():
    hs = [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs


def compile_one(src, verbose_ptxas=False):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in headers()])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep and not verbose_ptxas:
        return obj, ""
    inc = ["-I", INCLUDE, "-I", CSRC]
    if src.endswith(".cu"):
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
               "--expt-relaxed-constexpr", *inc, "-c", src, "-o", obj]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = ["g++", "-O3", "-fPIC", "-std=c++17", "-Wall", "-Wextra", "-ffp-contract=off",
               "-I", "/usr/local/cuda/include", *inc, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose_ptxas=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(jobs or os.cpu_count()) as ex:
        results = list(ex.map(lambda s: compile_one(s, verbose_ptxas), srcs))
    objs = [o for o, _ in results]
    if verbose_ptxas:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lpthread", "-ldl", "-lrt"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(verbose_ptxas=a.verbose_ptxas))
