"""Build the reference's own CUDA kernels for sm_100a as benchmark comparators (oracle/_ref/, git-ignored).

    python oracle/build_ref.py [--reference PATH]     (default: $MATVANS_REFERENCE, else /root/reference)

Each library is oracle/ref_shims.cu compiled with one unmodified reference source file included (the path is
passed on the command line; nothing is copied into this repository) and the reference program's main()
renamed, so that the kernel links as a shared library with an extern "C" launcher:

    libref_awr.so        buffered/ans-warp-rows-kernel.cu
    libref_dense.so      baselines/baseline_int8/baseline_matVec_custom.cu
    libref_wpr.so        matvansWarpPerRow/matvansWarpPerRow.cu (includes matvansWarpPerRow-kernel.cu)
    libref_wpr_local.so  matvansWarpPerRow/matvansWarpPerRow_local_cdf.cu

Outputs go to oracle/_ref/ only.  When the reference checkout is absent nothing is built and the benchmark
reports these comparators as unavailable.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "ref_shims.cu")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# (library, define, reference source relative to the checkout, extra link flags)
TARGETS = [
    ("libref_awr.so", "REF_AWR", "buffered/ans-warp-rows-kernel.cu", []),
    ("libref_dense.so", "REF_DENSE", "baselines/baseline_int8/baseline_matVec_custom.cu", ["-lcublas", "-lcublasLt"]),
    ("libref_wpr.so", "REF_WPR", "matvansWarpPerRow/matvansWarpPerRow.cu", []),
    ("libref_wpr_local.so", "REF_WPR_LOCAL", "matvansWarpPerRow/matvansWarpPerRow_local_cdf.cu", []),
]


def nvcc():
    return os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def build_one(ref, lib, define, rel, link):
    src = os.path.join(ref, rel)
    out = os.path.join(OUT, lib)
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(src), os.path.getmtime(SHIM)):
        return out, ""
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-w",
           f"-D{define}", f'-DREF_SOURCE="{src}"', "-Dmain=matvans_reference_program_main",
           "-I", os.path.dirname(src), SHIM, "-o", out + ".tmp", *link]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return None, f"{lib}: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    os.replace(out + ".tmp", out)
    return out, ""


def build(reference=None, quiet=False):
    ref = reference or os.environ.get("MATVANS_REFERENCE") or "/root/reference"
    if not os.path.isfile(os.path.join(ref, "buffered", "ans-warp-rows-kernel.cu")):
        if not quiet:
            print(f"build_ref: no reference checkout at {ref}; nothing built", file=sys.stderr)
        return []
    os.makedirs(OUT, exist_ok=True)
    with cf.ThreadPoolExecutor(len(TARGETS)) as ex:
        res = list(ex.map(lambda t: build_one(ref, *t), TARGETS))
    errs = [e for _, e in res if e]
    if errs:
        raise RuntimeError("build_ref failed:\n" + "\n".join(errs))
    return [o for o, _ in res]


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    a = ap.parse_args()
    for p in build(a.reference):
        print(p)
