"""Builds the engine's native library in-tree.

``libads_gpu.so`` (the C ABI of ``include/ads_gpu.h``) is compiled from
``csrc/*.cu`` with nvcc for sm_100a only and written to ``_lib/``.  Host code is
compiled with -ffp-contract=off so the m/z grid and the Gaussian kernel keep the
reference's f32 rounding.

Usage: ``python -m alphadia_search_rs_b200.build [--force] [-v]``
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "_lib")
OBJDIR = os.path.join(PKG, "_build")
LIBNAME = "libads_gpu.so"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    # no implicit multiply-add contraction anywhere in device code (the parity
    # arithmetic uses explicitly rounded ops; this keeps everything else alike)
    "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
    "-Xptxas", "-warn-spills",
    "-diag-suppress", "1444",  # deprecated cub iterators
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the engine needs the CUDA toolkit to build")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _digest(paths: list[str], extra: list[str]) -> str:
    h = hashlib.sha256()
    for p in paths:
        with open(p, "rb") as f:
            h.update(p.encode() + b"\0" + f.read())
    h.update("\0".join(extra).encode())
    return h.hexdigest()


def lib_path() -> str:
    return os.path.join(LIBDIR, LIBNAME)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    """Compile (if sources changed) and return the path of libads_gpu.so."""
    srcs = sources()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "ads_gpu.h"))
    flags = ARCH_FLAGS + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_verbose else [])
    digest = _digest(srcs + sorted(headers), flags)
    stamp = os.path.join(LIBDIR, ".stamp")
    out = lib_path()
    if not force and os.path.exists(out) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == digest:
                return out
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    nv = nvcc()

    def compile_one(src: str) -> str:
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        cmd = [nv, *flags, "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or ptxas_verbose or r.returncode:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError(f"nvcc failed on {os.path.basename(src)}")
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = out + ".tmp"
    cmd = [nv, *ARCH_FLAGS, "-shared", "-o", tmp, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode:
        raise RuntimeError("linking libads_gpu.so failed")
    os.replace(tmp, out)
    with open(stamp, "w") as f:
        f.write(digest)
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print ptxas register/spill report")
    a = ap.parse_args()
    print(build(force=a.force or a.ptxas, verbose=a.verbose, ptxas_verbose=a.ptxas))


if __name__ == "__main__":
    main()
