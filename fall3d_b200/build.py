"""Builds libfall3d_ads.so in-tree for sm_100a with nvcc.

The FP64 sweep and auxiliary kernels are compiled with --fmad=false so that
they keep the reference's separately rounded products and sums; the FP32
precision form and the host code use the default contraction.
Run: python -m fall3d_b200.build  (or call build()).
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfall3d_ads.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

SOURCES = [
    # (file, extra flags)
    ("ads_fp64.cu", ["--fmad=false"]),
    ("aux_fp64.cu", ["--fmad=false"]),
    ("ads_fp32.cu", []),
    ("ens.cu", []),
    ("mlp.cu", ["--fmad=false"]),
    ("noalloc.cu", ["--fmad=false"]),
    ("meteo_dev.cu", ["--fmad=false"]),
    ("deposit_dev.cu", ["--fmad=false"]),
    ("output_dev.cu", ["--fmad=false"]),
    ("f3d_capi.cu", ["-Xcompiler", "-ffp-contract=off"]),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _needs_rebuild(objs: list[str]) -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "fall3d_ads.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every CUDA source for sm_100a and link the shared library."""
    present = [(f, fl) for f, fl in SOURCES if os.path.exists(os.path.join(CSRC, f))]
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, f.replace(".cu", ".o")) for f, _ in present]
    if not force and not _needs_rebuild(objs):
        return LIB
    nv = nvcc()
    common = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-I" + os.path.join(HERE, "..", "include")]
    cmds = [[nv, "-c", os.path.join(CSRC, f), "-o", o] + common + fl for (f, fl), o in zip(present, objs)]
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd), flush=True)
    # the translation units are independent: compile them side by side
    # (the two sweep files take minutes each)
    workers = max(1, min(len(cmds), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as pool:
        for r in pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args, r.stdout, r.stderr)
    tmp = LIB + ".tmp"
    cmd = [nv, "-shared", "-o", tmp] + objs + ARCH + ["-cudart=static"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
