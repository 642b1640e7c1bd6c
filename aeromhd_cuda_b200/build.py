"""Build libaeromhd.so in-tree for sm_100a.

    python -m aeromhd_cuda_b200.build [--force] [--verbose]

The float64 translation unit is compiled with -fmad=false so that its
arithmetic rounds exactly as the reference's float64 path does; the float32
one keeps multiply-add contraction.  Objects go to ``_build/`` (git-ignored);
the shared library lands next to this file, where ``_lib.py`` loads it.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libaeromhd.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC,
          "--expt-relaxed-constexpr"]
UNITS = {
    "amhd_f64.cu": ["-fmad=false"],
    "amhd_f32.cu": [],
    "amhd_capi.cu": [],
    "amhd_nn.cu": [],
}


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def source_hash() -> str:
    """Hash of every source, header and this recipe (file copies may not keep mtimes)."""
    h = hashlib.sha256()
    files = [os.path.join(d, f) for d in (CSRC, INCLUDE) for f in sorted(os.listdir(d))] + [__file__]
    for path in files:
        h.update(os.path.basename(path).encode())
        with open(path, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def is_current() -> bool:
    try:
        with open(LIB + ".srchash") as f:
            return os.path.exists(LIB) and f.read().strip() == source_hash()
    except OSError:
        return False


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and is_current():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    objs, cmds = [], []
    for src, extra in UNITS.items():
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        cmd = [nvcc, *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), flush=True)
        cmds.append(cmd)
        objs.append(obj)
    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
        for f in [pool.submit(subprocess.check_call, c) for c in cmds]:
            f.result()
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    with open(LIB + ".srchash", "w") as f:
        f.write(source_hash())
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose, ptxas_info=a.ptxas_info))
    return 0


if __name__ == "__main__":
    sys.exit(main())
