"""Builds the CUDA path-tracer library in-tree for sm_100a.

    python -m naivetrace_b200.build [--force]

Output: naivetrace_b200/_build/libtoytrace_gpu.so (the C ABI of include/toytrace_gpu.h).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_build"
LIB = OUT_DIR / "libtoytrace_gpu.so"

SOURCES = ["tt_kernels.cu", "tt_capi.cu", "tt_noalloc.cu", "tt_build.cu", "tt_guide.cu", "tt_tree.cu", "tt_bvh.cpp",
           "tt_quadtree.cpp"]
HEADERS = ["tt_internal.h", "tt_device.cuh", "tt_bvh.h", "tt_build.h", "tt_guide.h", "tt_guide.cuh", "tt_tables.h", "tt_pt2.cuh", "tt_sobol_data.h", "tt_tree.h", "tt_guide_tc.cuh", "tt_quadtree.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    OUT_DIR.mkdir(exist_ok=True)
    deps = [CSRC / s for s in SOURCES] + [CSRC / h for h in HEADERS] + [ROOT / "include" / "toytrace_gpu.h", Path(__file__)]
    if not force and not _stale(LIB, deps):
        return LIB
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include")]
    cmds, objs = [], []
    for src in SOURCES:
        obj = OUT_DIR / (Path(src).stem + ".o")
        cmd = [nvcc(), *ARCH, "-lineinfo", *common, "-c", str(CSRC / src), "-o", str(obj)]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        else:
            cmd += ["-x", "c++"]
        cmds.append(cmd)
        objs.append(str(obj))
    # The translation units are independent: compile them side by side.
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(subprocess.run, c, check=True) for c in cmds]:
            f.result()
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill report")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
