"""Build libimpes_b200.so for sm_100a with nvcc (in-tree).

Usage: python oil-simulator-py_b200/csrc/build.py [--force]

physics.cu is compiled with -fmad=false so the assembly and saturation
arithmetic rounds operation by operation like the reference's CPU evaluation;
the solver translation units keep fused multiply-add.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "impes_b200")
REPO = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(PKG, "libimpes_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", "-I" + os.path.join(REPO, "include")]
SOURCES = {
    "common.cu": [],
    "physics.cu": ["-fmad=false"],
    "amg_setup.cu": [],
    "amg_cycle.cu": [],
    "adjoint.cu": [],
    "ensemble.cu": [],
    "pcg.cu": [],
    "abi.cu": [],
}
HEADERS = ["common.cuh", "model.cuh", "amg.cuh", os.path.join(REPO, "include", "impes_b200.h")]


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def _compile(src, extra):
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    deps = [os.path.join(HERE, src)] + [h if os.path.isabs(h) else os.path.join(HERE, h) for h in HEADERS]
    if _mtime(obj) >= max(_mtime(d) for d in deps):
        return obj, None
    cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", os.path.join(HERE, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    if "warning" in r.stderr:
        sys.stderr.write(f"{src}: compiler warnings\n{r.stderr}")
    return obj, None


def build(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda kv: _compile(kv[0], kv[1]), SOURCES.items()))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if _mtime(OUT) < max(_mtime(o) for o in objs) or force:
        cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
