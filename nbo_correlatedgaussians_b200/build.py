"""Build libnecg_b200.so in-tree with nvcc for sm_100a.

The library is plain CUDA C++ behind the C ABI of include/necg.h, compiled one
object per source file (in parallel, under _build/) and linked with the
CUDA runtime statically so that it does not depend on which libcudart the
Python process has already loaded.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libnecg_b200.so")
SOURCES = ["necg_kernels.cu", "necg_capi.cu", "necg_count.cu", "necg_batch.cu", "necg_noalloc.cu"]
HEADERS = ["necg_math.cuh", "necg_kernels.cuh", "necg_lanes.cuh", "necg_handle.h", "necg_hostscalar.cuh",
           "necg_device.cuh", "necg_trace.h"]
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMPILE_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v"]
LINK_FLAGS = ["-Xcompiler", "-fPIC", "--shared", "-cudart", "static"]
OBJDIR = os.path.join(os.path.dirname(HERE), "_build")


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libnecg_b200.so")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "necg.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(nvcc: str, src: str, obj: str) -> str:
    cmd = [nvcc, *ARCH, *COMPILE_FLAGS, "-I", INCLUDE, "-c", os.path.join(CSRC, src), "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n" + res.stdout + res.stderr)
    return res.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if it is missing or older than its sources: one nvcc
    per source file in parallel, then one link."""
    if not force and not _stale():
        return LIB
    nvcc = _nvcc()
    os.makedirs(OBJDIR, exist_ok=True)
    objs = [os.path.join(OBJDIR, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        reports = list(ex.map(lambda so: _compile(nvcc, *so), zip(SOURCES, objs)))
    cmd = [nvcc, *ARCH, *LINK_FLAGS, *objs, "-o", LIB + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    report = "".join(reports)
    with open(os.path.join(HERE, "ptxas_report.txt"), "w") as fh:
        fh.write(report)
    if verbose:
        print(report, file=sys.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
