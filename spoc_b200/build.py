"""Builds the in-tree CUDA library spoc_b200/libspoc_gpu.so for sm_100a.

The library holds the C ABI declared in include/spoc_gpu.h: host set-up code
(g++, -ffp-contract=off) and the device kernels (nvcc, sm_100a).  It is built
in place so that it travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
ROOT = HERE.parent
LIB = HERE / "libspoc_gpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--fmad=false",  # no contraction: the FP64 path reproduces the reference rounding
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas", "-v",
]
SOURCES = ["spoc_kernels.cu", "spoc_fast.cu", "spoc_api.cu", "spoc_noalloc.cu", "spoc_adjoint.cu",
           "spoc_mixed.cu", "spoc_mixed_tc.cu", "spoc_tc_selftest.cu", "spoc_regrid.cu"]
# spoc_fast.cu is compiled a second time with fused multiply-adds
VARIANT_SOURCES = [("spoc_fast.cu", "spoc_fast_fma", ["-DSPOC_FMA=1"])]
HOST_SOURCES = ["spoc_host.cpp"]
HEADERS = ["spoc_device.cuh", "spoc_kernels.h", "spoc_launch.h", "spoc_bulk.cuh", "spoc_mixed.h", "spoc_tc.cuh",
           "spoc_mixed_dev.cuh"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HOST_SOURCES + HEADERS] + [ROOT / "include" / "spoc_gpu.h", Path(__file__)]
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if any source is newer than it; return its path."""
    if not force and not _stale():
        return LIB
    nvcc = _nvcc()
    bdir = HERE / "_build"
    bdir.mkdir(exist_ok=True)
    jobs = []
    for src in SOURCES:
        jobs.append((src, bdir / (src + ".o"),
                     [nvcc, *ARCH, *NVCC_FLAGS, "-c", str(CSRC / src), "-o", str(bdir / (src + ".o"))]))
    for src, stem, defs in VARIANT_SOURCES:
        jobs.append((src, bdir / (stem + ".o"),
                     [nvcc, *ARCH, *NVCC_FLAGS, *defs, "-c", str(CSRC / src), "-o", str(bdir / (stem + ".o"))]))
    for src in HOST_SOURCES:
        jobs.append((src, bdir / (src + ".o"),
                     ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                      "-Wall", "-c", str(CSRC / src), "-o", str(bdir / (src + ".o"))]))
    # the translation units are independent: compile them concurrently
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda j: subprocess.run(j[2], capture_output=True, text=True), jobs))
    log = []
    for (src, _, cmd), r in zip(jobs, results):
        log.append(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed on {src} ({' '.join(cmd[-6:])}):\n{r.stderr}")
    objs = [j[1] for j in jobs]
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    (bdir / "ptxas.log").write_text("\n".join(log))
    if verbose:
        print("\n".join(log))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
