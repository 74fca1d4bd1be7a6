"""Build libqm_gpu.so (the C ABI of include/qm_gpu.h) in-tree for sm_100a.

    python -m querymode_b200.build

nvcc compiles the CUDA sources for sm_100a only and links the CUDA runtime
statically, so the library depends on the NVIDIA driver alone.  Only the
`qm_*` entry points are exported.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "libqm_gpu.so")
SOURCES = ["qm_api.cu", "qm_kernels.cu", "qm_batch.cu", "qm_part.cu"] + [f"qm_scan_nv{n}.cu" for n in range(5)]
HEADERS = ["qm_plan.h", "qm_launch.h", "qm_kernels.cuh", "qm_batch.h", "qm_scan.cuh", "qm_scan_spec.cuh",
           "qm_server.cuh", "qm_parquet.cuh", os.path.join("..", "..", "include", "qm_gpu.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [__file__]
    if not force and not _stale(OUT, deps):
        return OUT
    build_dir = os.path.join(PKG, "_build")
    os.makedirs(build_dir, exist_ok=True)
    vers = os.path.join(build_dir, "exports.map")
    with open(vers, "w") as f:
        f.write("{ global: qm_*; local: *; };\n")
    nvcc = _nvcc()
    cmds = []
    for s in SOURCES:
        obj = os.path.join(build_dir, s.replace(".cu", ".o"))
        cmds.append((obj, [nvcc, *NVCC_FLAGS, "-c", os.path.join(CSRC, s), "-o", obj]))
    objs = [o for o, _ in cmds]

    def compile_one(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    # translation units compile in parallel (the scan kernel's specialised
    # instantiations are spread over several of them)
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(compile_one, c) for _, c in cmds]:
            f.result()
    tmp = OUT + ".tmp"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static",
           "-Xlinker", f"--version-script={vers}", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
