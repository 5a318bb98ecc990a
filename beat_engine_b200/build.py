"""Build libbeatb200.so in-tree with nvcc for sm_100a.

    python -m beat_engine_b200.build        # or: python beat_engine_b200/build.py

The library is plain CUDA C++ behind the C ABI of include/beat_b200.h; it
links only the CUDA runtime.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbeatb200.so")
SOURCES = ["context.cu", "assembly.cu", "lu.cu", "tc_gemm.cu", "gmres.cu", "field.cu", "adjoint.cu", "coupled.cu", "shape.cu", "abi.cu",
           "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# per-file flags: the FP32 element-pair quadrature flushes denormals (its values
# are nowhere near the FP32 denormal range; the FP64 paths are unaffected)
FILE_FLAGS = {"assembly.cu": ["-ftz=true"]}


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA 12.9 toolkit is required to build libbeatb200")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(CSRC, "internal.cuh"), os.path.join(CSRC, "phase.cuh"),
                                                        os.path.join(HERE, "..", "include", "beat_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    nvcc = nvcc_path()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++"]
    if verbose:
        flags += ["-Xptxas", "-v"]
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc, *flags, *FILE_FLAGS.get(src, []), "-c", os.path.join(CSRC, src), "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for cmd, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append(" ".join(cmd) + "\n" + text)
        elif verbose and text:
            print(text)
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(failed))
    tmp = LIB + ".tmp"
    subprocess.run([nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
