"""In-tree build of the native library for sm_100a (B200).

``build()`` compiles ``csrc/`` with nvcc into ``lib/libxyce_b200.so``. The result is placed
inside the package so it travels with the source tree; nothing is installed elsewhere.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libxyce_b200.so")
SOURCES = ["devload.cu", "tia.cu", "mlp.cu", "rf.cpp", "lu.cu", "sptrsv.cu", "bsim4_setup.cpp", "bsim3_setup.cpp",
           "mos1_setup.cpp"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-fmad=false",
              "-Xcompiler", "-fPIC", "-shared"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _which(prog: str) -> str:
    import shutil

    return prog if os.path.sep in prog else (shutil.which(prog) or "/usr/local/cuda/bin/nvcc")


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    inc = os.path.join(HERE, "..", "include")
    deps += [os.path.join(inc, f) for f in os.listdir(inc)]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


# Sources whose arithmetic is not held to bit parity with a CPU build keep fused multiply-add.
FMAD_ON = {"mlp.cu"}


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source to an object (in a temporary directory) and links the library."""
    import tempfile

    os.makedirs(LIB_DIR, exist_ok=True)
    if not force and not needs_build():
        return LIB
    with tempfile.TemporaryDirectory() as tmp:
        objs = []
        for src in SOURCES:
            obj = os.path.join(tmp, os.path.basename(src) + ".o")
            flags = [f for f in NVCC_FLAGS if f != "-shared"]
            if src in FMAD_ON:
                flags = ["-fmad=true" if f == "-fmad=false" else f for f in flags]
            if src == "rf.cpp":  # the refactorization API is marked deprecated (in favour of cuDSS, not installed)
                flags = flags + ["-Xcompiler", "-Wno-deprecated-declarations"]
            cmd = [_nvcc()] + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            objs.append(obj)
        cuda_lib = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(_which(_nvcc())))), "lib64")
        cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC"] + objs + \
              ["-L" + cuda_lib, "-lcusolver", "-Xlinker", "-rpath=" + cuda_lib, "-o", LIB]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
