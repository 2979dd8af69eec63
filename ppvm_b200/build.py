"""Build recipe of the CUDA library (sm_100a), used by __graft_entry__.build().

The library is built in-tree as ppvm_b200/libppvm_cuda.so with nvcc directly from
csrc/engine.cu (the kernels and the C ABI of include/ppvm_cuda.h) and csrc/noalloc.cu.  -fmad=false keeps every coefficient product and sum a separately
rounded IEEE operation, as the reference's f64 arithmetic is.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libppvm_cuda.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("engine.cu", "batch.cu", "learned.cu", "noalloc.cu")]
HEADERS = sorted(
    os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc")) if f.endswith(".cuh")
) + [os.path.join(ROOT, "include", "ppvm_cuda.h")]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
    "-Xcompiler", "-ffp-contract=off",
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    """Compiles every source to an object (in parallel), then links the shared library."""
    if not force and not stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    procs = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [nvcc(), *compile_flags, *extra, "-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    errors = []
    for cmd, p in procs:
        out, err = p.communicate()
        if p.returncode != 0:
            errors.append(f"{' '.join(cmd)}\n{out}\n{err}")
        elif verbose and err:
            print(err, file=sys.stderr)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
            "-o", LIB, *objs]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
