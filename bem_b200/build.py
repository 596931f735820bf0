"""Build the sm_100a shared library in-tree: bem_b200/libspt_b200.so.

    python -m bem_b200.build

nvcc cross-compiles without a GPU.  The product loads only this library;
nothing is JIT-compiled at run time.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libspt_b200.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in (
    "spt_kernels.cu", "spt_mlp.cu", "spt_image.cu", "spt_trace_flat.cu", "spt_trace_tip.cu", "spt_trace_tipbem.cu",
    "spt_trace_well.cu", "spt_trace_post.cu")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", h) for h in ("spt_device.cuh", "spt_math.cuh", "spt_umma.cuh", "spt_abi.hpp")] + [
    os.path.join(REPO, "include", "spt_b200.h")]
OBJ_DIR = os.path.join(HERE, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "-Xptxas", "-v",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in DEPS)


def build(force=False, verbose=False):
    """Compile every translation unit (in parallel: one per geometry kind of
    the trace kernel, the C ABI, the MLP kernels) and link the library."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJ_DIR, exist_ok=True)
    inc = ["-I", os.path.join(REPO, "include")]

    def compile_one(src):
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        cmd = [nvcc()] + NVCC_FLAGS + inc + ["-c", "-o", obj, src]
        res = subprocess.run(cmd, capture_output=True, text=True)
        return src, obj, cmd, res

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    for src, obj, cmd, res in results:
        if verbose or res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed ({res.returncode}): {' '.join(cmd)}")
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp"] + [
        r[1] for r in results]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({res.returncode}): {' '.join(cmd)}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
