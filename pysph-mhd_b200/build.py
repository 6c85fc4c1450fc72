"""Build ``libmhd_b200.so`` (sm_100a) in-tree with nvcc.

    python pysph-mhd_b200/build.py [--force]

The shared library exports the C ABI declared in ``include/mhd_b200.h`` and
is loaded by ``src/_abi.py`` through ctypes.
"""

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmhd_b200.so")
OBJ = os.path.join(HERE, "_build")
SOURCES = ["mhd_abi.cu", "mhd_cells.cu", "mhd_pairs.cu", "mhd_force.cu", "mhd_integrate.cu", "mhd_noalloc.cu",
           "mhd_pairgrid.cu", "mhd_tangent.cu", "mhd_adjoint.cu"]
# The derivative forms follow the reference's expression order: no FMA contraction.
FILE_FLAGS = {"mhd_tangent.cu": ["--fmad=false"], "mhd_adjoint.cu": ["--fmad=false"]}
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
         "--extended-lambda", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "mhd_b200.h")]


def build(force=False, verbose=False):
    if not force and os.path.exists(OUT):
        newest = max(os.path.getmtime(p) for p in _deps())
        if os.path.getmtime(OUT) >= newest:
            return OUT
    os.makedirs(OBJ, exist_ok=True)
    headers = [p for p in _deps() if not p.endswith(".cu")]
    newest_header = max(os.path.getmtime(p) for p in headers)

    def compile_one(src):
        obj = os.path.join(OBJ, src.replace(".cu", ".o"))
        if not force and not verbose and os.path.exists(obj):
            # an object is current when newer than its source and every header
            if os.path.getmtime(obj) >= max(newest_header, os.path.getmtime(os.path.join(CSRC, src))):
                return obj, ""
        cmd = [NVCC, *FLAGS, *FILE_FLAGS.get(src, []), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
        return obj, r.stderr

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    if verbose:
        for _, err in results:
            sys.stderr.write(err)
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT, *[o for o, _ in results],
           "-lcudart"]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
