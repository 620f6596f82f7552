"""Build the in-tree CUDA library radix_b200/lib/libradix_b200.so for sm_100a,
and its bounds-checked twin libradix_b200_check.so (RDX_CHECK defined: every
index a kernel clamps is also recorded in the device error word, which the
calls then report; a stand-in for a memory checker, loaded when
RADIX_B200_CHECK=1).

Each source compiles to an object in parallel, then nvcc links the shared
library. Host code is compiled with -ffp-contract=off: the float64 camera and
object set-up must round as the CPU oracle does.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libradix_b200.so")
CHECK_LIB = os.path.join(LIB_DIR, "libradix_b200_check.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "--expt-relaxed-constexpr"]
SOURCES = ["sort.cu", "keys.cu", "project.cu", "rays.cu", "backward.cu", "ply.cu", "spz.cu", "rdxfile.cu", "noalloc.cu",
           "abi.cpp"]
# Per-file flags: the ray methods round every float64 step as the CPU oracle does
EXTRA = {"rays.cu": ["--fmad=false"]}


def _compile(src, verbose, check=False):
    obj = os.path.join(BUILD, "check" if check else "", src + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(HERE, "..", "include", "radix_b200.h"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj, ""
    cmd = [NVCC, *ARCH, *FLAGS, *EXTRA.get(src, []), *(["-DRDX_CHECK"] if check else []), "-c", path, "-o", obj]
    if verbose and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False, check=False):
    """Build the library (check: its bounds-checked twin); returns its path."""
    lib = CHECK_LIB if check else LIB
    os.makedirs(os.path.join(BUILD, "check") if check else BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        results = list(pool.map(lambda s: _compile(s, verbose, check), SOURCES))
    objs = [o for o, _ in results]
    if verbose:
        for (_, log), src in zip(results, SOURCES):
            if log:
                print(f"== {src}\n{log}")
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(lib) or os.path.getmtime(lib) < newest:
        # zlib inflates gzip SPZ files; libzstd (SPZ 4) is opened at run time with dlopen
        cmd = [NVCC, *ARCH, "-shared", "-o", lib, *objs, "-lcudart_static", "-lz", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, check="--check" in sys.argv))
