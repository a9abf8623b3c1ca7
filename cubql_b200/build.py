"""Build libbq.so (the CUDA library behind include/bq.h) in-tree, for sm_100a.

    python cubql_b200/build.py [--ptxas-verbose]

(run by path: importing the package itself requires the built library)

Each csrc/*.cu is compiled separately (in parallel) and linked into
cubql_b200/libbq.so.  Objects go to cubql_b200/_build/.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbq.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "--expt-relaxed-constexpr", "-diag-suppress=177"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _compile(src, ptxas_verbose):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    # every source of the directory: a .cu may include another (bq_elh.cu includes bq_sah.cu)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".cu"))]
    deps.append(os.path.join(HERE, "..", "include", "bq.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj, ""
    cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
    if ptxas_verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(ptxas_verbose=False, quiet=True):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    logs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = []
        for obj, log in ex.map(lambda s: _compile(s, ptxas_verbose), srcs):
            objs.append(obj)
            if log:
                logs.append(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if not quiet:
        for log in logs:
            sys.stderr.write(log)
    return LIB


if __name__ == "__main__":
    build(ptxas_verbose="--ptxas-verbose" in sys.argv, quiet=False)
    print(LIB)
