"""Build recipe of libphx.so (hand-written CUDA for sm_100a + C ABI).

Compiles every ``csrc/*.cu`` with nvcc for ``sm_100a`` only and links them
into ``phoebe_b200/libphx.so`` in-tree, so the library travels with the
source tree.  Object files go to ``phoebe_b200/_build/``.
"""
import concurrent.futures
import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libphx.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++"]


def _needs(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    objs = []
    jobs = []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if _needs(obj, [src] + headers):
            cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_verbose else []) + \
                ["-c", src, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
        return r.stdout + r.stderr

    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for out in ex.map(run, jobs):
            if verbose or ptxas_verbose:
                print(out)
    if _needs(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda", "-lcusolver", "-ldl", "-ccbin", "/usr/bin/g++"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    import sys
    build(verbose=True, ptxas_verbose="-v" in sys.argv)
