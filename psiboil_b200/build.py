"""Build recipe of the engine library: nvcc for sm_100a, in-tree output.

Produces psiboil_b200/libpsiboil_b200.so from psiboil_b200/csrc/*.cu.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libpsiboil_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--extended-lambda",
              "-gencode", "arch=compute_100a,code=sm_100a",
              "-Xcompiler", "-fPIC", "-Xptxas", "-O3"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps():
    return sources() + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(os.path.dirname(HERE), "include", "psiboil_b200.h")]


def build(force=False, verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    newest = max(os.path.getmtime(p) for p in deps())
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest:
        return OUT
    from concurrent.futures import ThreadPoolExecutor
    objs = []
    cmds = []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        cmds.append(["nvcc"] + NVCC_FLAGS + ["-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
        return r

    with ThreadPoolExecutor(jobs or os.cpu_count() or 4) as ex:
        list(ex.map(run, cmds))
    link = ["nvcc", "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT] + objs + \
        ["-lcudart"]
    subprocess.check_call(link)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
