#!/usr/bin/env python3
"""Build the unmodified PSI-BOIL reference library from its own sources.

This is test infrastructure (the parity checker), never product code.

Recipe (the reference's NOMPI configuration, `first:74-80`, without autotools):
  * every `.cpp` listed in a `*_SOURCES` variable of the per-directory
    `Makefile.am` of each `SUBDIRS` entry of `Src/Makefile.am` is compiled
    with `g++ -O3 -std=c++11` straight from where it lies in the reference
    tree (nothing is copied);
  * `Parallel/mpi_macros.h`, which `first NOMPI` creates as a symlink to
    `sequential.h`, is supplied instead by a one-line forwarding header in
    `oracle/_ref/shim/Parallel/`, reached through `-iquote` directories so
    that the reference's relative includes (`"mpi_macros.h"`,
    `"../Parallel/mpi_macros.h"`, `"../../Parallel/..."`, ...) resolve to it;
  * the objects go to `oracle/_ref/obj/` and are archived into
    `oracle/_ref/libboil.a`; the fixture harness `oracle/ref_harness.cpp` is
    linked against it into `oracle/_ref/ref_harness`.

All outputs stay under `oracle/_ref/` (git-ignored). The built harness
travels to the GPU host with the working tree; the reference sources do not
need to exist there.

Usage: python oracle/build_ref.py [--ref DIR] [-j N]   (DIR defaults to $PBG_REFERENCE)
"""
import argparse
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
CXXFLAGS = ["-O3", "-std=c++11", "-w", "-fPIC"]


def _sources_of(makefile_am):
    """Return the .cpp names listed in *_SOURCES of one Makefile.am."""
    text = open(makefile_am).read().replace("\\\n", " ")
    names = []
    for line in text.splitlines():
        m = re.match(r"\s*\w+_SOURCES\s*=\s*(.*)", line)
        if m:
            names += [t for t in m.group(1).split() if t.endswith(".cpp")]
    return names


def source_list(src_root):
    top = open(os.path.join(src_root, "Makefile.am")).read().replace("\\\n", " ")
    m = re.search(r"SUBDIRS\s*=\s*(.*)", top)
    subdirs = m.group(1).split()
    files = []
    for d in subdirs:
        mk = os.path.join(src_root, d, "Makefile.am")
        for name in _sources_of(mk):
            files.append(os.path.join(src_root, d, name))
    return files


def make_shim(src_root):
    shim = os.path.join(OUT, "shim")
    os.makedirs(os.path.join(shim, "Parallel"), exist_ok=True)
    os.makedirs(os.path.join(shim, "d1", "d2", "d3"), exist_ok=True)
    with open(os.path.join(shim, "Parallel", "mpi_macros.h"), "w") as f:
        f.write('#include "%s"\n' % os.path.join(src_root, "Parallel", "sequential.h"))
    return ["-iquote", os.path.join(shim, "Parallel"),
            "-iquote", os.path.join(shim, "d1"),
            "-iquote", os.path.join(shim, "d1", "d2"),
            "-iquote", os.path.join(shim, "d1", "d2", "d3")]


def compile_one(args):
    src, obj, flags = args
    if os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src):
        return None
    r = subprocess.run(["g++"] + CXXFLAGS + flags + ["-c", src, "-o", obj],
                       capture_output=True, text=True)
    return None if r.returncode == 0 else (src, r.stderr[-2000:])


def build(ref, jobs):
    src_root = os.path.join(ref, "Src")
    if not os.path.isdir(src_root):
        raise SystemExit("reference sources not found at %s" % src_root)
    os.makedirs(os.path.join(OUT, "obj"), exist_ok=True)
    flags = make_shim(src_root) + ["-I", src_root]
    files = source_list(src_root)
    work = []
    for src in files:
        rel = os.path.relpath(src, src_root).replace(os.sep, "__")
        work.append((src, os.path.join(OUT, "obj", rel[:-4] + ".o"), flags))
    with ThreadPoolExecutor(jobs) as ex:
        errs = [e for e in ex.map(compile_one, work) if e]
    if errs:
        for src, msg in errs:
            sys.stderr.write("FAILED %s\n%s\n" % (src, msg))
        raise SystemExit(1)
    lib = os.path.join(OUT, "libboil.a")
    objs = [w[1] for w in work]
    if not os.path.exists(lib) or max(os.path.getmtime(o) for o in objs) > os.path.getmtime(lib):
        if os.path.exists(lib):
            os.remove(lib)
        subprocess.check_call(["ar", "rcs", lib] + objs)
    # fixture harness linked against the reference library
    harness = os.path.join(HERE, "ref_harness.cpp")
    exe = os.path.join(OUT, "ref_harness")
    deps = [harness, lib, os.path.join(REPO, "psiboil_b200", "csrc", "problem_gen.h")]
    if not os.path.exists(exe) or max(os.path.getmtime(d) for d in deps) > os.path.getmtime(exe):
        subprocess.check_call(["g++"] + CXXFLAGS + flags +
                              ["-I", os.path.join(REPO, "psiboil_b200", "csrc"),
                               harness, lib, "-o", exe])
    # the same harness with the engine's Krylov classes plugged in through
    # include/psiboil_b200_psiboil.hpp (needs the built engine library)
    englib = os.path.join(REPO, "psiboil_b200", "libpsiboil_b200.so")
    exe_gpu = os.path.join(OUT, "ref_harness_gpu")
    if os.path.exists(englib):
        deps_gpu = deps + [englib, os.path.join(REPO, "include", "psiboil_b200_psiboil.hpp"),
                           os.path.join(REPO, "include", "psiboil_b200.h")]
        if not os.path.exists(exe_gpu) or max(os.path.getmtime(d) for d in deps_gpu) > os.path.getmtime(exe_gpu):
            cuda = "/usr/local/cuda"
            subprocess.check_call(["g++"] + CXXFLAGS + flags + ["-DPBG_WITH_ENGINE",
                                  "-I", os.path.join(REPO, "psiboil_b200", "csrc"),
                                  "-I", os.path.join(REPO, "include"),
                                  harness, lib, englib, "-L", os.path.join(cuda, "lib64"), "-lcudart",
                                  "-Wl,-rpath,$ORIGIN/../../psiboil_b200",
                                  "-o", exe_gpu])
    print("reference built: %d sources -> %s" % (len(files), exe))
    return exe


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PBG_REFERENCE"),
                    help="PSI-BOIL source tree (default: $PBG_REFERENCE)")
    ap.add_argument("-j", type=int, default=os.cpu_count() or 4)
    a = ap.parse_args()
    if not a.ref:
        raise SystemExit("name the reference source tree: --ref DIR or PBG_REFERENCE=DIR")
    build(a.ref, a.j)
