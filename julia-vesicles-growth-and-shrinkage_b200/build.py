"""Builds libvsav.so (the C-ABI CUDA library) in-tree for sm_100a.

    python julia-vesicles-growth-and-shrinkage_b200/build.py [--force]

Each .cu translation unit is compiled to an object in parallel (objects in
_build/, rebuilt when any source is newer), then linked into vsav/libvsav.so.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "vsav", "libvsav.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-diag-suppress", "177"]
UNITS = ("vsav.cu", "solver_f32.cu", "solver_f64.cu", "net.cu", "noalloc.cu")


def sources():
    return [os.path.join(SRC, f) for f in sorted(os.listdir(SRC)) if f.endswith((".cu", ".cuh"))] + \
        [os.path.join(os.path.dirname(HERE), "include", "vsav.h")]


def deps(path, seen=None):
    """path and every file it includes with #include "..." (recursively)."""
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    for line in open(path):
        line = line.strip()
        if line.startswith("#include \""):
            deps(os.path.join(os.path.dirname(path), line.split('"')[1]), seen)
    return seen


def up_to_date(path, inputs=None):
    inputs = sources() if inputs is None else inputs
    return os.path.exists(path) and os.path.getmtime(path) >= max(os.path.getmtime(s) for s in inputs)


def _compile(unit, verbose):
    obj = os.path.join(OBJ, unit.replace(".cu", ".o"))
    inputs = deps(os.path.join(SRC, unit))
    if up_to_date(obj, inputs):
        return obj
    # stamp the object with its inputs' newest time at the start, so that a source
    # edited while this compiles still counts as newer
    stamp = max(os.path.getmtime(s) for s in inputs)
    cmd = [NVCC] + FLAGS + ["-c", "-o", obj + ".tmp", os.path.join(SRC, unit)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(obj + ".tmp", obj)
    os.utime(obj, (stamp, stamp))
    return obj


def build(force=False, verbose=True):
    objs = [os.path.join(OBJ, u.replace(".cu", ".o")) for u in UNITS]
    if not force and all(up_to_date(o, deps(os.path.join(SRC, u))) for o, u in zip(objs, UNITS)) \
            and os.path.exists(OUT) and all(os.path.getmtime(o) <= os.path.getmtime(OUT) for o in objs):
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    if force:
        for u in UNITS:
            o = os.path.join(OBJ, u.replace(".cu", ".o"))
            if os.path.exists(o):
                os.remove(o)
    with ThreadPoolExecutor(len(UNITS)) as ex:
        objs = list(ex.map(lambda u: _compile(u, verbose), UNITS))
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT + ".tmp"] + objs
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
