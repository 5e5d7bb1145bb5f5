"""Build libprism_b200.so in-tree for sm_100a with nvcc.

Kernels that reproduce the reference's arithmetic term for term (assembly,
gradients, pressure-velocity coupling) are compiled with --fmad=false so no
multiply-add is contracted; the Krylov kernels keep FMA. Host code is compiled
with -ffp-contract=off for the same reason (mesh geometry, least-squares
operators).

    python -m prism_b200.build [--force] [-j N]
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libprism_b200.so")
OBJ = os.path.join(HERE, "..", "_build", "obj")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-O2"]
NO_FMA = {"assemble.cu", "gradient.cu", "coupling.cu", "pattern.cu", "adjoint.cu", "diag.cu"}
SOURCES = ["mesh_build.cpp", "runtime.cpp", "capi.cpp", "pattern.cu", "assemble.cu", "gradient.cu",
           "coupling.cu", "krylov.cu", "amg.cu", "adjoint.cu", "batched.cu", "noalloc.cu", "diag.cu"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + \
        [os.path.join(HERE, "..", "include", "prism_b200.h")]


def _compile(src, force):
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJ, src + ".o")
    newest = max(os.path.getmtime(p) for p in _deps())
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    flags = list(COMMON)
    if src.endswith(".cu"):
        flags += ARCH + (["--fmad=false"] if src in NO_FMA else [])
        flags += ["-Xptxas", "-v"] if os.environ.get("PRISM_PTXAS_VERBOSE") else []
    else:
        flags += ["-x", "c++"]
    cmd = [nvcc()] + flags + ["-c", path, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    if res.stderr.strip() and os.environ.get("PRISM_PTXAS_VERBOSE"):
        sys.stderr.write(res.stderr)
    return obj


def build(force=False, jobs=8):
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), SOURCES))
    newest = max(os.path.getmtime(o) for o in objs)
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest:
        return OUT
    cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT + ".tmp"] + objs + ["-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j))
