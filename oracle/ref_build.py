"""Build recipe of oracle/_ref/libprism_ref.so: the reference's own sources,
compiled where they lie (test infrastructure; nothing in the product loads it).

The reference (src/prism) is C++20 on Eigen3, spdlog/fmt, nlohmann::json and the
unvpp UNV reader. Eigen and unvpp are absent from this image and the reference's
build system (CMake + vcpkg) is not run. Instead its .cpp files are compiled
directly with g++ -O2 (its release flags, CMakeLists.txt:30-37) against:
  * project-written API shims under oracle/ref/shim (Eigen, unvpp, spdlog);
  * the header-only fmt 12 bundled with torch and nlohmann::json bundled with
    cudnn_frontend, both already in this image's site-packages;
plus oracle/ref/ref_cases.cpp, the project's extern "C" driver over the
reference's public C++ API. export.cpp (VTU output through the absent vtu11) and
turbulence/ (outside the path) are left out. Outputs go to oracle/_ref/ only.

    python -m oracle.ref_build [--force] [--reference PATH]
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libprism_ref.so")
SHIM = os.path.join(HERE, "ref", "shim")
DRIVER = os.path.join(HERE, "ref", "ref_cases.cpp")
EXCLUDE = {"export.cpp"}
EXCLUDE_DIRS = {"turbulence"}  # outside the path; KOmega.cpp references an undefined kProduction()


def _site():
    import sysconfig
    return sysconfig.get_paths()["purelib"]


def include_dirs():
    sp = _site()
    return [SHIM, os.path.join(sp, "torch", "include"),
            os.path.join(sp, "include", "cudnn_frontend", "thirdparty")]


def sources(ref_root):
    src = os.path.join(ref_root, "src", "prism")
    out = []
    for d, _, files in os.walk(src):
        if os.path.basename(d) in EXCLUDE_DIRS:
            continue
        for f in sorted(files):
            if f.endswith(".cpp") and f not in EXCLUDE:
                out.append(os.path.join(d, f))
    return sorted(out)


def flags(ref_root):
    f = ["-std=c++20", "-O2", "-fPIC", "-ffp-contract=off", "-DFMT_HEADER_ONLY", "-w"]
    for d in include_dirs() + [os.path.join(ref_root, "src")]:
        f += ["-I", d]
    return f


def _obj(path, ref_root):
    rel = os.path.relpath(path, ref_root) if path.startswith(ref_root) else os.path.basename(path)
    return os.path.join(OUT_DIR, "obj", rel.replace(os.sep, "_") + ".o")


def _deps():
    out = [DRIVER, __file__]
    for d, _, files in os.walk(SHIM):
        out += [os.path.join(d, f) for f in files]
    return out


def _compile(path, ref_root, force):
    obj = _obj(path, ref_root)
    newest = max(os.path.getmtime(p) for p in _deps() + [path])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, None
    cmd = ["g++"] + flags(ref_root) + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return None, f"{path}:\n{r.stderr[-4000:]}"
    return obj, None


def build(ref_root="/root/reference", force=False, jobs=8):
    """Compile the reference's sources and the driver into oracle/_ref/libprism_ref.so.
    Returns the library path, or None when the reference tree is absent."""
    if not os.path.isdir(os.path.join(ref_root, "src", "prism")):
        return None
    os.makedirs(os.path.join(OUT_DIR, "obj"), exist_ok=True)
    srcs = sources(ref_root) + [DRIVER]
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        res = list(ex.map(lambda p: _compile(p, ref_root, force), srcs))
    errs = [e for _, e in res if e]
    if errs:
        raise RuntimeError("reference build failed:\n" + "\n".join(errs))
    objs = [o for o, _ in res]
    newest = max(os.path.getmtime(o) for o in objs)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    cmd = ["g++", "-shared", "-Wl,--no-undefined", "-o", LIB + ".tmp"] + objs
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--reference", default="/root/reference")
    a = ap.parse_args()
    try:
        print(build(a.reference, a.force))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
