"""The device-memory arena of the AMG hierarchy (pb::DevArena in
prism_b200/csrc/common.h), checked on the host: tests/cpp/arena_check.cpp
compiles the header against fake CUDA allocation calls and replays random
hierarchy-shaped build sequences (alignment, containment, no overlap of live
buffers, geometric chunk growth, every chunk returned)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "arena_check.cpp")


def _cuda_include():
    for home in (os.environ.get("CUDA_HOME"), os.environ.get("CUDA_PATH"), "/usr/local/cuda"):
        if home and os.path.exists(os.path.join(home, "include", "cuda_runtime.h")):
            return os.path.join(home, "include")
    nvcc = shutil.which("nvcc")
    if nvcc:
        inc = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "include")
        if os.path.exists(os.path.join(inc, "cuda_runtime.h")):
            return inc
    return None


def test_arena_logic(tmp_path):
    inc = _cuda_include()
    if inc is None or shutil.which("g++") is None:
        pytest.skip("needs g++ and the CUDA headers")
    exe = str(tmp_path / "arena_check")
    subprocess.run(["g++", "-std=c++20", "-O1", "-I", inc, SRC, "-o", exe], check=True, capture_output=True,
                   text=True)
    out = subprocess.run([exe], capture_output=True, text=True)
    print(out.stdout, out.stderr)
    assert out.returncode == 0, out.stderr
