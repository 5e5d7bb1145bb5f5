"""The C++ mirror API (include/prism_b200.hpp): compiles and links against the
sm_100a library; on a GPU the example reproduces the oracle's Poisson solution."""
import os
import subprocess

import numpy as np
import pytest

from prism_b200 import api, io, meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "poisson_example.cpp")


def _compile(out):
    import prism_b200
    if not os.path.exists(prism_b200.LIB_PATH):
        pytest.skip("library not built")
    libdir = os.path.dirname(prism_b200.LIB_PATH)
    cmd = ["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-o", out,
           "-L", libdir, "-lprism_b200", f"-Wl,-rpath,{libdir}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_cpp_example_compiles(tmp_path):
    _compile(str(tmp_path / "poisson_example"))


@pytest.mark.gpu
def test_cpp_example_matches_oracle(tmp_path, orc):
    exe = str(tmp_path / "poisson_example")
    _compile(exe)
    n = 16
    out = subprocess.run([exe, str(n)], check=True, capture_output=True, text=True).stdout
    gpu_p = np.array([float(v) for v in out.split()])
    # the same case on the oracle through the Python mirror
    unv = meshgen.box_hex(n, n, 1, (1.0, 1.0, 0.1), origin=(0.0, -0.5, 0.0))
    case = io.Case.from_dict(meshgen.PATCHES, {"P": {p: ("fixed", 0.0) for p in ("left", "right", "bottom", "top")}
                                               | {"back": ("empty", None), "front": ("empty", None)}},
                             {"P": {"gradScheme": "greenGauss"}})
    mesh = api.Mesh(unv, case, lib=orc)
    cc = mesh.export()["cell_center"]
    P = api.Scalar("P", mesh, 0.0)
    S = api.Scalar("S", mesh, 2 * np.pi ** 2 * np.sin(np.pi * cc[0]) * np.cos(np.pi * cc[1]))
    eqn = api.Transport(api.diffusion.Corrected(api.Tensor("c", mesh, np.eye(3)), P), api.source.ConstantScalar(S))
    for _ in range(5):
        api.BiCGSTAB().solve(eqn, 15, 1e-20)
    ref = P.values()
    err = np.linalg.norm(gpu_p - ref) / np.linalg.norm(ref)
    print(f"C++ API Poisson {n}x{n}: rel L2 vs oracle {err:.3e}")
    assert err < 1e-8
