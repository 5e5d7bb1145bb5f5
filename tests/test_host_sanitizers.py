"""Host code under AddressSanitizer and UndefinedBehaviorSanitizer (CPU): the
library's host mesh builder, and the CPU oracle every parity test compares with.

prism_b200/csrc/mesh_build.cpp is the index-heavy host part of the library: UNV
elements to faces (counting-sort face matching, the reference's face order,
unv.cpp:124-372 and pmesh.cpp:10-119), face and cell geometry on host threads,
and the Cuthill-McKee renumbering (reorder.cpp:8-130). Here it is compiled with
-fsanitize=address,undefined beside a small C shim (tests/cpp/mesh_build_check.cpp)
and driven from a child Python process with the ASan runtime preloaded, on the
reference's meshes and on generated hex and tet boxes, plain and renumbered
(forward and reversed). Any sanitizer report makes the child exit non-zero. The
arrays it builds are compared with the oracle's converter along the way, so the
run covers what the device upload reads.

The oracle (oracle/prism_oracle.cpp) is compiled the same way and runs the
reference's own test cases and the synthetic configurations (SIMPLE, transient,
advection, MUSCL transport with Green-Gauss gradients, least squares on tets,
renumbered meshes, diagnostics); every result must equal, bit for bit, the one of
the ordinary oracle build.
"""
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SRC = os.path.join(ROOT, "oracle", "prism_oracle.cpp")
SHIM = os.path.join(ROOT, "tests", "cpp", "mesh_build_check.cpp")
BUILDER = os.path.join(ROOT, "prism_b200", "csrc", "mesh_build.cpp")

CHILD = r"""
import ctypes as C
import sys

import numpy as np

sys.path.insert(0, sys.argv[2])
import oracle
from prism_b200 import _abi as A
from prism_b200 import api, meshgen
from tests import cases


class Shim:
    # the two entry points api.Mesh calls, served by the sanitized host builder
    def __init__(self, path):
        self.so = C.CDLL(path)
        self.so.mb_last_error.restype = C.c_char_p
        self.mesh_from_unv = self.so.mb_mesh_from_unv
        self.mesh_from_unv.argtypes = [C.POINTER(A.UnvMesh), C.POINTER(C.c_void_p)]
        self.mesh_info = self.so.mb_mesh_info
        self.mesh_info.argtypes = [C.c_void_p, C.POINTER(A.MeshInfo)]
        self.so.mb_reorder.argtypes = [C.c_void_p, C.c_int]
        self.so.mb_export.argtypes = [C.c_void_p] + [C.c_void_p] * 7
        self.so.mb_destroy.argtypes = [C.c_void_p]

    def check(self, status):
        if status != 0:
            raise RuntimeError(self.so.mb_last_error().decode())

    def export(self, mesh):
        i = mesh.info
        nc, nf = i.n_cells, i.n_faces
        owner, nbr = np.zeros(nf, np.int32), np.zeros(nf, np.int32)
        area, vol, cc = np.zeros(nf), np.zeros(nc), np.zeros(3 * nc)
        cf_off = np.zeros(nc + 1, np.int64)
        self.so.mb_export(mesh.h, owner.ctypes.data, nbr.ctypes.data, area.ctypes.data, vol.ctypes.data,
                          cc.ctypes.data, cf_off.ctypes.data, None)
        cf = np.zeros(max(1, int(cf_off[-1])), np.int32)
        self.so.mb_export(mesh.h, owner.ctypes.data, nbr.ctypes.data, area.ctypes.data, vol.ctypes.data,
                          cc.ctypes.data, cf_off.ctypes.data, cf.ctypes.data)
        return owner, nbr, area, vol, cc.reshape(3, nc), cf_off, cf[:cf_off[-1]]


shim, orc = Shim(sys.argv[1]), oracle.lib()
meshes = [(name, *cases.load_golden(name)[:2]) for name in ("cavity_hex", "coarse_pipe", "duct_simple",
                                                             "poisson_hex", "poisson_wedge")]
box = cases.box_case({"T": {}})
meshes += [("hex_jitter", meshgen.box_hex(7, 5, 6, jitter=0.2, seed=1), box),
           ("tets", meshgen.box_tet(4, 5, 3, jitter=0.15, seed=2), box),
           ("hex_shuffled", meshgen.shuffle_cells(meshgen.box_hex(6, 6, 5, jitter=0.1, seed=4), seed=5), box)]
checked = 0
for name, unv, case in meshes:
    for reorder in (None, False, True):
        s = api.Mesh(unv, case, lib=shim)
        o = api.Mesh(unv, case, lib=orc)
        if reorder is not None:
            shim.check(shim.so.mb_reorder(s.h, 1 if reorder else 0))
            o.reorder(reverse=reorder)
        owner, nbr, area, vol, cc, cf_off, cf = shim.export(s)
        e = o.export()
        assert s.info.n_cells == o.info.n_cells and s.info.n_faces == o.info.n_faces, name
        assert s.info.n_boundary_faces == o.info.n_boundary_faces, name
        np.testing.assert_array_equal(owner, e["owner"], err_msg=name)
        np.testing.assert_array_equal(np.where(nbr < 0, -1, nbr), np.where(e["neighbor"] < 0, -1, e["neighbor"]),
                                      err_msg=name)
        np.testing.assert_array_equal(area, e["face_area"], err_msg=name)
        np.testing.assert_array_equal(vol, e["cell_volume"], err_msg=name)
        np.testing.assert_array_equal(cc, e["cell_center"], err_msg=name)
        np.testing.assert_array_equal(cf_off, e["cell_face_offsets"], err_msg=name)
        np.testing.assert_array_equal(cf, e["cell_faces"][:len(cf)], err_msg=name)
        shim.so.mb_destroy(s.h)
        checked += 1
print(f"sanitized host mesh builds: {checked}")
"""


def _toolchain():
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not found")
    asan = subprocess.run([gxx, "-print-file-name=libasan.so"], capture_output=True, text=True).stdout.strip()
    if not asan or not os.path.exists(asan):
        pytest.skip("the AddressSanitizer runtime is not installed")
    cuda_inc = None
    for cand in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if cand and os.path.exists(os.path.join(cand, "include", "cuda_runtime.h")):
            cuda_inc = os.path.join(cand, "include")
            break
    if cuda_inc is None:
        pytest.skip("CUDA headers not found")
    return gxx, asan, cuda_inc


def test_mesh_builder_under_asan_and_ubsan(tmp_path):
    gxx, asan, cuda_inc = _toolchain()
    so = str(tmp_path / "libmesh_build_check.so")
    cmd = [gxx, "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=undefined", "-fPIC", "-shared", "-pthread", "-I", cuda_inc, "-I",
           os.path.join(ROOT, "include"), SHIM, BUILDER, "-o", so]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    env = dict(os.environ, LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0:exitcode=23",
               UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1:exitcode=24")
    r = subprocess.run([sys.executable, "-c", CHILD, so, ROOT], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-4000:])
    assert "sanitized host mesh builds: 24" in r.stdout, r.stdout[-2000:]


ORACLE_CHILD = r"""
import ctypes as C
import sys

import numpy as np

sys.path.insert(0, sys.argv[2])
import oracle
from prism_b200 import _abi as A
from prism_b200 import api, meshgen
from tests import cases

san, plain = A.bind(C.CDLL(sys.argv[1]), "orc_"), oracle.lib()


def same(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, what
    if a.dtype.kind in "fc":
        assert np.array_equal(a, b, equal_nan=True), what
    else:
        assert np.array_equal(a, b), what


def refcases(lib):
    out = {}
    for name in ("cavity_hex", "versteeg_advection_1d", "versteeg_trans_1d", "poisson_wedge"):
        r = cases.run_reference_test(name, lib)
        out[name] = r if isinstance(r, dict) else {"x": r}
    unv, case, _ = cases.load_golden("duct_simple")
    out["duct"] = cases.simple_reference(unv, case, lib, 8, symmetry=True)
    return out


def synthetic(lib):
    out = {}
    mesh, T, U, eqn = cases.transport_c3(6, lib, conv="MUSCL")
    for _ in range(2):
        api.BiCGSTAB().solve(eqn, 2, 1e-12)
    out["muscl"] = T.values()
    c = cases.adjoint_c5(2, lib)
    api.BiCGSTAB().solve(c["eqn"], 5, 1e-12)
    out["tets_ls"] = c["T"].values()
    m2, U2, p2, nu2, mdot2, eqs2 = cases.cavity(12, lib)
    simple = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=api.BiCGSTAB())
    for _ in range(4):
        simple.step(eqs2, U2, mdot2, p2)
    out["cavity_U"], out["cavity_p"] = U2.values(), p2.values()
    out["div"] = api.ops.div(mdot2).values()
    unv = meshgen.shuffle_cells(meshgen.box_hex(5, 4, 3, jitter=0.1, seed=4), seed=5)
    mesh = api.Mesh(unv, cases.box_case({"T": {"left": ("fixed", 1.0)}}), lib=lib)
    mesh.reorder(reverse=True)
    T = api.Scalar("T", mesh, 0.0)
    eqn = api.Transport(api.diffusion.Corrected(api.Scalar("k", mesh, 1.0), T))
    api.BiCGSTAB().solve(eqn, 3, 1e-12)
    out["reordered"] = T.values()
    return out


checked = 0
for name, fn in (("reference cases", refcases), ("synthetic", synthetic)):
    a, b = fn(san), fn(plain)
    for k in b:
        if isinstance(b[k], dict):
            for kk in b[k]:
                same(a[k][kk], b[k][kk], f"{k}.{kk}")
                checked += 1
        else:
            same(a[k], b[k], k)
            checked += 1
print(f"sanitized oracle results equal: {checked}")
"""


def test_oracle_under_asan_and_ubsan(tmp_path):
    gxx, asan, _ = _toolchain()
    so = str(tmp_path / "liboracle_sanitized.so")
    cmd = [gxx, "-std=c++20", "-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=undefined", "-fPIC", "-shared", "-fvisibility=hidden", "-ffp-contract=off",
           ORACLE_SRC, "-o", so]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    env = dict(os.environ, LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0:exitcode=23",
               UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1:exitcode=24")
    r = subprocess.run([sys.executable, "-c", ORACLE_CHILD, so, ROOT], env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-4000:])
    assert "sanitized oracle results equal" in r.stdout, r.stdout[-2000:]
