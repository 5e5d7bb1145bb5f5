"""Cell reordering on the GPU library vs the oracle.

The library computes the reference's Cuthill-McKee permutation in O(n log n)
(an enqueued flag per cell instead of the linear search of a deque); the
oracle restates the reference's O(n^2) procedure. The permutations, and the
renumbered meshes built from them, must be identical; a SIMPLE run on the
renumbered mesh must agree with the oracle's on the same numbering; and on a
shuffled 128^3 mesh the renumbering must restore a narrow matrix band."""
import time

import numpy as np
import pytest

from prism_b200 import api, meshgen
from tests import cases
from tests.test_reorder import _case, bandwidth

pytestmark = pytest.mark.gpu

KEYS = ("cell_original", "cell_center", "cell_volume", "owner", "neighbor", "csr_rowptr", "csr_col",
        "cell_face_offsets", "cell_faces", "cell_vertex_offsets", "cell_vertices")


def _meshes():
    unv_w, case_w, _ = cases.load_golden("poisson_wedge")
    unv_p, case_p, _ = cases.load_golden("coarse_pipe")
    return {
        "hex-shuffled": (meshgen.shuffle_cells(meshgen.box_hex(10, 9, 8, jitter=0.2, seed=1), seed=5), _case()),
        "tet-shuffled": (meshgen.shuffle_cells(meshgen.box_tet(5, 5, 5, jitter=0.2, seed=2), seed=6), _case()),
        "tet": (meshgen.box_tet(4, 4, 4), _case()),
        "wedge": (unv_w, case_w),
        "pipe": (unv_p, case_p),
    }


@pytest.mark.parametrize("reverse", [False, True])
@pytest.mark.parametrize("name", ["hex-shuffled", "tet-shuffled", "tet", "wedge", "pipe"])
def test_permutation_matches_oracle(gpu, orc, name, reverse):
    unv, case = _meshes()[name]
    out = {}
    for which, lib in (("gpu", gpu), ("orc", orc)):
        mesh = api.Mesh(unv, case, lib=lib)
        mesh.reorder(reverse=reverse)
        out[which] = mesh.export()
    for k in KEYS:
        np.testing.assert_array_equal(out["gpu"][k], out["orc"][k], err_msg=f"{name}:{k}")


def test_simple_on_reordered_mesh(gpu, orc):
    out = {}
    for which, lib in (("gpu", gpu), ("orc", orc)):
        unv = meshgen.shuffle_cells(meshgen.box_hex(16, 16, 1, (1.0, 1.0, 1.0 / 16)), seed=3)
        wall = ("no-slip", [0.0, 0.0, 0.0])
        case = cases.box_case({"U": {"top": ("fixed", [1.0, 0.0, 0.0]), "left": wall, "right": wall,
                                     "bottom": wall, "back": ("empty", None), "front": ("empty", None)},
                               "P": {"back": ("empty", None), "front": ("empty", None)}})
        mesh = api.Mesh(unv, case, lib=lib)
        mesh.reorder(reverse=True)
        U, p, nu, mdot = cases.simple_fields(mesh, 0.01)
        eqs = cases.momentum_eqns(U, p, nu, mdot, conv="Upwind")
        simple = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=api.BiCGSTAB())
        for _ in range(8):
            simple.step(eqs, U, mdot, p)
        out[which] = (U.values(), p.values(), mdot.face_flux())
    for i, k in enumerate(("U", "p", "mdot")):
        err = cases.rel_l2(out["gpu"][i], out["orc"][i])
        print(f"reordered cavity 16x16 {k}: rel L2 vs oracle {err:.3e}")
        assert err < 1e-8


def test_large_shuffled_mesh(gpu):
    n = 128
    unv = meshgen.shuffle_cells(meshgen.box_hex(n, n, n), seed=7)
    mesh = api.Mesh(unv, _case(), lib=gpu)
    bw0 = bandwidth(mesh)
    t0 = time.perf_counter()
    mesh.reorder(reverse=True)
    dt = time.perf_counter() - t0
    bw1 = bandwidth(mesh)
    orig = mesh.export()["cell_original"]
    print(f"128^3 shuffled hex: reorder {dt * 1e3:.0f} ms, bandwidth {bw0} -> {bw1}")
    assert np.array_equal(np.sort(orig), np.arange(n ** 3))
    assert bw1 <= 2 * n * n
    # the renumbered mesh solves like any other
    T = api.Scalar("T", mesh, 0.0)
    k = api.Scalar("kappa", mesh, 1.0)
    r = api.BiCGSTAB(krylov_tol=1e-10).solve(api.Transport(api.diffusion.NonCorrected(k, T)), 1, 0.0)
    assert r.status == 0
    x = mesh.export()["cell_center"][0]
    assert np.abs(T.values() - (1.0 - x)).max() < 1e-6
