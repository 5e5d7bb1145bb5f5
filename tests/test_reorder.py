"""Cell reordering (mesh/reorder.cpp, CuthillMckee) on the oracle.

The oracle restates the reference's algorithm with its own data structures
(degree-sorted node list, linear search of the not-visited deque, per-step
degree sort of the new neighbours), so its permutation is the reference's.
Checked here: the permutation is one, it brings a shuffled mesh's matrix
bandwidth down to that of a structured numbering, reverse is its reversal,
geometry and topology move with their cells, and a solve on the renumbered
mesh gives the same field up to the renumbering."""
import numpy as np
import pytest

from prism_b200 import PrismError, api, meshgen
from prism_b200 import _abi as A
from tests import cases


def _case():
    return cases.box_case({"T": {"left": ("fixed", 1.0), "right": ("fixed", 0.0)}})


def bandwidth(mesh):
    ex = mesh.export()
    rp, col = ex["csr_rowptr"], ex["csr_col"]
    rows = np.repeat(np.arange(mesh.n_cells), np.diff(rp))
    return int(np.abs(col[:rp[-1]] - rows).max())


def test_chain_pin(orc):
    # 1 x 1 x 5 chain in natural order: degrees 1,2,2,2,1; the first lowest-degree cell is 0
    mesh = api.Mesh(meshgen.box_hex(1, 1, 5), _case(), lib=orc)
    mesh.reorder()
    np.testing.assert_array_equal(mesh.export()["cell_original"], [0, 1, 2, 3, 4])
    mesh = api.Mesh(meshgen.box_hex(1, 1, 5), _case(), lib=orc)
    mesh.reorder(reverse=True)
    np.testing.assert_array_equal(mesh.export()["cell_original"], [4, 3, 2, 1, 0])


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_shuffled_bandwidth(orc, kind):
    n = 6
    unv = (meshgen.box_hex if kind == "hex" else meshgen.box_tet)(n, n, n)
    ref = api.Mesh(unv, _case(), lib=orc)
    shuffled = meshgen.shuffle_cells(unv, seed=1)
    mesh = api.Mesh(shuffled, _case(), lib=orc)
    before = mesh.export()
    bw0 = bandwidth(mesh)
    mesh.reorder(reverse=True)
    after = mesh.export()
    orig = after["cell_original"]
    assert sorted(orig) == list(range(mesh.n_cells))
    np.testing.assert_array_equal(after["cell_center"], before["cell_center"][:, orig])
    np.testing.assert_array_equal(after["cell_volume"], before["cell_volume"][orig])
    bw1 = bandwidth(mesh)
    print(f"{kind} {n}^3 shuffled: bandwidth {bw0} -> {bw1} (structured numbering {bandwidth(ref)})")
    assert bw1 <= 1.5 * bandwidth(ref) and bw1 < bw0 / 3
    # faces keep their ids; owner / neighbour are renamed
    new_id = np.empty_like(orig)
    new_id[orig] = np.arange(len(orig))
    np.testing.assert_array_equal(after["owner"], new_id[before["owner"]])
    inner = before["neighbor"] >= 0
    np.testing.assert_array_equal(after["neighbor"][inner], new_id[before["neighbor"][inner]])
    np.testing.assert_array_equal(after["face_center"], before["face_center"])
    # cell vertex lists move with their cells
    bo, bv = before["cell_vertex_offsets"], before["cell_vertices"]
    ao, av = after["cell_vertex_offsets"], after["cell_vertices"]
    for i in (0, len(orig) // 2, len(orig) - 1):
        np.testing.assert_array_equal(av[ao[i]:ao[i + 1]], bv[bo[orig[i]]:bo[orig[i] + 1]])


def test_reverse_is_reversal(orc):
    unv = meshgen.shuffle_cells(meshgen.box_tet(4, 4, 4, jitter=0.2, seed=3), seed=2)
    perm = {}
    for rev in (False, True):
        mesh = api.Mesh(unv, _case(), lib=orc)
        mesh.reorder(reverse=rev)
        perm[rev] = mesh.export()["cell_original"]
    np.testing.assert_array_equal(perm[True], perm[False][::-1])


def test_solution_follows_cells(orc):
    unv = meshgen.shuffle_cells(meshgen.box_hex(8, 8, 8, jitter=0.2, seed=4), seed=3)
    res = {}
    for reordered in (False, True):
        mesh = api.Mesh(unv, _case(), lib=orc)
        if reordered:
            mesh.reorder(reverse=True)
        T = api.Scalar("T", mesh, 0.0)
        k = api.Scalar("kappa", mesh, 1.0)
        eqn = api.Transport(api.diffusion.NonCorrected(k, T))
        api.BiCGSTAB().solve(eqn, 3, 1e-14)
        res[reordered] = (T.values(), mesh.export()["cell_original"])
    T0, _ = res[False]
    T1, orig = res[True]
    err = cases.rel_l2(T1, T0[orig])
    print(f"reordered vs original numbering: rel L2 {err:.2e}")
    assert err < 1e-10


def test_reorder_after_fields_rejected(orc):
    mesh = api.Mesh(meshgen.box_hex(3, 3, 3), _case(), lib=orc)
    api.Scalar("T", mesh, 0.0)
    with pytest.raises(PrismError) as e:
        mesh.reorder()
    assert e.value.status == A.BAD_ARG
