"""The CPU oracle against the reference's own known answers (its Catch2 tests),
on the reference's own meshes (tests/golden/*.npz, re-encoded from the
reference's tests/cases). These pins are what makes the oracle trustworthy."""
import numpy as np
import pytest

from prism_b200 import api
from tests import cases


def test_poisson_structured_pin(orc):
    # tests/test_poisson.cpp:58-62: relative L2 error < 4e-4 on poisson/mesh_hex.unv
    unv, case, _ = cases.load_golden("poisson_hex")
    r = cases.poisson_reference(unv, case, orc)
    assert r["rel_l2"] < 4e-4


def test_poisson_unstructured_pin(orc):
    # tests/test_poisson.cpp:52-56: relative L2 error < 0.078 on poisson/mesh.unv (wedges)
    unv, case, _ = cases.load_golden("poisson_wedge")
    r = cases.poisson_reference(unv, case, orc)
    assert r["rel_l2"] < 0.078


def test_advection_1d_pin(orc):
    # tests/test_advection_1d.cpp:52-64: ||T - T_exact|| < 0.25 ("around 0.209"), monotone
    unv, case, _ = cases.load_golden("versteeg_advection_1d")
    r = cases.advection_reference(unv, case, orc)
    assert r["diff_norm"] < 0.25
    assert abs(float(r["diff_norm"]) - 0.209) < 5e-4
    assert np.all(np.diff(r["T"]) <= 0)


def test_simple_coarse_pipe_pin(orc):
    # tests/test_simple_coarse_pipe.cpp:36-49 against OpenFOAM after 100 SIMPLE iterations
    unv, case, extra = cases.load_golden("coarse_pipe")
    r = cases.simple_reference(unv, case, orc, 100)
    assert cases.rel_l2(r["p"], extra["foam_p"]) < 0.005
    assert cases.rel_l2(r["U"][0], extra["foam_U"][:, 0]) < 0.005
    assert cases.rel_l2(r["U"][1], extra["foam_U"][:, 1]) < 0.09
    rates = dict(zip(case.patch_names, r["rates"]))
    assert abs(rates["Inlet"] + rates["Outlet"]) / abs(rates["Inlet"]) < 1e-6
    assert not r["needs_ref"]


@pytest.mark.parametrize("name, expected", [("cavity_hex", True), ("coarse_pipe", False),
                                            ("duct_simple", False)])
def test_needs_pressure_reference_pin(orc, name, expected):
    # tests/test_needs_pressure_ref.cpp:10-29
    unv, case, _ = cases.load_golden(name)
    mesh = api.Mesh(unv, case, lib=orc)
    p = api.Scalar("P", mesh, 0.0)
    assert api.needs_pressure_reference(p) == expected


def test_simple_duct_symmetry_pin(orc):
    # tests/test_simple_duct_symmetry.cpp:38-53: duct with a symmetry plane against OpenFOAM
    unv, case, extra = cases.load_golden("duct_simple")
    r = cases.run_reference_test("duct_simple", orc)
    assert cases.rel_l2(r["p"], extra["foam_p"]) < 0.025
    assert cases.rel_l2(r["U"][0], extra["foam_U"][:, 0]) < 0.07
    assert cases.rel_l2(r["U"][1], extra["foam_U"][:, 1]) < 0.007
    assert not r["needs_ref"]
    # the stored oracle result (compared with the GPU path on the B200) is this run, bit for bit
    ref = cases.load_oracle_results("duct_simple")
    for k in ref:
        np.testing.assert_array_equal(r[k], ref[k], err_msg=f"duct_simple:{k}")


def test_golden_files_match_oracle(orc):
    # the stored oracle results are reproduced bit for bit by the current oracle
    for name in ("poisson_hex", "poisson_wedge", "versteeg_advection_1d", "versteeg_trans_1d", "cavity_hex",
                 "coarse_pipe"):
        ref = cases.load_oracle_results(name)
        got = cases.run_reference_test(name, orc)
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{name}:{k}")


def _tridiag(n=10):
    # tests/test_solver.cpp:10-33: 4 on the diagonal, -1 off-diagonal, b = A * ones
    rp, col, val = [0], [], []
    for i in range(n):
        for j in (i - 1, i, i + 1):
            if 0 <= j < n:
                col.append(j)
                val.append(4.0 if i == j else -1.0)
        rp.append(len(col))
    A = np.zeros((n, n))
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            A[i, col[k]] = val[k]
    x_exact = np.arange(1, n + 1, dtype=float)
    return np.array(rp), np.array(col), np.array(val), A @ x_exact, x_exact


@pytest.mark.parametrize("solver", [api.BiCGSTAB, api.Jacobi])
def test_solver_tridiagonal_pin(orc, solver):
    # tests/test_solver.cpp:35-57: 20 steps reach a relative L2 error below 1e-4
    rp, col, val, b, x_exact = _tridiag()
    x = np.zeros(10)
    s = solver()
    for _ in range(20):
        x = s.step(orc, rp, col, val, x, b)
    assert np.linalg.norm(x - x_exact) / np.linalg.norm(x_exact) < 1e-4


def test_transient_1d_pin(orc):
    # tests/test_transient_1d.cpp:70-82: errors at t = 40 and 60 below 0.10 and decreasing,
    # below 0.02 after 200 steps (AdamMoulton + Corrected, dt = 2)
    got = cases.run_reference_test("versteeg_trans_1d", orc)
    n40, n60 = got["diff_norms"]
    assert n40 < 0.10 and n60 < 0.10 and n60 < n40
    assert got["final_diff_norm"] < 0.02
    ref = cases.load_oracle_results("versteeg_trans_1d")
    np.testing.assert_array_equal(got["T"], ref["T"])


def _history_sections(lib):
    """tests/test_scalar_history.cpp:6-132, section by section, on the advection mesh."""
    unv, case, _ = cases.load_golden("versteeg_advection_1d")
    mesh = api.Mesh(unv, case, lib=lib)
    n = mesh.n_cells
    t = [np.full(n, float(k + 1)) for k in range(6)]

    def fresh():
        return api.Scalar("T", mesh, t[0])

    # basic tracking
    T = fresh()
    T.set_history_size(3)
    assert T.prev_values() is None
    T.update(t[1])
    np.testing.assert_array_equal(T.values(), t[1])
    np.testing.assert_array_equal(T.prev_values(), t[0])
    assert T.prev_prev_values() is None
    T.update(t[2])
    np.testing.assert_array_equal(T.prev_values(), t[1])
    np.testing.assert_array_equal(T.prev_prev_values(), t[0])
    assert T.history(3) is None
    T.update(t[3])
    np.testing.assert_array_equal(T.history(2), t[0])
    T.update(t[4])
    np.testing.assert_array_equal(T.values(), t[4])
    np.testing.assert_array_equal(T.prev_values(), t[3])
    np.testing.assert_array_equal(T.prev_prev_values(), t[2])
    np.testing.assert_array_equal(T.history(2), t[1])
    assert T.history(3) is None
    # truncation
    T = fresh()
    T.set_history_size(4)
    for k in range(1, 5):
        T.update(t[k])
    for i in range(4):
        np.testing.assert_array_equal(T.history(i), t[3 - i])
    T.set_history_size(2)
    np.testing.assert_array_equal(T.history(0), t[3])
    np.testing.assert_array_equal(T.history(1), t[2])
    assert T.history(2) is None
    T.update(t[5])
    np.testing.assert_array_equal(T.prev_values(), t[4])
    np.testing.assert_array_equal(T.prev_prev_values(), t[3])
    assert T.history(2) is None
    # expansion
    T = fresh()
    T.set_history_size(1)
    T.update(t[1])
    T.update(t[2])
    np.testing.assert_array_equal(T.prev_values(), t[1])
    assert T.prev_prev_values() is None
    T.set_history_size(3)
    np.testing.assert_array_equal(T.prev_values(), t[1])
    assert T.prev_prev_values() is None
    T.update(t[3])
    np.testing.assert_array_equal(T.prev_values(), t[2])
    np.testing.assert_array_equal(T.prev_prev_values(), t[1])
    T.update(t[4])
    np.testing.assert_array_equal(T.history(2), t[1])
    # clearing
    T = fresh()
    T.set_history_size(2)
    T.update(t[1])
    T.update(t[2])
    assert T.prev_values() is not None
    T.set_history_size(0)
    assert T.prev_values() is None and T.prev_prev_values() is None
    T.update(t[3])
    assert T.prev_values() is None


def test_scalar_history_pin(orc):
    _history_sections(orc)
