"""Linear solves and the pressure-velocity drivers on the GPU vs the oracle.

The oracle's step() is Eigen-style ILUT-BiCGSTAB to machine precision; the GPU
step is Jacobi-preconditioned BiCGSTAB to ||b - Ax|| <= 1e-12 ||b|| (FP64) or
FP32 inner iterations in FP64 refinement (mixed). Solved fields must agree with
the oracle within 1e-8 relative L2 (the error is printed)."""
import numpy as np
import pytest

from prism_b200 import _abi as A
from prism_b200 import api
from tests import cases
from tests.test_oracle_pins import _tridiag

pytestmark = pytest.mark.gpu
SOL_TOL = 1e-8


@pytest.mark.parametrize("solver", [api.BiCGSTAB, api.Jacobi])
def test_solver_tridiagonal(gpu, solver):
    # tests/test_solver.cpp:35-57
    rp, col, val, b, x_exact = _tridiag()
    x = np.zeros(10)
    s = solver()
    for _ in range(20):
        x = s.step(gpu, rp, col, val, x, b)
    assert np.linalg.norm(x - x_exact) / np.linalg.norm(x_exact) < 1e-4


def test_jacobi_step_matches_oracle(gpu, orc):
    rng = np.random.default_rng(1)
    rp, col, val, b, _ = _tridiag(10)
    x0 = rng.normal(size=10)
    xg = api.Jacobi().step(gpu, rp, col, val, x0, b)
    xo = api.Jacobi().step(orc, rp, col, val, x0, b)
    np.testing.assert_allclose(xg, xo, rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
def test_poisson_c1_solve(gpu, orc, precision):
    res = {}
    for name, lib, solver in (("gpu", gpu, api.BiCGSTAB(precision=precision, krylov_tol=1e-12)),
                              ("orc", orc, api.BiCGSTAB())):
        mesh, P, eqn, exact = cases.poisson_c1(32, lib)
        r = solver.solve(eqn, 3, 1e-10)
        res[name] = (P.values(), r, exact)
    err = cases.rel_l2(res["gpu"][0], res["orc"][0])
    print(f"C1 32x32 precision={precision}: rel L2 vs oracle {err:.3e}, krylov it {res['gpu'][1].krylov_iterations}")
    assert err < SOL_TOL
    assert res["gpu"][1].converged


def test_auto_preconditioner_picks_by_diagonal_dominance(gpu):
    """PRISM_PC_AUTO at AMG sizes (36,864 rows): an equation relaxed by 0.7 is diagonally
    dominant (off-diagonal row sums 0.7 of the diagonal) and keeps Jacobi, bit for bit
    the solve that asks for Jacobi; the same equation unrelaxed gets AMG, bit for bit the
    solve that asks for AMG."""
    def solve(pc, urf):
        mesh, U, p, nu, mdot, eqs = cases.cavity(192, gpu)
        U.set_values(np.random.default_rng(5).normal(size=(3, mesh.n_cells)) * 0.1)
        eq = eqs[0]
        eq.set_under_relax_factor(urf)
        r = api.BiCGSTAB(preconditioner=pc, krylov_tol=1e-12).solve(eq, 1, 0.0)
        return U.values()[0], r.krylov_iterations
    for urf, expect in ((0.7, "jacobi"), (1.0, "amg")):
        auto, its = solve("auto", urf)
        forced, its_f = solve(expect, urf)
        other, _ = solve("amg" if expect == "jacobi" else "jacobi", urf)
        print(f"urf {urf}: auto took {expect} ({its} Krylov iterations, forced {its_f})")
        np.testing.assert_array_equal(auto, forced)
        assert not np.array_equal(auto, other)


@pytest.mark.parametrize("n", [32, 128])
def test_poisson_c1_flexible_cg(gpu, orc, n):
    """PRISM_SOLVER_FCG (flexible CG, FP32 AMG V-cycle) on the symmetric C1 Poisson system,
    at its stated 128^2 too, against the oracle's ILUT-BiCGSTAB."""
    res = {}
    for name, lib, solver in (("gpu", gpu, api.FCG(krylov_tol=1e-12)), ("orc", orc, api.BiCGSTAB())):
        mesh, P, eqn, exact = cases.poisson_c1(n, lib)
        r = solver.solve(eqn, 3, 1e-10)
        res[name] = (P.values(), r)
    err = cases.rel_l2(res["gpu"][0], res["orc"][0])
    print(f"C1 {n}x{n} flexible CG: rel L2 vs oracle {err:.3e}, krylov it {res['gpu'][1].krylov_iterations}")
    assert err < SOL_TOL
    assert res["gpu"][1].converged and res["gpu"][1].status == A.OK


@pytest.mark.parametrize("name", ["poisson_hex", "poisson_wedge", "versteeg_advection_1d"])
def test_reference_cases(gpu, name):
    ref = cases.load_oracle_results(name)
    got = cases.run_reference_test(name, gpu)
    key = {"poisson_hex": "P", "poisson_wedge": "P", "versteeg_advection_1d": "T"}[name]
    err = cases.rel_l2(got[key], ref[key])
    print(f"{name}: rel L2 vs oracle {err:.3e}")
    assert err < SOL_TOL
    if name == "poisson_hex":
        assert got["rel_l2"] < 4e-4        # tests/test_poisson.cpp:58-62
    if name == "poisson_wedge":
        assert got["rel_l2"] < 0.078       # tests/test_poisson.cpp:52-56
    if name == "versteeg_advection_1d":
        assert got["diff_norm"] < 0.25 and np.all(np.diff(got["T"]) <= 0)


@pytest.mark.parametrize("name", ["coarse_pipe", "cavity_hex", "duct_simple"])
def test_simple_reference_cases(gpu, name):
    unv, case, extra = cases.load_golden(name)
    ref = cases.load_oracle_results(name)
    got = cases.run_reference_test(name, gpu)
    for k in ("p", "U"):
        err = cases.rel_l2(got[k], ref[k])
        print(f"{name} {k}: rel L2 vs oracle {err:.3e}")
        assert err < SOL_TOL
    assert bool(got["needs_ref"]) == bool(ref["needs_ref"])
    if name == "coarse_pipe":  # tests/test_simple_coarse_pipe.cpp:36-49
        assert cases.rel_l2(got["p"], extra["foam_p"]) < 0.005
        assert cases.rel_l2(got["U"][0], extra["foam_U"][:, 0]) < 0.005
        assert cases.rel_l2(got["U"][1], extra["foam_U"][:, 1]) < 0.09
    if name == "duct_simple":  # tests/test_simple_duct_symmetry.cpp:38-53
        assert cases.rel_l2(got["p"], extra["foam_p"]) < 0.025
        assert cases.rel_l2(got["U"][0], extra["foam_U"][:, 0]) < 0.07
        assert cases.rel_l2(got["U"][1], extra["foam_U"][:, 1]) < 0.007


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
def test_cavity_simple_vs_oracle(gpu, orc, precision):
    out = {}
    for name, lib in (("gpu", gpu), ("orc", orc)):
        mesh, U, p, nu, mdot, eqs = cases.cavity(16, lib)
        solver = api.BiCGSTAB(precision=precision) if name == "gpu" else api.BiCGSTAB()
        simple = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=solver)
        for _ in range(10):
            reps = simple.step(eqs, U, mdot, p)
        out[name] = (U.values(), p.values(), mdot.face_flux(), reps)
    for i, k in enumerate(("U", "p", "mdot")):
        err = cases.rel_l2(out["gpu"][i], out["orc"][i])
        print(f"cavity 16x16 precision={precision} {k}: rel L2 vs oracle {err:.3e}")
        assert err < SOL_TOL
    assert [r.field_name for r in out["gpu"][3]] == [r.field_name for r in out["orc"][3]]


def test_piso_vs_oracle(gpu, orc):
    out = {}
    for name, lib in (("gpu", gpu), ("orc", orc)):
        mesh, U, p, nu, mdot, eqs = cases.cavity(12, lib, conv="LinearUpwind")
        piso = api.PISO(api.PISOControls(momentum_urf=0.7, pressure_urf=0.3))
        for _ in range(3):
            piso.step(eqs, U, mdot, p)
        out[name] = (U.values(), p.values())
    for i, k in enumerate(("U", "p")):
        err = cases.rel_l2(out["gpu"][i], out["orc"][i])
        print(f"PISO cavity {k}: rel L2 vs oracle {err:.3e}")
        assert err < SOL_TOL


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
def test_transport_linear_upwind_solve(gpu, orc, precision):
    # the nonsymmetric C3-type system (jittered hexes, LinearUpwind + Corrected)
    out = {}
    for name, lib in (("gpu", gpu), ("orc", orc)):
        mesh, T, U, eqn = cases.transport_c3(16, lib, conv="LinearUpwind")
        solver = api.BiCGSTAB(precision=precision, krylov_tol=1e-12) if name == "gpu" else api.BiCGSTAB()
        r = solver.solve(eqn, 1, 0.0)
        out[name] = (T.values(), r)
    err = cases.rel_l2(out["gpu"][0], out["orc"][0])
    print(f"transport 16^3 precision={precision}: rel L2 vs oracle {err:.3e}, "
          f"krylov it {out['gpu'][1].krylov_iterations}, status {out['gpu'][1].status}")
    assert err < SOL_TOL
