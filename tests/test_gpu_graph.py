"""Solves and SIMPLE / PRIME / PISO steps run as one CUDA graph launch.

With PrismSolveOpts.graph the solver's loops (Krylov batches, restarts,
accurate-residual passes, the outer steps of ISolver::solve) run as
device-side conditional graph nodes over the same kernels, in the same order,
as the ordinary path. So a run in graph mode must reproduce the ordinary run
bit for bit: fields, face fluxes and every reported count and residual. The
first call on new equations runs the ordinary way (it builds the hierarchies
and buffers the graph uses), so each comparison covers ordinary and graph
calls in sequence."""
import numpy as np
import pytest

from prism_b200 import _abi as A
from prism_b200 import api
from tests import cases

pytestmark = pytest.mark.gpu


def _graph_launches(lib, f):
    """Runs f with the profiling window open; returns the number of graph launches in it."""
    import ctypes
    lib.check(lib.profile_start(16))
    try:
        f()
    finally:
        prof = A.Profile()
        lib.check(lib.profile_stop(ctypes.byref(prof)))
    return prof.graph_launches


def _same_results(a, b):
    assert (a.iteration, a.converged, a.status, a.krylov_iterations) == \
        (b.iteration, b.converged, b.status, b.krylov_iterations)
    assert np.array_equal([a.initial_residual, a.final_residual, a.krylov_rel_residual],
                          [b.initial_residual, b.final_residual, b.krylov_rel_residual], equal_nan=True)


@pytest.mark.parametrize("preconditioner", ["amg", "jacobi"])
@pytest.mark.parametrize("n_iter, eps", [(1, 0.0), (3, 1e-30)])
def test_solve_graph_matches_ordinary(gpu, preconditioner, n_iter, eps):
    out = {}
    for graph in (False, True):
        mesh, T, U, eqn = cases.transport_c3(20, gpu, conv="LinearUpwind")
        solver = api.BiCGSTAB(krylov_tol=1e-11, preconditioner=preconditioner, graph=graph)
        res = []
        launches = _graph_launches(gpu, lambda: res.extend(solver.solve(eqn, n_iter, eps) for _ in range(3)))
        assert launches == (2 if graph else 0)  # the first call builds what the graph uses
        out[graph] = (T.values(), res)
    np.testing.assert_array_equal(out[True][0], out[False][0])
    for a, b in zip(out[True][1], out[False][1]):
        _same_results(a, b)
    print(f"{preconditioner} n_iter={n_iter}: krylov its {[r.krylov_iterations for r in out[True][1]]}, "
          f"outer {[r.iteration for r in out[True][1]]}")


@pytest.mark.parametrize("n_iter, eps", [(1, 0.0), (3, 1e-30)])
def test_fcg_solve_graph_matches_ordinary(gpu, n_iter, eps):
    """Flexible CG (PRISM_SOLVER_FCG) in graph mode, bit for bit against the ordinary path."""
    out = {}
    for graph in (False, True):
        mesh, P, eqn, exact = cases.poisson_c1(64, gpu)
        solver = api.FCG(krylov_tol=1e-11, graph=graph)
        res = []

        def from_zero():  # every solve starts from P = 0, so each one iterates
            P.set_values(np.zeros(mesh.n_cells))
            return solver.solve(eqn, n_iter, eps)
        launches = _graph_launches(gpu, lambda: res.extend(from_zero() for _ in range(3)))
        assert launches == (2 if graph else 0)
        out[graph] = (P.values(), res)
    np.testing.assert_array_equal(out[True][0], out[False][0])
    for a, b in zip(out[True][1], out[False][1]):
        _same_results(a, b)
    print(f"flexible CG n_iter={n_iter}: krylov its {[r.krylov_iterations for r in out[True][1]]}")


def test_mixed_precision_runs_ordinarily(gpu):
    out = {}
    for graph in (False, True):
        mesh, T, U, eqn = cases.transport_c3(16, gpu, conv="LinearUpwind")
        solver = api.BiCGSTAB(precision=A.PREC_MIXED, krylov_tol=1e-11, graph=graph)
        r = []
        assert _graph_launches(gpu, lambda: r.extend(solver.solve(eqn, 1, 0.0) for _ in range(2))) == 0
        out[graph] = (T.values(), r)
    np.testing.assert_array_equal(out[True][0], out[False][0])


@pytest.mark.parametrize("algo", ["simple", "prime", "piso"])
@pytest.mark.parametrize("preconditioner", ["amg", "jacobi"])
def test_step_graph_matches_ordinary(gpu, algo, preconditioner):
    out = {}
    for graph in (False, True):
        mesh, U, p, nu, mdot, eqs = cases.cavity(20, gpu, conv="LinearUpwind")
        solver = api.BiCGSTAB(preconditioner=preconditioner, graph=graph)
        if algo == "simple":
            driver = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=solver)
        elif algo == "prime":
            driver = api.PRIME(api.SIMPLEControls(), solver=solver)
        else:
            driver = api.PISO(api.PISOControls(momentum_urf=0.7, pressure_urf=0.3), solver=solver)
        reports = []
        launches = _graph_launches(gpu, lambda: reports.extend(driver.step(eqs, U, mdot, p) for _ in range(5)))
        assert launches == (4 if graph else 0)
        out[graph] = (U.values(), p.values(), mdot.face_flux(), reports)
    for i, k in enumerate(("U", "p", "mdot")):
        np.testing.assert_array_equal(out[True][i], out[False][i], err_msg=k)
    for rg, ro in zip(out[True][3], out[False][3]):
        assert [(e.field_name, e.n_iterations, e.converged) for e in rg] == \
            [(e.field_name, e.n_iterations, e.converged) for e in ro]
        assert np.array_equal([(e.initial_residual, e.final_residual) for e in rg],
                              [(e.initial_residual, e.final_residual) for e in ro])
    print(f"{algo} ({preconditioner}): last step reports {[(e.field_name, e.n_iterations) for e in out[True][3][-1]]}")


@pytest.mark.parametrize("kcycle", [None, "1"])
def test_simple_graph_at_amg_sizes(gpu, kcycle, monkeypatch):
    """SIMPLE steps of a 192 x 192 cavity (36,864 cells: the automatic preconditioner
    measures the momentum matrices and keeps Jacobi, the pressure correction runs
    flexible CG with the FP32 V-cycle, or with a K-cycle level) as one graph launch
    each, bit for bit against the ordinary path."""
    if kcycle:
        monkeypatch.setenv("PRISM_AMG_KCYCLE", kcycle)
    out = {}
    for graph in (False, True):
        mesh, U, p, nu, mdot, eqs = cases.cavity(192, gpu)
        driver = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=api.BiCGSTAB(graph=graph))
        reports = []
        launches = _graph_launches(gpu, lambda: reports.extend(driver.step(eqs, U, mdot, p) for _ in range(4)))
        assert launches == (3 if graph else 0)
        out[graph] = (U.values(), p.values(), mdot.face_flux(), reports)
    for i, k in enumerate(("U", "p", "mdot")):
        np.testing.assert_array_equal(out[True][i], out[False][i], err_msg=k)
    for rg, ro in zip(out[True][3], out[False][3]):
        assert np.array_equal([(e.initial_residual, e.final_residual) for e in rg],
                              [(e.initial_residual, e.final_residual) for e in ro])
