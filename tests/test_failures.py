"""Failure statuses on host-injected inputs (nothing here faults, traps or hangs a GPU).

The reference reports a failed solve only through SolverResult::hasConverged
(numerics/solver.h:8-23) and non-finite fields, and throws
error::NonImplementedBoundaryCondition for a patch whose kind has no handler
(boundary.h:109-114). The library returns the same converged flag plus a status:
NONFINITE (NaN in the system or the iterate), NOT_CONVERGED (Krylov cap),
BREAKDOWN (rho or omega collapsed past the restart budget) and NO_BC_HANDLER.
Each case is checked on the CPU oracle and the compiled reference (CPU tests)
and on the GPU path through prism_solve, prism_batch_solve and graph mode."""
import numpy as np
import pytest

from prism_b200 import PrismError, api, meshgen
from prism_b200 import _abi as A
from tests import cases

OK_OR_CAPPED = (A.NOT_CONVERGED, A.BREAKDOWN)  # statuses of a solve that cannot converge


def poisson(lib, n=16, bc="fixed", nan_at=None, kappa=1.0):
    """-div(kappa grad P) = S on an n x n x 1 box; bc "fixed" (P = 0 on the side walls) or
    "neumann" (zero-gradient everywhere, S with a non-zero mean: no solution)."""
    unv = meshgen.box_hex(n, n, 1, (1.0, 1.0, 1.0 / n))
    side = ("fixed", 0.0) if bc == "fixed" else ("zero-gradient", None)
    case = cases.box_case({"P": {"left": side, "right": side, "bottom": side, "top": side,
                                 "back": ("empty", None), "front": ("empty", None)}})
    mesh = api.Mesh(unv, case, lib=lib)
    cc = mesh.export()["cell_center"]
    s = 1.0 + np.sin(np.pi * cc[0]) * np.cos(np.pi * cc[1])
    if nan_at is not None:
        s[nan_at] = np.nan
    P = api.Scalar("P", mesh, 0.0)
    S = api.Scalar("S", mesh, s)
    k = api.Scalar("kappa", mesh, kappa)
    eqn = api.Transport(api.diffusion.NonCorrected(k, P), api.source.ConstantScalar(S))
    return mesh, P, S, eqn


def no_handler_case(lib):
    unv = meshgen.box_hex(4, 4, 4)
    case = cases.box_case({"T": {"left": ("inlet", 1.0)}})
    mesh = api.Mesh(unv, case, lib=lib)
    T = api.Scalar("T", mesh, 0.0)
    eqn = api.Transport(api.diffusion.NonCorrected(api.Scalar("kappa", mesh, 1.0), T))
    return unv, case, mesh, T, eqn


# ---------------------------------------------------------------- oracle and reference (CPU)
def test_oracle_nan_rhs_not_converged(orc, ref):
    # Eigen's BiCGSTAB loop test ||r||^2 > tol^2 ||b||^2 is false when b holds a NaN: no
    # iteration runs, the field keeps its values and the solve reports not converged
    mesh, P, S, eqn = poisson(orc, nan_at=37)
    r = api.BiCGSTAB().solve(eqn, 2, 1e-10)
    assert not r.converged and r.krylov_iterations == 0
    np.testing.assert_array_equal(P.values(), 0.0)
    unv = meshgen.box_hex(16, 16, 1, (1.0, 1.0, 1.0 / 16))
    case = cases.box_case({"T": {k: ("fixed", 0.0) for k in ("left", "right", "bottom", "top")} |
                           {"back": ("empty", None), "front": ("empty", None)}})
    T = ref.transport(ref.Mesh(unv, case), kappa=1.0, corrected=False, src=S.values(), n_iter=2)
    np.testing.assert_array_equal(T, 0.0)


def test_oracle_zero_diagonal_jacobi(orc, ref):
    # Jacobi on A = 0 (kappa = 0): D^-1 = inf, the iterate is not finite in the reference too
    mesh, P, S, eqn = poisson(orc, kappa=0.0)
    api.Jacobi().solve(eqn, 2, 1e-10)
    assert not np.isfinite(P.values()).all()
    unv = meshgen.box_hex(16, 16, 1, (1.0, 1.0, 1.0 / 16))
    case = cases.box_case({"T": {k: ("fixed", 0.0) for k in ("left", "right", "bottom", "top")} |
                           {"back": ("empty", None), "front": ("empty", None)}})
    T = ref.transport(ref.Mesh(unv, case), kappa=0.0, corrected=False, src=S.values(), n_iter=2, method="jacobi")
    np.testing.assert_array_equal(T, P.values())


def test_oracle_all_neumann_without_reference_cell(orc, ref):
    # no solution exists (zero-gradient everywhere, source with a non-zero mean): the
    # reference's solve drifts to a huge field whose scaled residual max|Ax - b| /
    # max|diag x| is small, so it reports convergence; the oracle does the same bit for bit
    mesh, P, S, eqn = poisson(orc, n=8, bc="neumann")
    r = api.BiCGSTAB().solve(eqn, 1, 1e-10)
    assert np.abs(P.values()).max() > 1e10 and r.converged
    unv = meshgen.box_hex(8, 8, 1, (1.0, 1.0, 1.0 / 8))
    case = cases.box_case({"T": {"back": ("empty", None), "front": ("empty", None)}})
    T = ref.transport(ref.Mesh(unv, case), kappa=1.0, corrected=False, src=S.values(), n_iter=1)
    np.testing.assert_array_equal(T, P.values())


def test_missing_handler_oracle_and_reference(orc, ref):
    unv, case, mesh, T, eqn = no_handler_case(orc)
    with pytest.raises(PrismError) as e:
        api.BiCGSTAB().solve(eqn, 1, 1e-10)
    assert e.value.status == A.NO_BC_HANDLER
    with pytest.raises(RuntimeError, match="Non-implemented boundary condition"):
        ref.transport(ref.Mesh(unv, case), kappa=1.0, corrected=False)


# ---------------------------------------------------------------- GPU path
@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
def test_gpu_nan_rhs_nonfinite(gpu, orc, graph):
    mesh, P, S, eqn = poisson(gpu)
    solver = api.BiCGSTAB(graph=graph)
    good = solver.solve(eqn, 2, 1e-10)  # builds what graph mode replays
    assert good.status == A.OK and good.converged
    s = S.values()
    s[37] = np.nan
    S.set_values(s)
    P.set_values(np.zeros(mesh.n_cells))
    r = solver.solve(eqn, 2, 1e-10)
    assert r.status == A.NONFINITE and not r.converged
    o = api.BiCGSTAB().solve(poisson(orc, nan_at=37)[3], 2, 1e-10)
    assert r.converged == o.converged


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
def test_gpu_krylov_cap_not_converged(gpu, graph):
    mesh, P, S, eqn = poisson(gpu, n=32)
    capped = api.BiCGSTAB(krylov_max_iter=1, preconditioner="jacobi", graph=graph)
    api.BiCGSTAB(preconditioner="jacobi", graph=graph).solve(eqn, 1, 1e-10)  # warm (graph build)
    P.set_values(np.zeros(mesh.n_cells))
    r = capped.solve(eqn, 1, 1e-10)
    assert r.status == A.NOT_CONVERGED and not r.converged and r.krylov_iterations <= 1


@pytest.mark.gpu
def test_gpu_zero_diagonal_jacobi_nonfinite(gpu, orc):
    mesh, P, S, eqn = poisson(gpu, kappa=0.0)
    r = api.Jacobi().solve(eqn, 2, 1e-10)
    assert r.status == A.NONFINITE and not r.converged
    assert not np.isfinite(P.values()).all()


@pytest.mark.gpu
@pytest.mark.parametrize("pc", ["jacobi", "amg"])
def test_gpu_all_neumann_without_reference_cell(gpu, pc):
    mesh, P, S, eqn = poisson(gpu, n=8, bc="neumann")
    # the Krylov solve cannot reach its tolerance on a system without a solution: it stops at
    # the iteration cap or on a breakdown, and says so (the reference has no such status)
    r = api.BiCGSTAB(preconditioner=pc, krylov_max_iter=400).solve(eqn, 1, 1e-10)
    assert r.status in OK_OR_CAPPED + (A.NONFINITE,)


@pytest.mark.gpu
def test_gpu_missing_handler(gpu):
    unv, case, mesh, T, eqn = no_handler_case(gpu)
    with pytest.raises(PrismError) as e:
        api.BiCGSTAB().solve(eqn, 1, 1e-10)
    assert e.value.status == A.NO_BC_HANDLER


@pytest.mark.gpu
def test_gpu_batch_statuses(gpu):
    # one persistent launch over three systems: a good one, one with NaN in b, a good one
    probs = [poisson(gpu, n=12), poisson(gpu, n=12, nan_at=20), poisson(gpu, n=16)]
    bs = api.BatchSolver(api.BiCGSTAB(precision=A.PREC_MIXED, krylov_tol=1e-10), lib=gpu)
    res = bs.solve([p[3] for p in probs])
    assert res[0].status == A.OK and res[2].status == A.OK
    assert res[1].status == A.NONFINITE
    capped = api.BatchSolver(api.BiCGSTAB(precision=A.PREC_MIXED, krylov_tol=1e-10, krylov_max_iter=1), lib=gpu)
    for p in probs:
        p[1].set_values(np.zeros(p[0].n_cells))
    res = capped.solve([probs[0][3], probs[2][3]])
    assert all(r.status == A.NOT_CONVERGED for r in res)


# ---------------------------------------------------------------- flexible CG (PRISM_SOLVER_FCG)
@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
def test_gpu_fcg_statuses(gpu, graph):
    """Flexible CG reports the same statuses as BiCGSTAB: NONFINITE for NaN in b,
    NOT_CONVERGED at the Krylov cap, and BAD_ARG for what it cannot run."""
    mesh, P, S, eqn = poisson(gpu, n=32)
    solver = api.FCG(graph=graph)
    good = solver.solve(eqn, 2, 1e-10)  # builds what graph mode replays
    assert good.status == A.OK and good.converged
    P.set_values(np.zeros(mesh.n_cells))
    r = api.FCG(krylov_max_iter=1, graph=graph).solve(eqn, 1, 1e-10)
    assert r.status == A.NOT_CONVERGED and not r.converged and r.krylov_iterations <= 1
    s = S.values()
    s[37] = np.nan
    S.set_values(s)
    P.set_values(np.zeros(mesh.n_cells))
    r = solver.solve(eqn, 2, 1e-10)
    assert r.status == A.NONFINITE and not r.converged
    for bad in (api.FCG(precision=A.PREC_MIXED), api.FCG(preconditioner="jacobi")):
        with pytest.raises(PrismError) as e:
            bad.solve(eqn, 1, 1e-10)
        assert e.value.status == A.BAD_ARG
