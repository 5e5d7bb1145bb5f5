"""Batched solves (one persistent launch for many independent systems) against
the oracle's solves of the same equations, one by one."""
import numpy as np
import pytest

from prism_b200 import _abi as A
from prism_b200 import PrismError, api
from tests import cases

pytestmark = pytest.mark.gpu
SOL_TOL = 1e-8


@pytest.mark.parametrize("precision", [A.PREC_MIXED, A.PREC_FP64])
def test_batch_matches_oracle(gpu, orc, precision):
    sizes = cases.batch_sizes(10, seed=4, nmin=3, nmax=14)
    probs = [cases.diffusion_box(N, gpu, seed=100 + i) for i, N in enumerate(sizes)]
    bs = api.BatchSolver(api.BiCGSTAB(precision=precision, krylov_tol=1e-12), lib=gpu)
    res = bs.solve([p["eqn"] for p in probs])
    worst = 0.0
    for i, (N, p, r) in enumerate(zip(sizes, probs, res)):
        q = cases.diffusion_box(N, orc, seed=100 + i)
        api.BiCGSTAB().solve(q["eqn"], 1, 0.0)
        err = cases.rel_l2(p["T"].values(), q["T"].values())
        worst = max(worst, err)
        assert r.status == A.OK, (N, r)
        assert r.krylov_rel_residual <= 1e-12
    print(f"batch of {len(sizes)} (N = {sizes}) precision={precision}: worst rel L2 vs oracle {worst:.2e}, "
          f"iterations {[r.krylov_iterations for r in res]}")
    assert worst < SOL_TOL


def test_batch_repeated_and_matches_single_solves(gpu):
    sizes = [5, 9, 4, 12, 7]
    probs = [cases.diffusion_box(N, gpu, seed=7 + i) for i, N in enumerate(sizes)]
    bs = api.BatchSolver(api.BiCGSTAB(precision=A.PREC_MIXED, krylov_tol=1e-12), lib=gpu)
    for rep in range(2):  # the second call reuses the plan and the tuned shape
        for p in probs:
            p["T"].set_values(np.zeros(p["mesh"].n_cells))
        res = bs.solve([p["eqn"] for p in probs])
        assert all(r.status == A.OK for r in res)
    single = [cases.diffusion_box(N, gpu, seed=7 + i) for i, N in enumerate(sizes)]
    for p, q in zip(probs, single):
        api.BiCGSTAB(krylov_tol=1e-12).solve(q["eqn"], 1, 0.0)
        assert cases.rel_l2(p["T"].values(), q["T"].values()) < SOL_TOL


def test_batch_zero_rhs_and_bad_args(gpu):
    # f = 0 and T = 0 with T = 0 on the walls: b = 0 exactly (no correction term either)
    p = cases.diffusion_box(4, gpu, seed=1)
    p["f"].set_values(np.zeros(p["mesh"].n_cells))
    q = cases.diffusion_box(6, gpu, seed=2)
    bs = api.BatchSolver(api.BiCGSTAB(precision=A.PREC_MIXED), lib=gpu)
    res = bs.solve([p["eqn"], q["eqn"]])
    assert res[0].status == A.OK and np.all(p["T"].values() == 0.0)
    assert res[1].status == A.OK
    with pytest.raises(PrismError):
        api.BatchSolver(api.Jacobi(), lib=gpu).solve([q["eqn"]])


def test_batch_call_is_one_graph_launch(gpu):
    # each call (gather, set-up, the persistent solve, scatter) is one CUDA graph launch,
    # captured on the first call and replayed while the systems' buffers stay the same
    import ctypes
    sizes = [6, 11, 4, 9]
    probs = [cases.diffusion_box(N, gpu, seed=40 + i) for i, N in enumerate(sizes)]
    bs = api.BatchSolver(api.BiCGSTAB(precision=A.PREC_MIXED, krylov_tol=1e-12), lib=gpu)
    sols = []
    gpu.check(gpu.profile_start(16))
    for _ in range(3):
        for p in probs:
            p["T"].set_values(np.zeros(p["mesh"].n_cells))
        res = bs.solve([p["eqn"] for p in probs])
        assert all(r.status == A.OK for r in res)
        sols.append(np.concatenate([p["T"].values() for p in probs]))
    prof = A.Profile()
    gpu.check(gpu.profile_stop(ctypes.byref(prof)))
    assert prof.graph_launches == 3
    np.testing.assert_array_equal(sols[1], sols[0])
    np.testing.assert_array_equal(sols[2], sols[0])


@pytest.mark.parametrize("algo", ["simple", "piso"])
def test_batched_momentum_steps(gpu, orc, algo):
    # the momentum components of each step solved together in one persistent launch:
    # the fields still match the oracle's (one solve per component)
    out = {}
    for name, lib in (("gpu", gpu), ("orc", orc)):
        mesh, U, p, nu, mdot, eqs = cases.cavity(24, lib)
        solver = api.BiCGSTAB(krylov_tol=1e-12) if name == "gpu" else api.BiCGSTAB()
        if algo == "simple":
            driver = api.IncompressibleSIMPLE(api.SIMPLEControls(batched_momentum=True), solver=solver)
        else:
            driver = api.PISO(api.PISOControls(momentum_urf=0.7, pressure_urf=0.3, batched_momentum=True),
                              solver=solver)
        for _ in range(6):
            reports = driver.step(eqs, U, mdot, p)
        out[name] = (U.values(), p.values(), reports)
    for i, k in enumerate(("U", "p")):
        err = cases.rel_l2(out["gpu"][i], out["orc"][i])
        print(f"{algo} with batched momentum, cavity 24^2 {k}: rel L2 vs oracle {err:.2e}")
        assert err < SOL_TOL
    assert [r.field_name for r in out["gpu"][2]] == [r.field_name for r in out["orc"][2]]
