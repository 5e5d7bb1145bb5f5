"""The configurations at the sizes the workload definitions state, where the CPU
oracle finishes in seconds, compared with the oracle (not with the GPU itself):

* C1: the 128 x 128 x 1 Poisson problem (16,384 cells), NonCorrected, BiCGSTAB;
* C2: the lid-driven cavity SIMPLE recipe (Re 100, Upwind + Corrected, urf 0.7/0.3)
  for 100 outer iterations on 64 x 64 x 1 hexes;
* C4: a batch of systems of N^3 = 32^3 .. 40^3 hexes (kappa ~ lognormal(0, 1),
  f ~ N(0, 1), Fixed 0) in one persistent launch, mixed precision.

Solved fields must agree with the oracle within 1e-8 relative L2 (printed)."""
import numpy as np
import pytest

from prism_b200 import _abi as A
from prism_b200 import api
from tests import cases

pytestmark = pytest.mark.gpu
SOL_TOL = 1e-8


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
def test_c1_128(gpu, orc, precision):
    out = {}
    for name, lib, solver in (("gpu", gpu, api.BiCGSTAB(precision=precision, krylov_tol=1e-12)),
                              ("orc", orc, api.BiCGSTAB())):
        mesh, P, eqn, exact = cases.poisson_c1(128, lib)
        r = solver.solve(eqn, 3, 1e-10)
        out[name] = (P.values(), r, cases.rel_l2(P.values(), exact))
    err = cases.rel_l2(out["gpu"][0], out["orc"][0])
    print(f"C1 128x128 precision={precision}: rel L2 vs oracle {err:.3e}, vs exact {out['gpu'][2]:.4e} "
          f"(oracle {out['orc'][2]:.4e}), krylov it {out['gpu'][1].krylov_iterations}")
    assert err < SOL_TOL
    assert out["gpu"][1].converged == out["orc"][1].converged


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
def test_c2_cavity_64_100_iterations(gpu, orc, precision):
    out = {}
    for name, lib in (("gpu", gpu), ("orc", orc)):
        mesh, U, p, nu, mdot, eqs = cases.cavity(64, lib)
        solver = api.BiCGSTAB(precision=precision) if name == "gpu" else api.BiCGSTAB()
        simple = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=solver)
        for _ in range(100):
            simple.step(eqs, U, mdot, p)
        out[name] = (U.values(), p.values(), mdot.face_flux())
    for i, k in enumerate(("U", "p", "mdot")):
        err = cases.rel_l2(out["gpu"][i], out["orc"][i])
        print(f"C2 cavity 64x64 x 100 SIMPLE precision={precision} {k}: rel L2 vs oracle {err:.3e}")
        assert err < SOL_TOL


def test_c4_batch_32_to_40(gpu, orc):
    sizes = [32, 40, 36]
    probs = [cases.diffusion_box(N, gpu, seed=400 + i) for i, N in enumerate(sizes)]
    bs = api.BatchSolver(api.BiCGSTAB(precision=A.PREC_MIXED, krylov_tol=1e-12), lib=gpu)
    res = bs.solve([p["eqn"] for p in probs])
    worst = 0.0
    for i, (N, p, r) in enumerate(zip(sizes, probs, res)):
        assert r.status == A.OK, (N, r)
        q = cases.diffusion_box(N, orc, seed=400 + i)
        api.BiCGSTAB().solve(q["eqn"], 1, 0.0)
        err = cases.rel_l2(p["T"].values(), q["T"].values())
        print(f"C4 N={N}: rel L2 vs oracle {err:.3e}, iterations {r.krylov_iterations}")
        worst = max(worst, err)
    assert worst < SOL_TOL
