"""Full-size cases checked through size-independent properties.

At these sizes the CPU oracle would take hours, so the GPU is checked against
itself and against the physics:
  * the 512 x 512 x 1 lid-driven cavity (262,144 cells, Re = 100, Upwind +
    Corrected, urf 0.7 / 0.3) for 500 SIMPLE iterations, FP64 and mixed
    precision (FP32 BiCGSTAB with FP64 reliable updates): the two runs agree
    within the solution tolerance of the parity tests, the closed cavity's net
    face flux is zero and the continuity residual has fallen;
  * the 128^3 jittered-hex transport (2,097,152 cells) with the C3 recipe (MUSCL +
    Corrected + Green-Gauss), one step() from T = 0: FP64 and mixed precision agree
    and, where tests/golden/c3_128_solution.npy is present (the reference's own CPU
    solution of the same system, checksum-verified), both are within 1e-8 of it.
    (The recipe's later outer steps have rows with negative diagonals that only an
    exact LU solves; tests/test_gpu_assembly.py covers them at 10^3.)"""
import hashlib
import json
import os

import numpy as np
import pytest

from prism_b200 import _abi as A
from prism_b200 import api
from tests import cases

pytestmark = pytest.mark.gpu
SOL_TOL = 1e-8


def _cavity(gpu, precision, iters):
    mesh, U, p, nu, mdot, eqs = cases.cavity(512, gpu)
    simple = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=api.BiCGSTAB(precision=precision))
    div0 = None
    for k in range(iters):
        simple.step(eqs, U, mdot, p)
        if k == 9:
            div0 = np.abs(api.ops.div(mdot).values()).max()
    vol = mesh.export()["cell_volume"]
    d = api.ops.div(mdot).values()
    return U.values(), p.values(), d, vol, div0


def test_cavity_512_fp64_vs_mixed(gpu):
    runs = {prec: _cavity(gpu, prec, 500) for prec in (A.PREC_FP64, A.PREC_MIXED)}
    U64, p64, d64, vol, div10 = runs[A.PREC_FP64]
    U32, p32, _, _, _ = runs[A.PREC_MIXED]
    eu, ep = cases.rel_l2(U32, U64), cases.rel_l2(p32, p64)
    net = abs((d64 * vol).sum()) / (np.abs(d64) * vol).sum()
    print(f"cavity 512^2, 500 SIMPLE iterations: mixed vs FP64 rel L2 U {eu:.2e} p {ep:.2e}; "
          f"max |div| after 10 iterations {div10:.2e}, after 500 {np.abs(d64).max():.2e}; net flux {net:.1e}")
    assert eu < SOL_TOL and ep < SOL_TOL
    assert np.abs(d64).max() < 0.1 * div10
    assert net < 1e-9
    assert np.isfinite(U64).all() and np.abs(U64[0]).max() <= 1.0 + 1e-6  # lid speed bounds the flow


def _cpu_solution(n):
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    npy, js = os.path.join(here, f"c3_{n}_solution.npy"), os.path.join(here, f"c3_{n}_solution.json")
    if not (os.path.exists(npy) and os.path.exists(js)):
        return None
    x = np.load(npy)
    with open(js) as fh:
        ok = hashlib.sha256(np.ascontiguousarray(x, np.float64).tobytes()).hexdigest() == json.load(fh)["sha256"]
    return x if ok else None


def test_transport_128_fp64_vs_mixed(gpu):
    sol = {}
    for prec in (A.PREC_FP64, A.PREC_MIXED):
        mesh, T, U, eqn = cases.transport_c3(128, gpu, conv="MUSCL")
        r = api.BiCGSTAB(precision=prec, krylov_tol=1e-12).solve(eqn, 1, 0.0)
        assert r.status == A.OK
        sol[prec] = T.values()
    err = cases.rel_l2(sol[A.PREC_MIXED], sol[A.PREC_FP64])
    t = sol[A.PREC_FP64]
    print(f"transport 128^3 MUSCL, step 1: mixed vs FP64 rel L2 {err:.2e}; T in [{t.min():.3e}, {t.max():.3e}]")
    assert err < SOL_TOL
    assert np.isfinite(t).all()
    x = _cpu_solution(128)
    if x is not None:
        e64, e32 = cases.rel_l2(sol[A.PREC_FP64], x), cases.rel_l2(sol[A.PREC_MIXED], x)
        print(f"  against the reference's CPU solution: FP64 {e64:.2e}, mixed {e32:.2e}")
        assert e64 < SOL_TOL and e32 < SOL_TOL
