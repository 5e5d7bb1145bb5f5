"""The pressure-velocity algorithms of the oracle pinned on the reference's
tests/test_algorithms_pipe.cpp: SIMPLE, PISO without and with PRIME correctors
conserve mass through the coarse pipe and the open duct (|inlet + outlet| /
|inlet| < 1e-6), and PISO with backward-Euler momentum keeps the closed cavity's
pressure finite with the automatic reference cell. The GPU path runs these
drivers within 1e-8..1e-11 of the oracle (tests/test_gpu_solve.py)."""
import numpy as np
import pytest

from prism_b200 import _abi as A
from prism_b200 import api
from tests import cases


def _imbalance(mesh, case, U, inlet, outlet):
    # flowRate (tests/test_utils.h): sum of U's face fluxes over a patch
    flux = U.face_flux()
    ex = mesh.export()
    pfo, pf = ex["patch_face_offsets"], ex["patch_faces"]
    rate = {n: float(flux[pf[pfo[i]:pfo[i + 1]]].sum()) for i, n in enumerate(case.patch_names)}
    return abs(rate[inlet] + rate[outlet]) / abs(rate[inlet])


def _pipe(orc, name="coarse_pipe", symmetry=False):
    unv, case, _ = cases.load_golden(name)
    mesh = api.Mesh(unv, case, lib=orc)
    U, p, nu, mdot = cases.simple_fields(mesh)
    eqs = cases.momentum_eqns(U, p, nu, mdot, symmetry=symmetry)
    return mesh, case, U, p, mdot, eqs


def test_simple_coarse_pipe_200(orc):
    # test_algorithms_pipe.cpp:14-40
    mesh, case, U, p, mdot, eqs = _pipe(orc)
    simple = api.IncompressibleSIMPLE(api.SIMPLEControls())
    for _ in range(200):
        simple.step(eqs, U, mdot, p)
    imb = _imbalance(mesh, case, U, "Inlet", "Outlet")
    print(f"SIMPLE coarse pipe, 200 iterations: imbalance {imb:.2e}")
    assert imb < 1e-6


def test_simple_duct_500(orc):
    # test_algorithms_pipe.cpp:85-113 (momentum symmetry handlers, open domain)
    mesh, case, U, p, mdot, eqs = _pipe(orc, "duct_simple", symmetry=True)
    simple = api.IncompressibleSIMPLE(api.SIMPLEControls())
    for _ in range(500):
        simple.step(eqs, U, mdot, p)
    assert not api.needs_pressure_reference(p)
    imb = _imbalance(mesh, case, U, "inlet", "outlet")
    print(f"SIMPLE duct, 500 iterations: imbalance {imb:.2e}")
    assert imb < 1e-6


@pytest.mark.parametrize("pressure_correction_steps, steps", [(1, 200), (2, 50)])
def test_piso_coarse_pipe(orc, pressure_correction_steps, steps):
    # test_algorithms_pipe.cpp:115-150 (PISO without PRIME) and :152-187 (with PRIME)
    mesh, case, U, p, mdot, eqs = _pipe(orc)
    piso = api.PISO(api.PISOControls(outer_iterations=1, momentum_implicit_steps=1,
                                     pressure_correction_steps=pressure_correction_steps, non_ortho_correctors=2,
                                     momentum_urf=0.7, pressure_urf=0.3, momentum_residual=1e-7,
                                     pressure_residual=1e-7))
    for _ in range(steps):
        piso.step(eqs, U, mdot, p)
    imb = _imbalance(mesh, case, U, "Inlet", "Outlet")
    print(f"PISO coarse pipe, {pressure_correction_steps} pressure corrections x {steps} steps: "
          f"imbalance {imb:.2e}")
    assert imb < 1e-6


def test_piso_cavity_auto_reference(orc):
    # test_algorithms_pipe.cpp:42-83: backward-Euler momentum, closed cavity, automatic p_ref
    unv, case, _ = cases.load_golden("cavity_hex")
    mesh = api.Mesh(unv, case, lib=orc)
    U, p, nu, mdot = cases.simple_fields(mesh, 0.01)
    comps = [U.x(), U.y()]
    for c in comps:
        c.set_history_size(2)
        c.update_prev_time_steps()
    eqs = [api.Transport(api.temporal.BackwardEuler(c, 0.005), api.convection.LinearUpwind(mdot, c),
                         api.diffusion.Corrected(nu, c), api.source.Gradient(p, k, A.SIGN_NEGATIVE))
           for k, c in enumerate(comps)]
    piso = api.PISO(api.PISOControls(outer_iterations=3, pressure_correction_steps=1, non_ortho_correctors=0))
    for _ in range(20):
        piso.step(eqs, U, mdot, p)
        for c in comps:
            c.update_prev_time_steps()
    assert api.needs_pressure_reference(p)
    pv = p.values()
    print(f"PISO cavity, 20 steps: max |p| {np.abs(pv).max():.3e}")
    assert np.all(np.isfinite(pv))
