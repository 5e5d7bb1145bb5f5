"""Transient path on the GPU vs the oracle: field history, the BackwardEuler and
AdamMoulton temporal schemes (assembly bit for bit, in any registration order),
the reference's transient 1-D test and a transient PISO run."""
import numpy as np
import pytest

from prism_b200 import _abi as A
from prism_b200 import PrismError, api
from tests import cases
from tests.test_gpu_assembly import check
from tests.test_oracle_pins import _history_sections

pytestmark = pytest.mark.gpu
SOL_TOL = 1e-8


def test_scalar_history(gpu):
    _history_sections(gpu)


@pytest.mark.parametrize("kind", ["BackwardEuler", "AdamMoulton"])
@pytest.mark.parametrize("steps", [1, 2, 3])
@pytest.mark.parametrize("first", [True, False])
def test_temporal_assembly(gpu, orc, kind, steps, first):
    # LinearUpwind + Corrected + temporal on a jittered box; `steps` history entries
    # (AdamMoulton is first order with one), the temporal scheme first or last
    def build(lib):
        mesh, T, U, _ = cases.transport_c3(6, lib, conv="LinearUpwind")
        cc = mesh.export()["cell_center"]
        T.set_history_size(2)
        for k in range(steps):
            T.update(np.sin(3 * cc[0] + k) + cc[1] ** 2 - 0.5 * cc[2] * k)
        kap = api.Scalar("kappa", mesh, 1e-3)
        tm = getattr(api.temporal, kind)(T, 0.37)
        sch = [api.convection.LinearUpwind(U, T), api.diffusion.Corrected(kap, T)]
        eqn = api.Transport(*([tm] + sch if first else sch + [tm]))
        return mesh, T, U, kap, eqn
    Ag, bg, Ao, bo = check(build, gpu, orc)
    np.testing.assert_array_equal(Ag, Ao)
    np.testing.assert_array_equal(bg, bo)


def test_transient_1d_reference_case(gpu):
    ref = cases.load_oracle_results("versteeg_trans_1d")
    got = cases.run_reference_test("versteeg_trans_1d", gpu)
    err = cases.rel_l2(got["T"], ref["T"])
    print(f"transient 1-D (AdamMoulton, 200 steps): rel L2 vs oracle {err:.3e}, errors vs series "
          f"{got['diff_norms']} final {got['final_diff_norm']:.4f}")
    assert err < SOL_TOL
    n40, n60 = got["diff_norms"]
    assert n40 < 0.10 and n60 < 0.10 and n60 < n40      # tests/test_transient_1d.cpp:76-80
    assert got["final_diff_norm"] < 0.02


def _piso_cavity(lib, steps=20):
    # tests/test_algorithms_pipe.cpp:43-82: BackwardEuler momentum, PISO, cavity_hex
    unv, case, _ = cases.load_golden("cavity_hex")
    mesh = api.Mesh(unv, case, lib=lib)
    U, p, nu, mdot = cases.simple_fields(mesh, 0.01)
    dt = 0.005
    for c in (U.x(), U.y()):
        c.set_history_size(2)
        c.update_prev_time_steps()
    eqs = [api.Transport(api.temporal.BackwardEuler(c, dt), api.convection.LinearUpwind(mdot, c),
                         api.diffusion.Corrected(nu, c), api.source.Gradient(p, k, A.SIGN_NEGATIVE))
           for k, c in enumerate((U.x(), U.y()))]
    ctl = api.PISOControls(outer_iterations=3, pressure_correction_steps=1, non_ortho_correctors=0)
    piso = api.PISO(ctl)
    for _ in range(steps):
        piso.step(eqs, U, mdot, p)
        U.x().update_prev_time_steps()
        U.y().update_prev_time_steps()
    return U.values(), p.values()


def test_transient_piso_cavity(gpu, orc):
    Ug, pg = _piso_cavity(gpu)
    Uo, po = _piso_cavity(orc)
    assert np.all(np.isfinite(pg))
    for a, b, k in ((Ug, Uo, "U"), (pg, po, "p")):
        err = cases.rel_l2(a, b)
        print(f"transient PISO cavity_hex {k}: rel L2 vs oracle {err:.3e}")
        assert err < SOL_TOL


def test_temporal_errors(gpu):
    mesh, T, U, _ = cases.transport_c3(4, gpu, conv="Upwind")
    kap = api.Scalar("kappa", mesh, 1e-3)
    eqn = api.Transport(api.temporal.BackwardEuler(T, 0.1), api.diffusion.Corrected(kap, T))
    with pytest.raises(PrismError):  # no history stored (backward_euler.cpp:68-74)
        eqn.update_coeffs()
    with pytest.raises(PrismError):
        eqn.set_time_step(0.0)
    with pytest.raises(ValueError):
        api.temporal.AdamMoulton(T, -1.0)
    with pytest.raises(PrismError):  # at most one temporal scheme
        api.Transport(api.temporal.BackwardEuler(T, 0.1), api.temporal.AdamMoulton(T, 0.1))
