"""Discrete adjoint of steady diffusion on tets (transposed assembly + transposed
BiCGSTAB) against the CPU transpose-solve reference and central finite
differences of J through the GPU forward solve (1e-6 relative)."""
import numpy as np
import pytest

from prism_b200 import PrismError, api
from tests import cases
from tests.adjoint_reference import adjoint_gradients, steady_state

pytestmark = pytest.mark.gpu
SOLVER = api.BiCGSTAB(krylov_tol=1e-14, krylov_max_iter=100000)


def _gpu_state(gpu, n, corrected=True):
    c = cases.adjoint_c5(n, gpu, corrected=corrected)
    fw = api.adjoint_forward(c["eqn"], SOLVER, max_outer=500, outer_tol=1e-14)
    assert fw.converged and fw.status == 0
    return c, fw


@pytest.mark.parametrize("n,corrected", [(3, True), (4, True), (3, False)])
def test_adjoint_matches_cpu_transpose_solve(gpu, orc, n, corrected):
    c, fw = _gpu_state(gpu, n, corrected)
    phi = c["T"].values()
    J, dJ = cases.objective(phi, c["T_star"], c["vol"])
    gk, gv, bw = api.adjoint_backward(c["eqn"], dJ, SOLVER, max_outer=500, outer_tol=1e-14)
    assert bw.converged and bw.status == 0
    co = cases.adjoint_c5(n, orc, corrected=corrected)
    phi_o, _ = steady_state(co)
    assert np.linalg.norm(phi - phi_o) <= 1e-10 * np.linalg.norm(phi_o)
    rk, rv, _ = adjoint_gradients(co, phi_o, co["kappa0"], co["v0"], cases.objective(phi_o, co["T_star"],
                                                                                     co["vol"])[1])
    ek = np.abs(gk - rk).max() / np.abs(rk).max()
    ev = np.abs(gv - rv).max() / np.abs(rv).max()
    print(f"tets n={n} corrected={corrected}: forward outer {fw.outer_iterations}, adjoint outer "
          f"{bw.outer_iterations}; dJ/dkappa rel {ek:.2e}, dJ/dv rel {ev:.2e}")
    assert ek < 1e-8 and ev < 1e-8


def test_adjoint_finite_differences_32_directions(gpu):
    n = 8
    c, fw = _gpu_state(gpu, n)
    phi0 = c["T"].values()
    J0, dJ = cases.objective(phi0, c["T_star"], c["vol"])
    gk, gv, bw = api.adjoint_backward(c["eqn"], dJ, SOLVER, max_outer=500, outer_tol=1e-14)
    rng = np.random.default_rng(32)
    # fourth-order central differences: O(eps^4) truncation, while the forward
    # solves' ~1e-10 relative accuracy stays well below 1e-6 of the slope
    eps = 1e-3
    worst = 0.0
    for _ in range(32):
        dk = rng.normal(size=c["mesh"].n_cells)
        dv = rng.normal(size=len(c["v0"]))

        def J_at(s):
            c["kappa"].set_values(c["kappa0"] * (1 + s * eps * dk))
            fv = np.zeros(c["mesh"].n_faces)
            fv[: len(dv)] = c["v0"] + s * eps * dv
            c["T"].set_face_values(fv)
            c["T"].set_values(phi0)
            r = api.adjoint_forward(c["eqn"], SOLVER, max_outer=500, outer_tol=1e-14)
            assert r.converged
            return cases.objective(c["T"].values(), c["T_star"], c["vol"])[0]

        fd = (8 * (J_at(1) - J_at(-1)) - (J_at(2) - J_at(-2))) / (12 * eps)
        an = np.sum(gk * c["kappa0"] * dk) + np.sum(gv * dv)
        worst = max(worst, abs(fd - an) / abs(an))
    print(f"tets n={n} ({c['mesh'].n_cells} cells): 32 directions, worst rel error vs central FD {worst:.2e}")
    assert worst <= 1e-6


def test_adjoint_autograd_function(gpu):
    torch = pytest.importorskip("torch")
    from prism_b200.autograd import SteadyDiffusionProblem, steady_diffusion
    c = cases.adjoint_c5(3, gpu)
    prob = SteadyDiffusionProblem(c["eqn"], c["T"], c["kappa"], solver=SOLVER, outer_tol=1e-14, max_outer=500)
    k = torch.tensor(c["kappa0"], dtype=torch.float64, requires_grad=True)
    v = torch.tensor(c["v0"], dtype=torch.float64, requires_grad=True)
    T = steady_diffusion(k, v, prob)
    ts = torch.tensor(c["T_star"], dtype=torch.float64)
    vol = torch.tensor(c["vol"], dtype=torch.float64)
    J = (vol * (T - ts) ** 2).sum()
    J.backward()
    J2, dJ = cases.objective(T.detach().numpy(), c["T_star"], c["vol"])
    gk, gv, _ = api.adjoint_backward(c["eqn"], dJ, SOLVER, max_outer=500, outer_tol=1e-14)
    assert abs(J.item() - J2) <= 1e-12 * abs(J2)
    np.testing.assert_allclose(k.grad.numpy(), gk, rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(v.grad.numpy(), gv, rtol=1e-10, atol=1e-14)


def test_adjoint_rejects_convection(gpu):
    mesh, T, U, eqn = cases.transport_c3(4, gpu, conv="Upwind")
    with pytest.raises(PrismError):
        api.adjoint_backward(eqn, np.ones(mesh.n_cells))
