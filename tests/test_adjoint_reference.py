"""The CPU adjoint reference (dense transpose solve on the oracle's probed
Jacobians) against central finite differences of J through the oracle's own
steady forward solve: this pins the reference the GPU adjoint is checked with."""
import numpy as np
import pytest

from tests import cases
from tests.adjoint_reference import adjoint_gradients, steady_state


@pytest.mark.parametrize("n", [2, 3])
def test_cpu_adjoint_matches_finite_differences(orc, n):
    c = cases.adjoint_c5(n, orc)
    phi, outer = steady_state(c)
    assert outer < 500
    J, dJ = cases.objective(phi, c["T_star"], c["vol"])
    gk, gv, _ = adjoint_gradients(c, phi, c["kappa0"], c["v0"], dJ)
    rng = np.random.default_rng(11)
    eps = 1e-5
    for _ in range(4):
        dk = rng.normal(size=c["mesh"].n_cells)
        dv = rng.normal(size=len(c["v0"]))

        def J_at(s):
            c["kappa"].set_values(c["kappa0"] * (1 + s * eps * dk))
            fv = np.zeros(c["mesh"].n_faces)
            fv[: len(dv)] = c["v0"] + s * eps * dv
            c["T"].set_face_values(fv)
            c["T"].set_values(phi)
            return cases.objective(steady_state(c)[0], c["T_star"], c["vol"])[0]

        fd = (J_at(1) - J_at(-1)) / (2 * eps)
        an = np.sum(gk * c["kappa0"] * dk) + np.sum(gv * dv)
        assert abs(fd - an) <= 1e-7 * abs(an)
