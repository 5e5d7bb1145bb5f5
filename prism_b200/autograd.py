"""torch.autograd binding of the steady-diffusion forward/backward pair.

    problem = SteadyDiffusionProblem(eqn, phi, kappa)       # api objects, phi Fixed patches
    T = steady_diffusion(kappa_t, face_t, problem)          # torch tensors, float64, CPU or CUDA
    J = ((T - T_star) ** 2 * V).sum(); J.backward()         # kappa_t.grad, face_t.grad

kappa_t holds one value per cell, face_t one Dirichlet value per boundary face
(faces of empty patches and of patches without a value are ignored). The
forward repeats the solve to the steady state (prism_adjoint_forward), the
backward solves the discrete adjoint (prism_adjoint_backward); nothing but the
problem's own fields is kept between the two.
"""
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import api


@dataclass
class SteadyDiffusionProblem:
    eqn: api.Transport
    phi: api.Scalar
    kappa: api.Scalar
    solver: api.BiCGSTAB = field(default_factory=lambda: api.BiCGSTAB(krylov_tol=1e-13))
    max_outer: int = 200
    outer_tol: float = 1e-13
    last_forward: Optional[api.FixedPointResult] = None
    last_backward: Optional[api.FixedPointResult] = None

    def set_inputs(self, kappa: np.ndarray, face_values: np.ndarray):
        mesh = self.phi.mesh
        self.kappa.set_values(kappa)
        fv = np.zeros(mesh.n_faces)
        fv[: mesh.info.n_boundary_faces] = face_values
        self.phi.set_face_values(fv)

    def forward(self, kappa: np.ndarray, face_values: np.ndarray, phi0=None) -> np.ndarray:
        self.set_inputs(kappa, face_values)
        if phi0 is not None:
            self.phi.set_values(phi0)
        self.last_forward = api.adjoint_forward(self.eqn, self.solver, self.max_outer, self.outer_tol)
        return self.phi.values()

    def backward(self, dJ_dphi: np.ndarray):
        gk, gv, self.last_backward = api.adjoint_backward(self.eqn, dJ_dphi, self.solver, self.max_outer,
                                                          self.outer_tol)
        return gk, gv


def _function():
    import torch

    class SteadyDiffusion(torch.autograd.Function):
        @staticmethod
        def forward(ctx, kappa, face_values, problem):
            phi = problem.forward(kappa.detach().cpu().double().numpy(), face_values.detach().cpu().double().numpy())
            ctx.problem = problem
            return torch.as_tensor(phi, dtype=torch.float64, device=kappa.device)

        @staticmethod
        def backward(ctx, grad_phi):
            gk, gv = ctx.problem.backward(grad_phi.detach().cpu().double().numpy())
            dev = grad_phi.device
            return (torch.as_tensor(gk, dtype=torch.float64, device=dev),
                    torch.as_tensor(gv, dtype=torch.float64, device=dev), None)

    return SteadyDiffusion


_FN = None


def steady_diffusion(kappa, face_values, problem: SteadyDiffusionProblem):
    """phi(kappa, face_values) at the steady state, differentiable in both inputs."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(kappa, face_values, problem)
