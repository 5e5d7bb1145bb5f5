"""CPU reference of the steady-diffusion adjoint (test infrastructure).

Built on the oracle's own assembly, with no adjoint code of its own: the
residual R(phi, kappa, v) = A phi - b is evaluated by assembling at given
fields, its Jacobians are probed column by column (R is affine in phi and in
v; central differences in kappa), and the adjoint is a dense transpose solve:
    (dR/dphi)^T lambda = dJ/dphi,  dJ/dp = -lambda^T dR/dp.
Small meshes only (one assembly per probe)."""
import numpy as np
import scipy.sparse as sp

from prism_b200 import api


class Residual:
    def __init__(self, case):
        self.c = case
        mesh = case["mesh"]
        ex = mesh.export()
        self.nc, self.nb, self.nf = mesh.n_cells, mesh.info.n_boundary_faces, mesh.n_faces
        self.col = ex["csr_col"][: mesh.info.nnz]
        self.rowptr = ex["csr_rowptr"]

    def __call__(self, phi, kappa, v):
        c = self.c
        c["T"].set_values(phi)
        c["kappa"].set_values(kappa)
        fv = np.zeros(self.nf)
        fv[: self.nb] = v
        c["T"].set_face_values(fv)
        eqn = c["eqn"]
        eqn.zero_out_coeffs()
        eqn.update_coeffs()
        vals, b = eqn.system()
        eqn.zero_out_coeffs()
        A = sp.csr_matrix((vals, self.col, self.rowptr), shape=(self.nc, self.nc))
        return A @ phi - b


def steady_state(case, max_outer=500, tol=1e-14):
    """Repeat solve() (n_iter=1) on the oracle until the relative change is <= tol."""
    T, eqn = case["T"], case["eqn"]
    solver = api.BiCGSTAB()
    prev = T.values()
    for k in range(max_outer):
        solver.solve(eqn, 1, 0.0)
        cur = T.values()
        ch = np.linalg.norm(cur - prev) / max(np.linalg.norm(cur), 1e-300)
        prev = cur
        if ch <= tol:
            return cur, k + 1
    return prev, max_outer


def adjoint_gradients(case, phi, kappa, v, dJ, h_rel=1e-6):
    """(dJ/dkappa, dJ/dv, lambda) at the state phi by dense Jacobians of the oracle residual."""
    R = Residual(case)
    nc, nb = R.nc, R.nb
    r0 = R(phi, kappa, v)
    z = np.zeros(nc)
    rz = R(z, kappa, v)
    Jphi = np.empty((nc, nc))
    for k in range(nc):
        e = np.zeros(nc)
        e[k] = 1.0
        Jphi[:, k] = R(e, kappa, v) - rz
    lam = np.linalg.solve(Jphi.T, dJ)
    gk = np.empty(nc)
    for k in range(nc):
        h = h_rel * kappa[k]
        kp, km = kappa.copy(), kappa.copy()
        kp[k] += h
        km[k] -= h
        gk[k] = -lam @ ((R(phi, kp, v) - R(phi, km, v)) / (2 * h))
    gv = np.empty(nb)
    for f in range(nb):
        vp = v.copy()
        vp[f] += 1.0
        gv[f] = -lam @ (R(phi, kappa, vp) - r0)
    # restore the case's inputs
    R(phi, kappa, v)
    return gk, gv, lam
