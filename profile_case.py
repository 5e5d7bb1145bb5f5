"""Short runs of the hot path on cases larger than L2, for kernel profiling
(bench tooling beside bench.py: profiles/*.md give the ncu commands that run it).

    python profile_case.py [--case c3|cavity|sweep|assemble] [--n N] [--conv MUSCL] [--grad gg|ls]
                           [--iters 3] [--mixed] [--preconditioner jacobi|amg] [--tol 1e-12] [--repeat R]

--case c3 (default): the 128^3 jittered-hex transport system (2,097,152 cells, 14.6M
nonzeros, 217 MB of FP64 CSR), assembled once (the assembly kernel, the Green-Gauss
sweep or the least-squares gradient) and one BiCGSTAB step capped at --iters
iterations, so that a profiler captures single launches with few launches before
them. --case cavity: one SIMPLE outer iteration of the n x n x 1 lid-driven cavity
(Upwind + Corrected, Rhie-Chow face fluxes, pressure correction). Prints the Krylov
iteration count. --case sweep / assemble: the C3 system's gradient sweep
(computeAllCellGradients) / assembly (updateCoeffs) repeated --repeat times after one
warm-up, timed between two device synchronizations (the library runs on the mesh's
own stream; prints milliseconds per call).
"""
import argparse
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from prism_b200 import _abi as A  # noqa: E402
from prism_b200 import api, io, lib, meshgen  # noqa: E402


def build_c3(n, library=None, conv="LinearUpwind", grad="gg"):
    unv = meshgen.box_hex(n, n, n, jitter=0.2, seed=3)
    names = meshgen.PATCHES
    fields = {"T": {p: ("zero-gradient", None) for p in names}, "U": {p: ("zero-gradient", None) for p in names}}
    fields["T"]["left"] = ("fixed", 1.0)
    fields["T"]["right"] = ("fixed", 0.0)
    info = {"T": {"gradScheme": "greenGauss"} if grad == "gg" else {}, "U": {}}
    case = io.Case.from_dict(names, fields, info)
    mesh = api.Mesh(unv, case, lib=library)
    cc = mesh.export()["cell_center"]
    U = api.Vector("U", mesh, np.stack([np.sin(np.pi * cc[0]) * np.cos(np.pi * cc[1]),
                                        -np.cos(np.pi * cc[0]) * np.sin(np.pi * cc[1]), 0 * cc[0]]))
    T = api.Scalar("T", mesh, 0.0)
    k = api.Scalar("kappa", mesh, 1e-3)
    eqn = api.Transport(getattr(api.convection, conv)(U, T), api.diffusion.Corrected(k, T))
    return mesh, T, U, k, eqn


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="c3", choices=["c3", "cavity", "sweep", "assemble"])
    ap.add_argument("--repeat", type=int, default=10)
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--conv", default="LinearUpwind")
    ap.add_argument("--grad", default="gg", choices=["gg", "ls"])
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--preconditioner", default="jacobi", choices=["jacobi", "amg", "auto"])
    ap.add_argument("--tol", type=float, default=1e-12)
    a = ap.parse_args()
    prec = A.PREC_MIXED if a.mixed else A.PREC_FP64
    solver = api.BiCGSTAB(precision=prec, krylov_tol=a.tol, krylov_max_iter=a.iters if a.iters > 0 else 100000,
                          preconditioner=a.preconditioner)
    if a.case in ("sweep", "assemble"):
        import torch
        mesh, T, U, k, eqn = build_c3(a.n or 128, lib(), a.conv, a.grad)
        cc = mesh.export()["cell_center"]
        T.set_values(np.sin(2 * cc[0]) * np.cos(cc[1]) + cc[2])

        def once():
            if a.case == "sweep":
                T.compute_all_cell_gradients()
            else:
                eqn.update_coeffs()
                eqn.zero_out_coeffs()
        once()
        torch.cuda.synchronize()  # the library works on the mesh's own stream: time the device
        t0 = time.perf_counter()
        for _ in range(a.repeat):
            once()
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1000.0 / a.repeat
        print(f"{a.case} cells {mesh.n_cells} ms per call {ms:.4f}")
        return
    if a.case == "c3":
        mesh, T, U, k, eqn = build_c3(a.n or 128, lib(), a.conv, a.grad)
        r = solver.solve(eqn, 1, 0.0)
        print(f"cells {mesh.n_cells} nnz {mesh.info.nnz} krylov iterations {r.krylov_iterations} status {r.status}")
    else:
        from tests import cases
        mesh, U, p, nu, mdot, eqs = cases.cavity(a.n or 1448, lib())
        reps = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=solver).step(eqs, U, mdot, p)
        print(f"cells {mesh.n_cells} reports {[(r.field_name, r.n_iterations) for r in reps]}")


if __name__ == "__main__":
    main()
