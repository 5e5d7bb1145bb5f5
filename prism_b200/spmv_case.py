"""A short BiCGSTAB run on a matrix larger than L2, for kernel profiling.

Builds the 128^3 jittered-hex transport system (LinearUpwind + Corrected,
2,097,152 cells, 14.6M nonzeros: 217 MB of FP64 CSR, larger than the 126 MB L2),
assembles it and runs one BiCGSTAB step capped at a few iterations, so that a
profiler can capture individual SELL-32 SpMV launches with few launches before
them. Prints the Krylov iteration count.

    python -m prism_b200.spmv_case [--n 128] [--iters 3] [--mixed] [--preconditioner jacobi|amg]
                                   [--tol 1e-12]

With --preconditioner amg the step also builds the AMG hierarchy (setup) and
runs V-cycles around every SpMV; --iters 0 runs the step to --tol.
"""
import argparse

import numpy as np

from . import _abi as A
from . import api, io, lib, meshgen


def build(n, library=None):
    unv = meshgen.box_hex(n, n, n, jitter=0.2, seed=3)
    names = meshgen.PATCHES
    fields = {"T": {p: ("zero-gradient", None) for p in names}, "U": {p: ("zero-gradient", None) for p in names}}
    fields["T"]["left"] = ("fixed", 1.0)
    fields["T"]["right"] = ("fixed", 0.0)
    case = io.Case.from_dict(names, fields, {"T": {"gradScheme": "greenGauss"}, "U": {}})
    mesh = api.Mesh(unv, case, lib=library)
    cc = mesh.export()["cell_center"]
    U = api.Vector("U", mesh, np.stack([np.sin(np.pi * cc[0]) * np.cos(np.pi * cc[1]),
                                        -np.cos(np.pi * cc[0]) * np.sin(np.pi * cc[1]), 0 * cc[0]]))
    T = api.Scalar("T", mesh, 0.0)
    k = api.Scalar("kappa", mesh, 1e-3)
    eqn = api.Transport(api.convection.LinearUpwind(U, T), api.diffusion.Corrected(k, T))
    return mesh, T, U, k, eqn


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--preconditioner", default="jacobi", choices=["jacobi", "amg"])
    ap.add_argument("--tol", type=float, default=1e-12)
    a = ap.parse_args()
    mesh, T, U, k, eqn = build(a.n, lib())
    prec = A.PREC_MIXED if a.mixed else A.PREC_FP64
    r = api.BiCGSTAB(precision=prec, krylov_tol=a.tol, krylov_max_iter=a.iters if a.iters > 0 else 100000,
                     preconditioner=a.preconditioner).solve(eqn, 1, 0.0)
    print(f"cells {mesh.n_cells} nnz {mesh.info.nnz} krylov iterations {r.krylov_iterations} status {r.status}")


if __name__ == "__main__":
    main()
