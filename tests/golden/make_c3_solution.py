"""FP64 reference solution x* of the 128^3 transport system (C3 shape), computed on
the CPU by the reference's own code (oracle/_ref/libprism_ref.so, built by
oracle/ref_build.py), or by the CPU oracle's restatement with --oracle.

The system is the one a single ISolver::solve step assembles from T = 0
(numerics/solver.cpp:27-82 with n_iter = 1): 128^3 hexes on the unit cube,
interior nodes jittered by +-0.2h (seed 3), U = (sin pi x cos pi y,
-cos pi x sin pi y, 0) at cell centroids, kappa = 1e-3, MUSCL convection +
Corrected diffusion, Green-Gauss gradients, T fixed 1 at x = 0 and 0 at x = 1.
The reference solves it with BiCGSTAB + ILUT to machine precision
(numerics/bicgstab.cpp:7-9).

Writes the full vector to tests/golden/c3_<n>_solution.npy (16.8 MB at 128^3; not
committed, generated once and read by bench.py) and a committed summary
tests/golden/c3_<n>_solution.json (norm, checksum and a sample of every 4096th
value) that bench.py and the tests check the vector against.

    python tests/golden/make_c3_solution.py [--n 128] [--oracle]
"""
import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SAMPLE_STRIDE = 4096


def paths(n):
    return os.path.join(HERE, f"c3_{n}_solution.npy"), os.path.join(HERE, f"c3_{n}_solution.json")


def summary(x):
    return {"cells": int(x.size), "norm2": float(np.linalg.norm(x)), "sum": float(np.sum(x)),
            "sha256": hashlib.sha256(np.ascontiguousarray(x, np.float64).tobytes()).hexdigest(),
            "sample_stride": SAMPLE_STRIDE, "sample": [float(v) for v in x[::SAMPLE_STRIDE]]}


def solve_reference(n):
    from oracle import ref_lib as R
    from prism_b200 import meshgen
    from tests import cases
    unv = meshgen.box_hex(n, n, n, jitter=0.2, seed=3)
    case = cases.box_case({"T": {"left": ("fixed", 1.0), "right": ("fixed", 0.0)}, "U": {}},
                          {"T": {"gradScheme": "greenGauss"}, "U": {}})
    mesh = R.Mesh(unv, case)
    cc = mesh.cells()["center"]
    U = np.stack([np.sin(np.pi * cc[0]) * np.cos(np.pi * cc[1]),
                  -np.cos(np.pi * cc[0]) * np.sin(np.pi * cc[1]), np.zeros(mesh.n_cells)])
    return R.transport(mesh, conv="MUSCL", U=U, kappa=1e-3, outer=1, n_iter=1, eps=0.0)


def solve_oracle(n):
    import oracle
    from prism_b200 import api
    from tests import cases
    mesh, T, U, eqn = cases.transport_c3(n, oracle.lib(), conv="MUSCL")
    api.BiCGSTAB().solve(eqn, 1, 0.0)
    return T.values()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--oracle", action="store_true", help="use the CPU oracle's restatement")
    a = ap.parse_args()
    t = time.time()
    x = solve_oracle(a.n) if a.oracle else solve_reference(a.n)
    secs = time.time() - t
    npy, js = paths(a.n)
    np.save(npy, x)
    s = summary(x)
    s.update({"n": a.n, "solver": "CPU oracle restatement" if a.oracle else "reference code (oracle/_ref)",
              "seconds": secs})
    with open(js, "w") as fh:
        json.dump(s, fh, indent=1)
    print(f"{npy}: {x.size} values, {secs:.0f} s")


if __name__ == "__main__":
    main()
