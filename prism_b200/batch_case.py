"""A batched diffusion solve (many independent systems in one persistent
launch), for profiling and timing the batched solver.

Builds `count` problems of N^3 unit-cube hexes, N = round(exp(U(ln nmin,
ln nmax))) (seed 4); per problem kappa ~ lognormal(0, 1) and f ~ N(0, 1) per
cell (seeded), T Fixed 0 on all walls, Corrected diffusion; then solves them
together (mixed precision unless --fp64) and prints sizes, iterations and time.
The first solve also autotunes the launch shape (a few steps of each candidate).

    python -m prism_b200.batch_case [--count 64] [--nmin 16] [--nmax 48] [--fp64] [--repeat 1]
"""
import argparse
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _abi as A
from . import api, io, lib, meshgen


def problem(N, library, seed):
    unv = meshgen.box_hex(N, N, N)
    names = meshgen.PATCHES
    case = io.Case.from_dict(names, {"T": {p: ("fixed", 0.0) for p in names}})
    mesh = api.Mesh(unv, case, lib=library)
    rng = np.random.default_rng(seed)
    kappa = api.Scalar("kappa", mesh, rng.lognormal(0.0, 1.0, mesh.n_cells))
    f = api.Scalar("f", mesh, rng.normal(0.0, 1.0, mesh.n_cells))
    T = api.Scalar("T", mesh, 0.0)
    eqn = api.Transport(api.diffusion.Corrected(kappa, T), api.source.ConstantScalar(f))
    return dict(mesh=mesh, T=T, kappa=kappa, f=f, eqn=eqn)


def sizes(count, seed=4, nmin=16, nmax=96):
    rng = np.random.default_rng(seed)
    return [int(round(float(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))) for _ in range(count)]


def build(count, nmin, nmax, library=None, threads=16):
    """The problems, built on `threads` host threads (mesh construction releases the GIL)."""
    library = library or lib()
    ns = sizes(count, 4, nmin, nmax)
    with ThreadPoolExecutor(threads) as ex:
        return ns, list(ex.map(lambda a: problem(a[1], library, 1000 + a[0]), enumerate(ns)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--nmin", type=int, default=16)
    ap.add_argument("--nmax", type=int, default=48)
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args()
    ns, probs = build(a.count, a.nmin, a.nmax)
    prec = A.PREC_FP64 if a.fp64 else A.PREC_MIXED
    bs = api.BatchSolver(api.BiCGSTAB(precision=prec, krylov_tol=1e-10))
    for _ in range(a.repeat):
        for p in probs:
            p["T"].set_values(np.zeros(p["mesh"].n_cells))
        t = time.perf_counter()
        res = bs.solve([p["eqn"] for p in probs])
        dt = time.perf_counter() - t
        print(f"{len(ns)} systems, {sum(p['mesh'].n_cells for p in probs)} cells, max iterations "
              f"{max(r.krylov_iterations for r in res)}, worst rel residual "
              f"{max(r.krylov_rel_residual for r in res):.2e}, {dt:.3f} s")


if __name__ == "__main__":
    main()
