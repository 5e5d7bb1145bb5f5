"""Benchmark of the sm_100a Prism hot path.

Headline workload (N=1): steady lid-driven cavity, Re=100 (nu=0.01, lid u=1),
Upwind convection + Corrected diffusion + pressure-gradient source, SIMPLE with
urf 0.7/0.3 (the 512x512 cavity recipe) on 1448x1448x1 hexes (2,096,704 cells): the
"2M-cell SIMPLE it/s" of the metric. One step = one SIMPLE outer iteration
(2 momentum solves + 3 pressure solves, each step() solved to ||b-Ax|| <=
1e-12 ||b|| like the reference's machine-precision step: the momentum predictors by
BiCGSTAB with the Jacobi preconditioner that PRISM_PC_AUTO picks for their
diagonally dominant matrices, the pressure correction by flexible CG preconditioned
by an FP32 AMG V-cycle), run as one CUDA graph
launch (PrismSolveOpts.graph: the solver loops are device-side conditional nodes
and the kernels are those of the ordinary path, so the fields are identical).
Inputs live in HBM; the working set (~1 GB) is larger than L2, so no flush is
needed. The same steps on the ordinary path (every kernel launched from the host)
are reported as "simple_eager", with the live bandwidth samples, and the same solver
timed again after --late-steps more iterations as "simple_later" (the developed flow).

Also reported: time to 1e-8 relative error of the 128^3 jittered-hex transport
solve (MUSCL + Corrected + Green-Gauss, one step() of the system assembled at
T = 0) against the FP64 reference solution computed on the CPU by the
reference's own code (tests/golden/c3_128_solution.npy, made by
tests/golden/make_c3_solution.py and checked against its committed summary),
FP64 vs FP32/FP64-reliable-update BiCGSTAB, both AMG-preconditioned, and FP64
with the Jacobi preconditioner ("s_to_1e8"); the live bandwidth of the dominant
kernels (the finest-level AMG post-smoothing and restriction SpMVs, the flexible-CG
SpMV and the BiCGSTAB SpMV: CUDA events around sampled launches of the ordinary-path
run);
the discrete adjoint of steady diffusion on 64^3 x 6 tets ("adjoint": times and
finite-difference agreement) and 256 independent diffusion solves in one
persistent launch ("batched").

--impl reference times the reference's own code (oracle/_ref/libprism_ref.so,
compiled from the reference's sources; single-threaded, like the reference) on a
bounded sample of the same workload: one SIMPLE outer iteration of the 724x724x1
cavity after one untimed one, it/s scaled to the 1448x1448x1 cavity by the cell
ratio (a full-size iteration takes the reference about ten minutes; its cost grows
faster than the cell count, so the scaled figure flatters it). The CPU restatement
(the oracle) stands in when the compiled reference is absent.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s-to-1e-8 err (FP32+refine vs FP64 GPU), 2M-cell SIMPLE it/s, SpMV HBM GB/s"
N_CAVITY = 1448
REF_SAMPLE_N = 724  # the reference arm's sample: a quarter of the cells
N_CPU = 362  # the bounded CPU sample of the GPU arm: 1/16 of the cells
UNIT = "SIMPLE it/s"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([t.strip() for t in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
            except (ValueError, IndexError):
                continue
            for k, name in enumerate(names):
                if len(r) > 3 + k and r[3 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        import datetime
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cavity_case(n):
    """Mesh and boundary conditions of the lid-driven cavity (the same case as tests/cases.cavity)."""
    from prism_b200 import meshgen
    from tests import cases
    unv = meshgen.box_hex(n, n, 1, (1.0, 1.0, 1.0 / n))
    wall = ("no-slip", [0.0, 0.0, 0.0])
    case = cases.box_case({"U": {"top": ("fixed", [1.0, 0.0, 0.0]), "left": wall, "right": wall, "bottom": wall,
                                 "back": ("empty", None), "front": ("empty", None)},
                           "P": {"back": ("empty", None), "front": ("empty", None)}})
    return unv, case


def cpu_simple(n, warm=1, timed=1):
    """SIMPLE outer iterations of the n x n cavity on the CPU by the reference's own code
    (oracle/_ref, "reference"), else by the oracle's restatement ("port"): seconds of each
    timed iteration after `warm` untimed ones, single-threaded like the reference."""
    from oracle import ref_lib
    if ref_lib.available():
        unv, case = cavity_case(n)
        mesh = ref_lib.Mesh(unv, case)
        r = ref_lib.simple(mesh, warm + timed, nu=0.01, conv="Upwind", timings=True)
        return list(r["seconds"][warm:]), "reference"
    import oracle
    from prism_b200 import api
    from tests import cases
    mesh, U, p, nu, mdot, eqs = cases.cavity(n, oracle.lib())
    simple = api.IncompressibleSIMPLE(api.SIMPLEControls())
    out = []
    for i in range(warm + timed):
        t0 = time.perf_counter()
        simple.step(eqs, U, mdot, p)
        if i >= warm:
            out.append(time.perf_counter() - t0)
    return out, "port"


def run_reference(args, world, rank):
    """The reference's own CPU code (oracle/_ref, else the oracle's restatement) on a bounded
    sample of the bench workload: one SIMPLE outer iteration of the --ref-n cavity after one
    untimed one (about three minutes on one core at 724^2), its it/s scaled to the stated
    1448^2 cavity by the cell ratio. The reference's iteration cost grows faster than the cell
    count (its ILUT-BiCGSTAB pressure solves need more iterations on finer meshes), so the
    scaled figure overstates the reference's speed at the full size."""
    if rank != 0:
        return
    n = args.ref_n
    secs, kind = cpu_simple(n, warm=1, timed=1)
    dt = sum(secs) / len(secs)
    scale = (n * n) / float(N_CAVITY * N_CAVITY)
    value = scale / dt
    who = "the reference's own code (oracle/_ref)" if kind == "reference" else "the oracle's restatement"
    sample = (f"{len(secs)} SIMPLE outer iteration of the {n}x{n}x1 cavity ({n * n} cells, {dt:.1f} s each, "
              f"ms_per_step) after 1 untimed one, by {who}, single-threaded like the reference; it/s scaled by "
              f"the cell ratio {n * n}/{N_CAVITY * N_CAVITY} to the stated cavity (a bounded sample: a full-size "
              f"iteration takes the reference about ten minutes); one iteration is timed whatever --steps asks "
              f"({args.steps})")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": len(secs), "steps_requested": args.steps, "warmup": 1, "ms_per_step": 1000.0 * dt,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"cavity SIMPLE {N_CAVITY}x{N_CAVITY}x1 ({N_CAVITY * N_CAVITY} cells), Re=100, "
                                   "Upwind + Corrected, urf 0.7/0.3, BiCGSTAB + ILUT to machine precision (the "
                                   "reference's solver::BiCGSTAB)", "cells": N_CAVITY * N_CAVITY,
                       "sample_cells": n * n},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def transport_mesh(lib, n):
    """The C3 mesh: n^3 hexes, interior nodes jittered by +-0.2h (seed 3)."""
    from tests import cases
    mesh, T, U, eqn = cases.transport_c3(n, lib, conv="MUSCL")
    return mesh


def transport_eqn(mesh):
    """Fresh fields and equation on the C3 mesh (fresh Green-Gauss state, T = 0): MUSCL
    convection + Corrected diffusion, Green-Gauss gradients (the mesh's case sets them)."""
    import numpy as np
    from prism_b200 import api
    cc = mesh.export()["cell_center"]
    U = api.Vector("U", mesh, np.stack([np.sin(np.pi * cc[0]) * np.cos(np.pi * cc[1]),
                                        -np.cos(np.pi * cc[0]) * np.sin(np.pi * cc[1]), np.zeros(mesh.n_cells)]))
    T = api.Scalar("T", mesh, 0.0)
    k = api.Scalar("kappa", mesh, 1e-3)
    eqn = api.Transport(api.convection.MUSCL(U, T), api.diffusion.Corrected(k, T))
    return T, (U, k), eqn


def cpu_reference_solution(n):
    """x* of the system assembled at T = 0, solved on the CPU by the reference's own code
    (BiCGSTAB + ILUT to machine precision), as written by tests/golden/make_c3_solution.py:
    returned only when the stored vector matches its committed summary (checksum)."""
    import hashlib
    import numpy as np
    npy = os.path.join(ROOT, "tests", "golden", f"c3_{n}_solution.npy")
    js = os.path.join(ROOT, "tests", "golden", f"c3_{n}_solution.json")
    if not (os.path.exists(npy) and os.path.exists(js)):
        return None, None
    with open(js) as fh:
        summ = json.load(fh)
    x = np.load(npy)
    if hashlib.sha256(np.ascontiguousarray(x, np.float64).tobytes()).hexdigest() != summ["sha256"]:
        return None, None
    return x, summ


def transport_exact(mesh):
    """x* of the system assembled at T = 0 on the GPU: FP64 BiCGSTAB to ||b - Ax|| <= 1e-14 ||b||."""
    from prism_b200 import api
    T, keep, eqn = transport_eqn(mesh)
    api.BiCGSTAB(krylov_tol=1e-14, krylov_max_iter=100000, preconditioner="jacobi").solve(eqn, 1, 0.0)
    return T.values()


def transport_time_to_tol(mesh, precision, ref, tol=1e-8, preconditioner="auto"):
    """Seconds (CUDA events) for one solve() step from T = 0 (assembly included) to reach
    ||T - x*|| / ||x*|| <= tol: the loosest Krylov tolerance of a 10^-0.5 ladder that meets
    the error is timed (the fastest of five identical runs, so that a one-off host stall in
    one run does not decide the figure)."""
    import numpy as np
    import torch
    from prism_b200 import api
    nref = np.linalg.norm(ref)
    last = None
    for e in np.arange(8.0, 14.01, 0.5):
        ktol = 10.0 ** (-e)
        solver = api.BiCGSTAB(precision=precision, krylov_tol=ktol, krylov_max_iter=100000,
                              preconditioner=preconditioner)
        best = None
        for rep in range(5):
            T, keep, eqn = transport_eqn(mesh)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = solver.solve(eqn, 1, 0.0)
            e1.record()
            torch.cuda.synchronize()
            secs = e0.elapsed_time(e1) / 1000.0
            best = secs if best is None else min(best, secs)
        secs = best
        err = float(np.linalg.norm(T.values() - ref) / nref)
        last = {"seconds": secs, "krylov_tol": ktol, "krylov_iterations": r.krylov_iterations, "error": err}
        if err <= tol:
            return last
    last["error_not_reached"] = True
    return last


def adjoint_measure(lib, n=64, directions=2):
    """Discrete adjoint of steady diffusion on n^3 x 6 tets (kappa ~ lognormal(0, 0.5), Fixed face values
    ~ U(0, 1), J = sum V (T - T*)^2): forward and backward times, and fourth-order central differences
    of J along random directions against the adjoint gradient."""
    import numpy as np
    import torch
    from prism_b200 import api
    from tests import cases
    t = time.perf_counter()
    c = cases.adjoint_c5(n, lib)
    t_build = time.perf_counter() - t
    S = api.BiCGSTAB(krylov_tol=1e-13, krylov_max_iter=100000)
    torch.cuda.synchronize()
    t = time.perf_counter()
    fw = api.adjoint_forward(c["eqn"], S, max_outer=500, outer_tol=1e-13)
    t_fw = time.perf_counter() - t
    phi0 = c["T"].values()
    _, dJ = cases.objective(phi0, c["T_star"], c["vol"])
    t = time.perf_counter()
    gk, gv, bw = api.adjoint_backward(c["eqn"], dJ, S, max_outer=500, outer_tol=1e-13)
    t_bw = time.perf_counter() - t
    rng = np.random.default_rng(32)
    eps, errs = 1e-3, []
    for _ in range(directions):
        dk = rng.normal(size=c["mesh"].n_cells)
        dv = rng.normal(size=len(c["v0"]))

        def J_at(sgn):
            c["kappa"].set_values(c["kappa0"] * (1 + sgn * eps * dk))
            fv = np.zeros(c["mesh"].n_faces)
            fv[: len(dv)] = c["v0"] + sgn * eps * dv
            c["T"].set_face_values(fv)
            c["T"].set_values(phi0)
            api.adjoint_forward(c["eqn"], S, max_outer=500, outer_tol=1e-13)
            return cases.objective(c["T"].values(), c["T_star"], c["vol"])[0]

        fd = (8 * (J_at(1) - J_at(-1)) - (J_at(2) - J_at(-2))) / (12 * eps)
        an = float(np.sum(gk * c["kappa0"] * dk) + np.sum(gv * dv))
        errs.append(abs(fd - an) / abs(an))
    return {"workload": f"{n}^3 cubes x 6 tets ({c['mesh'].n_cells} cells), kappa ~ lognormal(0,0.5), Fixed face "
                        f"values ~ U(0,1), Corrected diffusion, least-squares gradient, J = sum V (T - T*)^2",
            "mesh_build_s": t_build, "forward_s": t_fw, "forward_outer": fw.outer_iterations,
            "forward_krylov": fw.krylov_iterations, "backward_s": t_bw, "backward_outer": bw.outer_iterations,
            "backward_krylov": bw.krylov_iterations, "fd_rel_errors": errs,
            "fd": f"fourth-order central differences, eps = {eps} (relative in kappa)"}


def batched_measure(lib, count=256, nmin=16, nmax=96):
    """count independent diffusion problems (N^3 hexes, N log-uniform in [nmin, nmax], seed 4) solved in one
    persistent launch (mixed precision), against the same systems solved one by one (FP64, Jacobi)."""
    import numpy as np
    import torch
    from prism_b200 import _abi as A
    from prism_b200 import api
    from prism_b200.batch_case import build
    t = time.perf_counter()
    sizes, probs = build(count, nmin, nmax, lib)
    t_build = time.perf_counter() - t
    cells = sum(p["mesh"].n_cells for p in probs)
    bs = api.BatchSolver(api.BiCGSTAB(precision=A.PREC_MIXED, krylov_tol=1e-10), lib=lib)
    times = []
    for rep in range(2):  # the first call builds the plan and tunes the launch shape
        for p in probs:
            p["T"].set_values(np.zeros(p["mesh"].n_cells))
        torch.cuda.synchronize()
        t = time.perf_counter()
        res = bs.solve([p["eqn"] for p in probs])
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t)
    for p in probs:
        p["T"].set_values(np.zeros(p["mesh"].n_cells))
    s = api.BiCGSTAB(krylov_tol=1e-10, preconditioner="jacobi")
    torch.cuda.synchronize()
    t = time.perf_counter()
    seq_its = [s.solve(p["eqn"], 1, 0.0).krylov_iterations for p in probs]
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t

    def iter_bytes(n, nnz, w):
        # one Jacobi-preconditioned BiCGSTAB iteration at fused-minimum traffic: two SpMVs
        # (values, columns, row offsets, x read, y written) and 23 vector passes
        return 2 * (nnz * (w + 4) + 4 * (n + 1) + 2 * w * n) + 23 * w * n
    shapes = [(p["mesh"].n_cells, p["mesh"].info.nnz) for p in probs]
    bytes_batched = sum(r.krylov_iterations * iter_bytes(n, z, 4) for r, (n, z) in zip(res, shapes))
    bytes_seq = sum(k * iter_bytes(n, z, 8) for k, (n, z) in zip(seq_its, shapes))
    return {"workload": f"{count} problems, N^3 hexes with N = round(exp(U(ln {nmin}, ln {nmax}))) (seed 4), "
                        f"{cells} cells; kappa ~ lognormal(0,1), f ~ N(0,1), Fixed 0 walls, Corrected diffusion; "
                        f"||b - Ax|| <= 1e-10 ||b||",
            "mesh_build_s": t_build, "first_call_s": times[0], "batched_s": times[1],
            "solves_per_s": count / times[1], "max_iterations": max(r.krylov_iterations for r in res),
            "worst_rel_residual": max(r.krylov_rel_residual for r in res),
            "failed": sum(r.status != 0 for r in res),
            "sequential_fp64_jacobi_s": t_seq, "sequential_max_iterations": max(seq_its),
            "speedup_vs_sequential": t_seq / times[1],
            "total_iterations": sum(r.krylov_iterations for r in res), "sequential_total_iterations": sum(seq_its),
            "achieved_gbs": bytes_batched / times[1] / 1e9, "sequential_achieved_gbs": bytes_seq / t_seq / 1e9,
            "achieved_note": "algorithmic bytes of the Krylov iterations (FP32 for the batch, its FP64 refinement "
                             "steps not counted; FP64 one by one, each call's assembly not counted) / wall time"}


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    import prism_b200
    from prism_b200 import _abi as A
    from prism_b200 import api
    from tests import cases

    torch.cuda.set_device(local)
    lib = prism_b200.lib()
    hbm, peak_kind = peaks()

    t_build = time.perf_counter()
    mesh, U, p, nu, mdot, eqs = cases.cavity(N_CAVITY, lib)
    t_build = time.perf_counter() - t_build
    n = mesh.n_cells

    def fresh():
        # identical initial state (fields at rest) for every run below
        U_, p_, nu_, mdot_ = cases.simple_fields(mesh, 0.01)
        return U_, p_, nu_, mdot_, cases.momentum_eqns(U_, p_, nu_, mdot_, conv="Upwind")

    # headline: each SIMPLE outer iteration is one CUDA graph launch (PrismSolveOpts.graph: the
    # solver loops run as device-side conditional nodes; the kernels and their order are those of
    # the ordinary path, so the fields are identical). The first warm-up step builds the AMG
    # hierarchies and work buffers the graph uses.
    gsolver = api.BiCGSTAB(krylov_tol=1e-12, krylov_max_iter=30000, graph=True)
    gsimple = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=gsolver)
    for _ in range(args.warmup):
        gsimple.step(eqs, U, mdot, p)
    clocks = Clocks(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    lib.check(lib.profile_start(16))
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record()
    reports = []
    for _ in range(args.steps):
        reports = gsimple.step(eqs, U, mdot, p)
    g1.record()
    torch.cuda.synchronize()
    gprof = A.Profile()
    lib.check(lib.profile_stop(ctypes.byref(gprof)))
    clk = clocks.stop()
    barrier(world)
    t_dev = max_over_ranks(world, g0.elapsed_time(g1) / 1000.0)
    value = world * args.steps / t_dev

    # later in the run: the same solver continued for late_steps untimed steps (the pressure
    # solves cost differently once the flow has developed), then steps timed again
    late = None
    if args.late_steps > 0:
        for _ in range(args.late_steps):
            gsimple.step(eqs, U, mdot, p)
        torch.cuda.synchronize()
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0.record()
        late_reports = []
        for _ in range(args.steps):
            late_reports = gsimple.step(eqs, U, mdot, p)
        l1.record()
        torch.cuda.synchronize()
        t_late = max_over_ranks(world, l0.elapsed_time(l1) / 1000.0)
        late = {"value": world * args.steps / t_late, "unit": UNIT, "ms_per_step": 1000.0 * t_late / args.steps,
                "timed_after_iterations": args.warmup + args.steps + args.late_steps,
                "last_step_reports": [(r.field_name, r.n_iterations, r.initial_residual, r.final_residual)
                                      for r in late_reports]}

    # end to end through the public API with pinned host buffers, same initial state
    U, p, nu, mdot, eqs = fresh()
    for _ in range(args.warmup):
        gsimple.step(eqs, U, mdot, p)
    hU = torch.empty(3 * n, dtype=torch.float64, pin_memory=True).numpy()
    hp = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    hU[:] = U.values().reshape(-1)
    hp[:] = p.values()
    barrier(world)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(args.steps):
        lib.check(lib.vector_set_values(U.h, hU.ctypes.data_as(A.pf64)))
        lib.check(lib.scalar_set_values(p.h, hp.ctypes.data_as(A.pf64)))
        gsimple.step(eqs, U, mdot, p)
        lib.check(lib.vector_get_values(U.h, hU.ctypes.data_as(A.pf64)))
        lib.check(lib.scalar_get_values(p.h, hp.ctypes.data_as(A.pf64)))
    t1.record()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(world, t0.elapsed_time(t1) / 1000.0)
    e2e = world * args.steps / t_e2e

    # the same steps launched kernel by kernel from the host (the ordinary path), with the live
    # samples of the dominant kernels (CUDA events around sampled launches on the mesh's stream)
    # and the count of kernel launches per step (the graph runs the same kernels)
    solver = api.BiCGSTAB(krylov_tol=1e-12, krylov_max_iter=30000)
    simple = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=solver)
    U, p, nu, mdot, eqs = fresh()
    for _ in range(args.warmup):
        simple.step(eqs, U, mdot, p)
    barrier(world)
    torch.cuda.synchronize()
    lib.check(lib.profile_start(4096))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        simple.step(eqs, U, mdot, p)
    e1.record()
    torch.cuda.synchronize()
    prof = A.Profile()
    lib.check(lib.profile_stop(ctypes.byref(prof)))
    barrier(world)
    t_eager = max_over_ranks(world, e0.elapsed_time(e1) / 1000.0)
    eager_line = {"value": world * args.steps / t_eager, "unit": UNIT, "ms_per_step": 1000.0 * t_eager / args.steps,
                  "kernel_launches": int(prof.kernel_launches),
                  "note": "the ordinary path: every kernel launched from the host, solver loops on the host"}

    # live samples: BiCGSTAB SpMV and the finest-level AMG cycle kernels
    def live(launches, ms, nbytes):
        if not launches:
            return None, None, None
        avg_ms, avg_b = ms / launches, nbytes / launches
        return avg_b / (avg_ms * 1e-3) / 1e9, avg_ms, avg_b

    spmv_gbs, spmv_ms, spmv_bytes = live(prof.fp64_launches, prof.fp64_ms, prof.fp64_bytes)
    fcg_gbs, fcg_ms, fcg_bytes = live(prof.fcg_launches, prof.fcg_ms, prof.fcg_bytes)
    # the pressure correction's cycle runs in FP32 (flexible CG), other AMG solves in FP64
    a32 = prof.amg32_post_launches > 0
    prec = "float" if a32 else "double"
    post_gbs, post_ms, post_bytes = live(*((prof.amg32_post_launches, prof.amg32_post_ms, prof.amg32_post_bytes) if a32
                                          else (prof.amg_post_launches, prof.amg_post_ms, prof.amg_post_bytes)))
    down_gbs, down_ms, down_bytes = live(*((prof.amg32_down_launches, prof.amg32_down_ms, prof.amg32_down_bytes) if a32
                                          else (prof.amg_down_launches, prof.amg_down_ms, prof.amg_down_bytes)))

    def traffic_for(name, nbytes):
        # DRAM bytes of one launch measured by ncu, scaled to this launch by its algorithmic
        # bytes (same workload: the ratio is the measured traffic per algorithmic byte)
        f = os.path.join(ROOT, "profiles", name)
        if nbytes is None or not os.path.exists(f):
            return None
        with open(f) as fh:
            return json.load(fh)["traffic_per_algorithmic_byte"] * nbytes

    def kernel_line(kernel, gbs, ms, nbytes, launches, traffic_file):
        return {"kernel": kernel, "bound": "hbm", "achieved": gbs, "peak": hbm, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": gbs / hbm if gbs else None, "traffic": traffic_for(traffic_file, nbytes),
                "algorithmic_bytes_per_launch": nbytes, "avg_launch_ms": ms, "sampled_launches": launches}

    spmv = kernel_line("spmv_kernel<double,1> (SELL-32 SpMV + fused dot, BiCGSTAB v = A y: the momentum predictors)",
                spmv_gbs, spmv_ms, spmv_bytes, prof.fp64_launches, "spmv_fp64_traffic.json")
    fcg = kernel_line("fcg_spmv_kernel<4,6,float> (flexible CG u = A z + three fused dots: the pressure correction)",
               fcg_gbs, fcg_ms, fcg_bytes, prof.fcg_launches, "fcg_spmv_traffic.json")
    if post_gbs:
        roof = kernel_line(f"post_kernel<{prec},1> (AMG finest level: prolongation + post-smoothing SpMV)",
                    post_gbs, post_ms, post_bytes, prof.amg32_post_launches if a32 else prof.amg_post_launches,
                    f"amg{'32' if a32 else ''}_post_traffic.json")
        roof["down_kernel"] = kernel_line(f"down_kernel<{prec},1> (AMG finest level: smoothed restriction SpMV)",
                                   down_gbs, down_ms, down_bytes,
                                   prof.amg32_down_launches if a32 else prof.amg_down_launches,
                                   f"amg{'32' if a32 else ''}_down_traffic.json")
    else:
        roof = spmv
    extra = {}
    if rank == 0 and not args.skip_transport:
        nt = args.transport_n
        tmesh = transport_mesh(lib, nt)
        gpu_x = transport_exact(tmesh)
        cpu_x, summ = cpu_reference_solution(nt)
        ref = cpu_x if cpu_x is not None else gpu_x
        r64 = transport_time_to_tol(tmesh, A.PREC_FP64, ref, preconditioner="amg")
        r32 = transport_time_to_tol(tmesh, A.PREC_MIXED, ref, preconditioner="amg")
        rj = transport_time_to_tol(tmesh, A.PREC_FP64, ref, preconditioner="jacobi")
        if cpu_x is not None:
            refsol = (f"CPU FP64 solution by {summ['solver']} (BiCGSTAB + ILUT to machine precision), "
                      f"tests/golden/c3_{nt}_solution.npy, checksum-verified")
        else:
            refsol = "GPU FP64 BiCGSTAB(Jacobi) to ||b-Ax|| <= 1e-14 ||b|| (no stored CPU solution for this size)"
        extra["s_to_1e8"] = {"workload": f"{nt}^3 hexes jittered +-0.2h (seed 3), U = (sin pi x cos pi y, "
                                         f"-cos pi x sin pi y, 0), kappa 1e-3, MUSCL + Corrected + Green-Gauss, "
                                         f"T fixed 1/0 at x=0/1; one step() of the system assembled at T=0 "
                                         f"(assembly, gradient sweep, AMG setup and iterations timed)",
                             "fp64": r64, "mixed": r32, "fp64_jacobi": rj,
                             "speedup": r64["seconds"] / r32["seconds"] if r32["seconds"] > 0 else None,
                             "speedup_vs_fp64_jacobi": rj["seconds"] / r32["seconds"] if r32["seconds"] > 0 else None,
                             "reference_solution": refsol,
                             "gpu_fp64_1e-14_vs_reference_solution": float(
                                 np.linalg.norm(gpu_x - ref) / np.linalg.norm(ref))}

    if rank == 0 and not args.skip_adjoint:
        extra["adjoint"] = adjoint_measure(lib)
    if rank == 0 and not args.skip_batch:
        extra["batched"] = batched_measure(lib)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        # bounded sample: the full-size cavity takes the CPU minutes per iteration (the reference
        # arm, --impl reference, times it); here one iteration of a 1/16-size cavity, scaled
        secs, kind = cpu_simple(N_CPU, warm=1, timed=1)
        dt = secs[0]
        scale = (N_CPU * N_CPU) / float(N_CAVITY * N_CAVITY)
        cpu = {"value": scale / dt, "unit": UNIT, "cores": 1, "kind": kind,
               "sample": f"the second SIMPLE outer iteration of the {N_CPU}x{N_CPU}x1 cavity ({dt:.1f} s, "
                         f"{'the reference' + chr(39) + 's own code' if kind == 'reference' else 'the oracle'}, "
                         f"one core), it/s scaled by the cell ratio {N_CPU * N_CPU}/{N_CAVITY * N_CAVITY}; the "
                         f"full-size iteration is timed by --impl reference"}

    if rank == 0:
        # kernel launches per step, counted from the solver's iteration counts
        kry = sum(r.n_iterations for r in reports)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000.0 * t_dev / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"cavity SIMPLE {N_CAVITY}x{N_CAVITY}x1 ({n} cells), Re=100, Upwind + "
                                       "Corrected, urf 0.7/0.3, solves to 1e-12 (PRISM_PC_AUTO: momentum BiCGSTAB "
                                       "with Jacobi, pressure correction flexible CG with an FP32 AMG V-cycle), "
                                       "each outer iteration one CUDA graph launch (PrismSolveOpts.graph)",
                           "cells": n, "l2": "inputs larger than L2 (no flush)",
                           "parallelism": f"{world} independent replicas" if world > 1 else "1 GPU",
                           "mesh_build_s": t_build},
                "spmv_gbs": spmv_gbs, "roofline": roof, "spmv": spmv, "fcg_spmv": fcg, "clocks": clk,
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(hU.nbytes + hp.nbytes),
                        "d2h_bytes_per_step": int(hU.nbytes + hp.nbytes)},
                "gpu_launches": int(prof.kernel_launches),
                "gpu_launches_note": "kernels of the timed steps: the graph launches run the ordinary path's "
                                     "kernels, counted there over the same number of steps",
                "graph_launches": int(gprof.graph_launches), "cpu_baseline": cpu,
                "last_step_reports": [(r.field_name, r.n_iterations) for r in reports],
                "simple_eager": eager_line, "simple_later": late}
        line.update(extra)
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--skip-transport", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--transport-n", type=int, default=128)
    ap.add_argument("--skip-adjoint", action="store_true")
    ap.add_argument("--skip-batch", action="store_true")
    ap.add_argument("--ref-n", type=int, default=REF_SAMPLE_N, help="cavity size of the reference arm's sample")
    ap.add_argument("--late-steps", type=int, default=175,
                    help="untimed steps before the second timing of the SIMPLE run (0: skip it)")
    args = ap.parse_args()
    world, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
