"""Case builders shared by the tests: the reference's own test cases (from the
golden fixtures) and the synthetic configurations, built on any library that
exposes the C-ABI (the sm_100a library or the CPU oracle)."""
import json
import os

import numpy as np

from prism_b200 import _abi as A
from prism_b200 import api, io, meshgen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# ---------------------------------------------------------------- golden cases
def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    goff = z["group_offsets"]
    gel = z["group_elements"].astype(np.int64)
    groups = [(g, bool(z["group_is_vertex"][i]), gel[goff[i]:goff[i + 1]])
              for i, g in enumerate(meta["groups"])]
    unv = io.UnvData(z["xyz"], z["elem_kind"].astype(np.int32), z["elem_offsets"].astype(np.int64),
                     z["elem_nodes"].astype(np.int64), groups)
    case = io.case_from_docs(meta["fields"], meta["docs"])
    extra = {k: z[k] for k in z.files if k.startswith("foam_")}
    return unv, case, extra


def load_oracle_results(name):
    z = np.load(os.path.join(GOLDEN, name + "_oracle.npz"))
    return {k: z[k] for k in z.files}


def rel_l2(x, ref):
    return float(np.linalg.norm(x - ref) / np.linalg.norm(ref))


def poisson_reference(unv, case, lib, solver=None, correctors=5, steps=15):
    """tests/test_poisson.cpp:24-50: Corrected(c = I, P) + ConstantScalar(S), 5 x solve(15, 1e-20)."""
    mesh = api.Mesh(unv, case, lib=lib)
    cc = mesh.export()["cell_center"]
    P = api.Scalar("P", mesh, 0.0)
    S = api.Scalar("S", mesh, 2 * np.pi ** 2 * np.sin(np.pi * cc[0]) * np.cos(np.pi * cc[1]))
    c = api.Tensor("c", mesh, np.eye(3))
    eqn = api.Transport(api.diffusion.Corrected(c, P), api.source.ConstantScalar(S))
    solver = solver or api.BiCGSTAB()
    for _ in range(correctors):
        solver.solve(eqn, steps, 1e-20)
    exact = np.sin(np.pi * cc[0]) * np.cos(np.pi * cc[1])
    x = P.values()
    return {"P": x, "rel_l2": np.array(rel_l2(x, exact))}


def advection_reference(unv, case, lib, solver=None):
    """tests/test_advection_1d.cpp:24-65: Upwind(U, T) + NonCorrected(0.1, T), 5 x solve(5, 1e-20)."""
    mesh = api.Mesh(unv, case, lib=lib)
    cc = mesh.export()["cell_center"]
    T = api.Scalar("T", mesh, 0.0)
    pi = case.patch_names.index("Inlet")
    uin = case.fields["U"][pi].vector
    U = api.Vector("U", mesh, uin)
    kappa = api.Scalar("kappa", mesh, 0.1)
    eqn = api.Transport(api.convection.Upwind(U, T), api.diffusion.NonCorrected(kappa, T))
    solver = solver or api.BiCGSTAB()
    for _ in range(5):
        solver.solve(eqn, 5, 1e-20)
    u = uin[0]
    exact = -((np.exp(u * cc[0] / 0.1) - 1) / (np.exp(u / 0.1) - 1)) + 1
    x = T.values()
    return {"T": x, "diff_norm": np.array(np.linalg.norm(x - exact))}


def transient_exact(x, t, kappa, modes=100):
    """The series solution the reference's transient test compares with
    (tests/test_transient_1d.cpp:14-26)."""
    s = np.zeros_like(x)
    for n in range(modes):
        lam = ((2 * n) - 1) * np.pi / 2
        v = ((-1.0) ** (n + 1)) * np.exp(-kappa * t * lam ** 2) * np.cos(lam * x) / ((2 * n) - 1)
        s = s + v
    return s * (4.0 / np.pi) * 100


def transient_reference(unv, case, lib, solver=None, steps=200, dt=2.0):
    """tests/test_transient_1d.cpp:29-83: T = 200 with a 2-step history, AdamMoulton(T, dt) +
    Corrected(1e-3, T); per time step solve(10, 1e-20) then updatePrevTimeSteps. Returns the
    final field and the relative L2 errors against the series at t = 40, 60 and at the end."""
    mesh = api.Mesh(unv, case, lib=lib)
    x = mesh.export()["cell_center"][0]
    T = api.Scalar("T", mesh, 200.0)
    T.set_history_size(2)
    T.update_prev_time_steps()
    kappa = 1e-3
    k = api.Scalar("kappa", mesh, kappa)
    eqn = api.Transport(api.temporal.AdamMoulton(T, dt), api.diffusion.Corrected(k, T))
    solver = solver or api.BiCGSTAB()
    norms, final = [], None
    for step in range(steps):
        solver.solve(eqn, 10, 1e-20)
        exact = transient_exact(x, dt * step, kappa)
        err = float(np.linalg.norm(T.values() - exact) / np.linalg.norm(exact))
        if dt * step in (40, 60):
            norms.append(err)
        final = err
        T.update_prev_time_steps()
    return {"T": T.values(), "diff_norms": np.array(norms), "final_diff_norm": np.array(final)}


def simple_fields(mesh, nu=1e-3):
    """makePressureVelocityFields (tests/test_utils.h:176-195)."""
    U = api.Vector("U", mesh, (0.0, 0.0, 0.0))
    p = api.Scalar("P", mesh, 0.0)
    nuf = api.Scalar("nu", mesh, nu)
    mdot = U.clone()
    return U, p, nuf, mdot


def momentum_eqns(U, p, nu, mdot, conv="LinearUpwind", symmetry=False, n=2):
    """MomentumEquations<div, Corrected, Gradient<Negative>> (tests/test_utils.h:197-217)."""
    eqs = []
    comps = [U.x(), U.y(), U.z()]
    for k in range(n):
        e = api.Transport(getattr(api.convection, conv)(mdot, comps[k]),
                          api.diffusion.Corrected(nu, comps[k]),
                          api.source.Gradient(p, k, A.SIGN_NEGATIVE))
        if symmetry:
            e.add_symmetry_handler()
        eqs.append(e)
    return eqs


def simple_reference(unv, case, lib, iters=100, symmetry=False, nu=1e-3, solver=None):
    """tests/test_simple_coarse_pipe.cpp / test_simple_duct_symmetry.cpp: SIMPLE x iters."""
    mesh = api.Mesh(unv, case, lib=lib)
    U, p, nuf, mdot = simple_fields(mesh, nu)
    eqs = momentum_eqns(U, p, nuf, mdot, symmetry=symmetry)
    simple = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=solver)
    reps = []
    for _ in range(iters):
        reps = simple.step(eqs, U, mdot, p)
    flux = U.face_flux()
    ex = mesh.export()
    pfo, pf = ex["patch_face_offsets"], ex["patch_faces"]
    rates = {}
    for i, name in enumerate(case.patch_names):
        rates[name] = float(flux[pf[pfo[i]:pfo[i + 1]]].sum())
    return {"p": p.values(), "U": U.values(), "mdot_flux": mdot.face_flux(),
            "rates": np.array([rates[n] for n in case.patch_names]),
            "needs_ref": np.array(api.needs_pressure_reference(p)),
            "last_report_iters": np.array([r.n_iterations for r in reps])}


def run_reference_test(name, lib, solver=None):
    unv, case, extra = load_golden(name)
    if name.startswith("poisson"):
        return poisson_reference(unv, case, lib, solver)
    if name == "versteeg_advection_1d":
        return advection_reference(unv, case, lib, solver)
    if name == "coarse_pipe":
        return simple_reference(unv, case, lib, 100, solver=solver)
    if name == "cavity_hex":
        return simple_reference(unv, case, lib, 20, nu=0.01, solver=solver)
    if name == "duct_simple":
        return simple_reference(unv, case, lib, 100, symmetry=True, solver=solver)
    if name == "versteeg_trans_1d":
        return transient_reference(unv, case, lib, solver=solver)
    raise KeyError(name)


# ---------------------------------------------------------------- synthetic configurations
def box_case(bcs, fields_info=None):
    """Case over the box patches; bcs: field -> {patch: (kind, value)} (missing -> zero-gradient)."""
    fields = {}
    for f, per in bcs.items():
        fields[f] = {p: per.get(p, ("zero-gradient", None)) for p in meshgen.PATCHES}
    return io.Case.from_dict(meshgen.PATCHES, fields, fields_info)


def poisson_c1(n, lib, nz=1, lengths=(1.0, 1.0, 0.01)):
    """-div(grad P) = 2 pi^2 sin(pi x) cos(pi y) on an n x n x nz box; Fixed P = exact on the
    four side walls (face values), symmetry front/back; NonCorrected, kappa = 1."""
    unv = meshgen.box_hex(n, n, nz, lengths)
    case = box_case({"P": {"left": ("fixed", 0.0), "right": ("fixed", 0.0), "bottom": ("fixed", 0.0),
                           "top": ("fixed", 0.0), "back": ("symmetry", None), "front": ("symmetry", None)}})
    mesh = api.Mesh(unv, case, lib=lib)
    ex = mesh.export()
    cc, fc = ex["cell_center"], ex["face_center"]
    P = api.Scalar("P", mesh, 0.0)
    P.set_face_values(np.sin(np.pi * fc[0]) * np.cos(np.pi * fc[1]))
    S = api.Scalar("S", mesh, 2 * np.pi ** 2 * np.sin(np.pi * cc[0]) * np.cos(np.pi * cc[1]))
    kappa = api.Scalar("kappa", mesh, 1.0)
    eqn = api.Transport(api.diffusion.NonCorrected(kappa, P), api.source.ConstantScalar(S))
    return mesh, P, eqn, np.sin(np.pi * cc[0]) * np.cos(np.pi * cc[1])


def cavity(n, lib, nu=0.01, conv="Upwind"):
    """Lid-driven cavity on n x n x 1 hexes: lid (top) fixed [1,0,0], other walls no-slip,
    front/back empty, P zero-gradient everywhere (auto reference cell 0)."""
    unv = meshgen.box_hex(n, n, 1, (1.0, 1.0, 1.0 / n))
    wall = ("no-slip", [0.0, 0.0, 0.0])
    case = box_case({"U": {"top": ("fixed", [1.0, 0.0, 0.0]), "left": wall, "right": wall, "bottom": wall,
                           "back": ("empty", None), "front": ("empty", None)},
                     "P": {"back": ("empty", None), "front": ("empty", None)}})
    mesh = api.Mesh(unv, case, lib=lib)
    U, p, nuf, mdot = simple_fields(mesh, nu)
    eqs = momentum_eqns(U, p, nuf, mdot, conv=conv)
    return mesh, U, p, nuf, mdot, eqs


def transport_c3(n, lib, conv="MUSCL", jitter=0.2, seed=3, kappa=1e-3):
    """div(U T) - div(kappa grad T) = 0 on a jittered n^3 box, U = (sin pi x cos pi y,
    -cos pi x sin pi y, 0) at cell centroids; T fixed 1 at x=0 and 0 at x=1, zero-gradient
    elsewhere; Corrected diffusion; Green-Gauss gradients."""
    unv = meshgen.box_hex(n, n, n, jitter=jitter, seed=seed)
    case = box_case({"T": {"left": ("fixed", 1.0), "right": ("fixed", 0.0)}, "U": {}},
                    {"T": {"gradScheme": "greenGauss"}, "U": {}})
    mesh = api.Mesh(unv, case, lib=lib)
    cc = mesh.export()["cell_center"]
    Uv = np.stack([np.sin(np.pi * cc[0]) * np.cos(np.pi * cc[1]),
                   -np.cos(np.pi * cc[0]) * np.sin(np.pi * cc[1]), np.zeros(mesh.n_cells)])
    U = api.Vector("U", mesh, Uv)
    T = api.Scalar("T", mesh, 0.0)
    k = api.Scalar("kappa", mesh, kappa)
    eqn = api.Transport(getattr(api.convection, conv)(U, T), api.diffusion.Corrected(k, T))
    return mesh, T, U, eqn


def adjoint_c5(n, lib, seed=5, corrected=True):
    """Steady diffusion for the adjoint: n^3 unit cubes x 6 tets (Kuhn split) on the unit cube,
    kappa ~ lognormal(0, 0.5) per cell, T Fixed on all six walls with face values ~ U(0, 1) per
    boundary face, target T* ~ N(0, 1) per cell; Corrected (or NonCorrected) diffusion with the
    least-squares gradient. J = sum_c V_c (T_c - T*_c)^2.
    Returns dict(mesh, T, kappa, eqn, kappa0, v0, T_star, vol)."""
    unv = meshgen.box_tet(n, n, n)
    case = box_case({"T": {p: ("fixed", 0.0) for p in meshgen.PATCHES}})
    mesh = api.Mesh(unv, case, lib=lib)
    rng = np.random.default_rng(seed)
    nc, nb = mesh.n_cells, mesh.info.n_boundary_faces
    kappa0 = rng.lognormal(0.0, 0.5, nc)
    v0 = rng.uniform(0.0, 1.0, nb)
    T_star = rng.normal(0.0, 1.0, nc)
    T = api.Scalar("T", mesh, 0.0)
    fv = np.zeros(mesh.n_faces)
    fv[:nb] = v0
    T.set_face_values(fv)
    kappa = api.Scalar("kappa", mesh, kappa0)
    scheme = api.diffusion.Corrected if corrected else api.diffusion.NonCorrected
    eqn = api.Transport(scheme(kappa, T))
    vol = mesh.export()["cell_volume"]
    return dict(mesh=mesh, T=T, kappa=kappa, eqn=eqn, kappa0=kappa0, v0=v0, T_star=T_star, vol=vol)


def objective(T, T_star, vol):
    """J = sum_c V_c (T_c - T*_c)^2 and dJ/dT."""
    r = T - T_star
    return float(np.sum(vol * r * r)), 2.0 * vol * r


def batch_sizes(count, seed=4, nmin=16, nmax=96):
    """Per-problem cube edge counts N = round(exp(U(ln nmin, ln nmax))) (seeded)."""
    rng = np.random.default_rng(seed)
    return [int(round(float(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))) for _ in range(count)]


def diffusion_box(N, lib, seed):
    """One batched problem: N^3 unit-cube hexes, kappa ~ lognormal(0, 1) per cell, f ~ N(0, 1) per
    cell as ConstantScalar, T Fixed 0 on all walls, Corrected diffusion."""
    unv = meshgen.box_hex(N, N, N)
    case = box_case({"T": {p: ("fixed", 0.0) for p in meshgen.PATCHES}})
    mesh = api.Mesh(unv, case, lib=lib)
    rng = np.random.default_rng(seed)
    kappa = api.Scalar("kappa", mesh, rng.lognormal(0.0, 1.0, mesh.n_cells))
    f = api.Scalar("f", mesh, rng.normal(0.0, 1.0, mesh.n_cells))
    T = api.Scalar("T", mesh, 0.0)
    eqn = api.Transport(api.diffusion.Corrected(kappa, T), api.source.ConstantScalar(f))
    return dict(mesh=mesh, T=T, kappa=kappa, f=f, eqn=eqn)
