"""AMG-preconditioned BiCGSTAB (and flexible CG for the pressure correction) on the GPU vs the oracle.

The preconditioner changes only the path to the solution: every solved field
must agree with the oracle (ILUT-BiCGSTAB to machine precision) within 1e-8
relative L2, as with the Jacobi-preconditioned solver. Iteration counts are
printed and must drop against the Jacobi preconditioner."""
import numpy as np
import pytest

from prism_b200 import _abi as A
from prism_b200 import PrismError, api
from tests import cases
from tests.test_oracle_pins import _tridiag

pytestmark = pytest.mark.gpu
SOL_TOL = 1e-8


def _transport(lib, n, solver):
    mesh, T, U, eqn = cases.transport_c3(n, lib, conv="LinearUpwind")
    r = solver.solve(eqn, 1, 0.0)
    return T.values(), r


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
@pytest.mark.parametrize("n", [16, 24])
def test_transport_amg(gpu, orc, precision, n):
    ref, _ = _transport(orc, n, api.BiCGSTAB())
    got, r = _transport(gpu, n, api.BiCGSTAB(precision=precision, krylov_tol=1e-12, preconditioner="amg"))
    _, rj = _transport(gpu, n, api.BiCGSTAB(precision=precision, krylov_tol=1e-12, preconditioner="jacobi"))
    err = cases.rel_l2(got, ref)
    print(f"transport {n}^3 precision={precision}: AMG rel L2 vs oracle {err:.3e}, "
          f"krylov it AMG {r.krylov_iterations} vs Jacobi {rj.krylov_iterations}")
    assert r.status == A.OK
    assert err < SOL_TOL
    assert r.krylov_iterations < rj.krylov_iterations


def test_transport_auto_selects_amg(gpu, orc):
    # 32^3 rows reach the automatic AMG threshold
    n = 32
    assert n ** 3 >= A.PC_AUTO_MIN_ROWS
    ref, _ = _transport(orc, n, api.BiCGSTAB())
    got, r = _transport(gpu, n, api.BiCGSTAB(krylov_tol=1e-12))
    _, ra = _transport(gpu, n, api.BiCGSTAB(krylov_tol=1e-12, preconditioner="amg"))
    err = cases.rel_l2(got, ref)
    print(f"transport 32^3 auto: rel L2 {err:.3e}, krylov it {r.krylov_iterations} (amg {ra.krylov_iterations})")
    assert err < SOL_TOL
    assert r.krylov_iterations == ra.krylov_iterations


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
def test_poisson_c1_amg(gpu, orc, precision):
    res = {}
    for name, lib, solver in (("gpu", gpu, api.BiCGSTAB(precision=precision, preconditioner="amg")),
                              ("orc", orc, api.BiCGSTAB())):
        mesh, P, eqn, exact = cases.poisson_c1(64, lib)
        r = solver.solve(eqn, 3, 1e-10)
        res[name] = (P.values(), r)
    err = cases.rel_l2(res["gpu"][0], res["orc"][0])
    print(f"C1 64x64 AMG precision={precision}: rel L2 vs oracle {err:.3e}, "
          f"krylov it {res['gpu'][1].krylov_iterations}")
    assert err < SOL_TOL
    assert res["gpu"][1].converged


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
def test_cavity_simple_amg(gpu, orc, precision):
    # the pressure-correction hierarchy is built once and refreshed every step
    out = {}
    for name, lib in (("gpu", gpu), ("orc", orc)):
        mesh, U, p, nu, mdot, eqs = cases.cavity(24, lib)
        solver = (api.BiCGSTAB(precision=precision, preconditioner="amg") if name == "gpu"
                  else api.BiCGSTAB())
        simple = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=solver)
        for _ in range(8):
            simple.step(eqs, U, mdot, p)
        out[name] = (U.values(), p.values(), mdot.face_flux())
    for i, k in enumerate(("U", "p", "mdot")):
        err = cases.rel_l2(out["gpu"][i], out["orc"][i])
        print(f"cavity 24x24 AMG precision={precision} {k}: rel L2 vs oracle {err:.3e}")
        assert err < SOL_TOL


_CAVITY160 = {}


def _cavity160(lib, solver, steps=3):
    mesh, U, p, nu, mdot, eqs = cases.cavity(160, lib)
    simple = api.IncompressibleSIMPLE(api.SIMPLEControls(), solver=solver)
    for _ in range(steps):
        simple.step(eqs, U, mdot, p)
    return U.values(), p.values(), mdot.face_flux()


@pytest.mark.parametrize("kcycle", [None, "1"])
def test_cavity_simple_flexible_cg(gpu, orc, kcycle, monkeypatch):
    """The FP64 pressure correction at AMG sizes runs flexible CG: preconditioned by an
    FP32 V-cycle by default, by the FP64 K-cycle with PRISM_AMG_KCYCLE=1 (160 x 160:
    level 1 has 5,000+ rows and lies above the fused tail, so it is a K level)."""
    if kcycle:
        monkeypatch.setenv("PRISM_AMG_KCYCLE", kcycle)
    got = _cavity160(gpu, api.BiCGSTAB(preconditioner="amg"))
    if "orc" not in _CAVITY160:
        _CAVITY160["orc"] = _cavity160(orc, api.BiCGSTAB())
    for i, k in enumerate(("U", "p", "mdot")):
        err = cases.rel_l2(got[i], _CAVITY160["orc"][i])
        print(f"cavity 160x160, 3 SIMPLE iterations, K-cycle levels {kcycle or 0} {k}: rel L2 vs oracle {err:.3e}")
        assert err < SOL_TOL


def _laplacian_2d(m, neumann, shift=0.0, conv=0.0):
    """Five-point operator on an m x m grid, row-major CSR with sorted columns:
    Neumann walls (singular for shift = 0) or Dirichlet walls; conv adds an
    upwind x-convection term (nonsymmetric)."""
    n = m * m
    rows = []
    for i in range(m):
        for j in range(m):
            r = i * m + j
            ent = {r: shift}
            for di, dj in ((-1, 0), (0, -1), (0, 1), (1, 0)):
                ii, jj = i + di, j + dj
                if 0 <= ii < m and 0 <= jj < m:
                    c = ii * m + jj
                    ent[r] += 1.0
                    ent[c] = ent.get(c, 0.0) - 1.0
                elif not neumann:
                    ent[r] += 2.0
            if conv and j > 0:
                ent[r] += conv
                ent[r - 1] -= conv
            rows.append(sorted(ent.items()))
    rp = np.zeros(n + 1, np.int64)
    col, val = [], []
    for r, ent in enumerate(rows):
        rp[r + 1] = rp[r] + len(ent)
        col += [c for c, _ in ent]
        val += [v for _, v in ent]
    return rp, np.array(col, np.int64), np.array(val)


def _dense(rp, col, val):
    n = len(rp) - 1
    M = np.zeros((n, n))
    for r in range(n):
        M[r, col[rp[r]:rp[r + 1]]] += val[rp[r]:rp[r + 1]]
    return M


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
@pytest.mark.parametrize("kind", ["dirichlet", "nonsymmetric", "neumann"])
def test_solve_csr_amg(gpu, precision, kind):
    m = 48
    rp, col, val = _laplacian_2d(m, neumann=(kind == "neumann"), conv=(3.0 if kind == "nonsymmetric" else 0.0))
    M = _dense(rp, col, val)
    rng = np.random.default_rng(5)
    x_true = rng.normal(size=m * m)
    if kind == "neumann":
        x_true -= x_true.mean()
    b = M @ x_true  # consistent also for the singular Neumann operator
    x = api.BiCGSTAB(precision=precision, krylov_tol=1e-12, preconditioner="amg").step(
        gpu, rp, col, val, np.zeros(m * m), b)
    res = np.linalg.norm(M @ x - b) / np.linalg.norm(b)
    print(f"solve_csr AMG {kind} precision={precision}: rel residual {res:.3e}")
    assert res < 1e-10
    if kind != "neumann":
        assert np.linalg.norm(x - x_true) / np.linalg.norm(x_true) < 1e-8


def test_tridiagonal_single_level(gpu):
    # 10 rows: the hierarchy is one dense level and one step solves exactly
    rp, col, val, b, x_exact = _tridiag()
    x = api.BiCGSTAB(preconditioner="amg").step(gpu, rp, col, val, np.zeros(10), b)
    assert np.linalg.norm(x - x_exact) / np.linalg.norm(x_exact) < 1e-4
    M = _dense(rp, col, val)
    assert np.linalg.norm(M @ x - b) / np.linalg.norm(b) < 1e-12


def test_bad_preconditioner_rejected(gpu):
    rp, col, val, b, _ = _tridiag()
    with pytest.raises(PrismError):
        api.BiCGSTAB(preconditioner=7).step(gpu, rp, col, val, np.zeros(10), b)
