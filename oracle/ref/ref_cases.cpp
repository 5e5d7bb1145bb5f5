// extern "C" driver over the reference's own public C++ API (test
// infrastructure, compiled with the reference's sources into
// oracle/_ref/libprism_ref.so by oracle/ref_build.py).
//
// Each entry point builds a case the way the reference's tests and examples do
// (the file:line each one follows is given beside it), runs it with the
// reference's classes, and copies the results into caller buffers. Nothing here
// restates an algorithm: the arithmetic is the reference's. Errors (the
// reference throws) are caught and reported through ref_last_error().
#include <prism/prism.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <span>
#include <string>
#include <vector>

#include "prism/algorithm/PISO.h"
#include "prism/algorithm/SIMPLE.h"

using namespace prism;

namespace {
thread_local std::string g_error;

struct MeshHandle {
    SharedPtr<mesh::PMesh> mesh;
};

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    } catch (...) {
        g_error = "unknown exception";
        return 1;
    }
}

auto toVec(const double* p, size_t n) -> VectorXd {
    VectorXd v(static_cast<Eigen::Index>(n));
    for (size_t i = 0; i < n; ++i) v[static_cast<Eigen::Index>(i)] = p[i];
    return v;
}

void fromVec(const VectorXd& v, double* out) {
    for (Eigen::Index i = 0; i < v.size(); ++i) out[i] = v[i];
}

// a field::Vector / field::Velocity with per-cell components (component-major input)
template <typename V, typename Comp>
auto makeVector(const std::string& name, const SharedPtr<mesh::PMesh>& m, const double* xyz) -> SharedPtr<V> {
    const size_t n = m->cellCount();
    std::array<Comp, 3> comps {Comp(name + "_x", m, toVec(xyz, n), VectorCoord::X),
                               Comp(name + "_y", m, toVec(xyz + n, n), VectorCoord::Y),
                               Comp(name + "_z", m, toVec(xyz + 2 * n, n), VectorCoord::Z)};
    return makeShared<V>(name, m, comps);
}

// the matrix and right-hand side of an equation as CSR (rows = cells)
int64_t exportSystem(const eqn::Transport& eq, int64_t cap, int64_t* rowptr, int64_t* col, double* val,
                     double* rhs) {
    const auto& A = eq.matrix();
    const auto n = A.rows();
    std::vector<std::vector<std::pair<int64_t, double>>> rows(static_cast<size_t>(n));
    const auto* op = A.outerIndexPtr();
    const auto* ip = A.innerIndexPtr();
    const auto* vp = A.valuePtr();
    for (Eigen::Index j = 0; j < A.cols(); ++j)
        for (auto k = op[j]; k < op[j + 1]; ++k) rows[ip[k]].emplace_back(j, vp[k]);
    int64_t nnz = A.nonZeros();
    if (nnz > cap) return nnz;
    int64_t p = 0;
    rowptr[0] = 0;
    for (Eigen::Index i = 0; i < n; ++i) {
        for (auto& [j, v] : rows[i]) {
            col[p] = j;
            val[p] = v;
            ++p;
        }
        rowptr[i + 1] = p;
    }
    fromVec(eq.rhs(), rhs);
    return nnz;
}

template <typename Conv>
void addSymmetry(eqn::Momentum& e, int symmetry) {
    if (symmetry) e.boundaryHandlersManager().addHandler<eqn::boundary::Symmetry<eqn::Transport>>();
}

// MomentumEquations<Div, Corrected, Gradient<Negative>> (tests/test_utils.h:197-217)
template <typename Div>
auto momentumPair(const SharedPtr<field::Velocity>& U, const SharedPtr<field::Pressure>& p,
                  const SharedPtr<field::Scalar>& nu, const SharedPtr<field::Velocity>& mdot, int symmetry)
    -> std::vector<eqn::Momentum> {
    using namespace prism::scheme;
    using grad = source::Gradient<Sign::Negative>;
    std::vector<eqn::Momentum> eqs;
    eqs.reserve(2);
    eqs.emplace_back(Div(mdot, U->x()), diffusion::Corrected(nu, U->x()), grad(p, VectorCoord::X));
    eqs.emplace_back(Div(mdot, U->y()), diffusion::Corrected(nu, U->y()), grad(p, VectorCoord::Y));
    for (auto& e : eqs) addSymmetry<Div>(e, symmetry);
    return eqs;
}

// convection schemes by index
enum Conv { kUpwind = 0, kCentral, kLinearUpwind, kQUICK, kFROMM, kMINMOD, kMUSCL, kSMART };

template <typename F>
void withConv(int conv, F&& f) {
    using namespace prism::scheme::convection;
    switch (conv) {
        case kUpwind: f(static_cast<Upwind*>(nullptr)); break;
        case kCentral: f(static_cast<CentralDifference*>(nullptr)); break;
        case kLinearUpwind: f(static_cast<LinearUpwind*>(nullptr)); break;
        case kQUICK: f(static_cast<QUICK*>(nullptr)); break;
        case kFROMM: f(static_cast<FROMM*>(nullptr)); break;
        case kMINMOD: f(static_cast<MINMOD*>(nullptr)); break;
        case kMUSCL: f(static_cast<MUSCL*>(nullptr)); break;
        case kSMART: f(static_cast<SMART*>(nullptr)); break;
        default: throw std::invalid_argument("unknown convection scheme index");
    }
}

void writeSimpleOutputs(const SharedPtr<mesh::PMesh>& m, const SharedPtr<field::Velocity>& U,
                        const SharedPtr<field::Velocity>& mdot, const SharedPtr<field::Pressure>& p,
                        double* U_out, double* p_out, double* flux_out, double* mdot_flux_out) {
    const size_t nc = m->cellCount();
    if (U_out) {
        fromVec(U->x()->values(), U_out);
        fromVec(U->y()->values(), U_out + nc);
        fromVec(U->z()->values(), U_out + 2 * nc);
    }
    if (p_out) fromVec(p->values(), p_out);
    // faces of empty patches carry no flux (the reference has no handler for them): 0
    for (const auto& face : m->faces()) {
        if (flux_out) flux_out[face.id()] = 0.0;
        if (mdot_flux_out) mdot_flux_out[face.id()] = 0.0;
    }
    auto write = [&](std::span<const mesh::Face> faces) {
        for (const auto& face : faces) {
            if (flux_out) flux_out[face.id()] = U->fluxAtFace(face);
            if (mdot_flux_out) mdot_flux_out[face.id()] = mdot->fluxAtFace(face);
        }
    };
    write(m->nonEmptyBoundaryFaces());
    write(m->interiorFaces());
}
} // namespace

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

// UnvToPMeshConverter(mesh, fields.json).toPMesh() (mesh/unv.cpp:61-121, tests/test_utils.h:26-29)
void* ref_mesh_load(const char* unv_path, const char* fields_json) {
    MeshHandle* h = nullptr;
    int rc = guarded([&] {
        auto m = mesh::UnvToPMeshConverter(unv_path, fields_json).toPMesh();
        h = new MeshHandle {m};
    });
    return rc == 0 ? h : nullptr;
}

void ref_mesh_free(void* h) { delete static_cast<MeshHandle*>(h); }

// counts: cells, faces, boundary faces, non-empty boundary faces, interior faces, patches
int ref_mesh_sizes(void* h, int64_t* out) {
    return guarded([&] {
        const auto& m = *static_cast<MeshHandle*>(h)->mesh;
        out[0] = static_cast<int64_t>(m.cellCount());
        out[1] = static_cast<int64_t>(m.faceCount());
        out[2] = static_cast<int64_t>(m.boundaryFaces().size());
        out[3] = static_cast<int64_t>(m.nonEmptyBoundaryFaces().size());
        out[4] = static_cast<int64_t>(m.interiorFaces().size());
        out[5] = static_cast<int64_t>(m.boundaryPatches().size());
    });
}

// per face (PMesh order): owner, neighbour (-1 on the boundary), patch (-1 inside), area,
// unit normal (3 x nf, component-major), centre (3 x nf)
int ref_mesh_faces(void* h, int64_t* owner, int64_t* nbr, int64_t* patch, double* area, double* normal,
                   double* center) {
    return guarded([&] {
        const auto& m = *static_cast<MeshHandle*>(h)->mesh;
        const size_t nf = m.faceCount();
        for (size_t f = 0; f < nf; ++f) {
            const auto& face = m.faces()[f];
            owner[f] = static_cast<int64_t>(face.owner());
            nbr[f] = face.neighbor().has_value() ? static_cast<int64_t>(face.neighbor().value()) : -1;
            patch[f] = face.isBoundary() ? static_cast<int64_t>(face.boundaryPatchId().value()) : -1;
            area[f] = face.area();
            for (int d = 0; d < 3; ++d) {
                normal[d * nf + f] = face.normal()[d];
                center[d * nf + f] = face.center()[d];
            }
        }
    });
}

// per cell: centre (3 x nc) and volume
int ref_mesh_cells(void* h, double* center, double* volume) {
    return guarded([&] {
        const auto& m = *static_cast<MeshHandle*>(h)->mesh;
        const size_t nc = m.cellCount();
        for (size_t c = 0; c < nc; ++c) {
            const auto& cell = m.cells()[c];
            volume[c] = cell.volume();
            for (int d = 0; d < 3; ++d) center[d * nc + c] = cell.center()[d];
        }
    });
}

// tests/test_poisson.cpp:24-50: Corrected(c = I, P) + ConstantScalar<Positive>(S),
// S = 2 pi^2 sin(pi x) cos(pi y) at cell centres, then solveWithBiCGSTAB(eqn) =
// correctors x solve(steps, 1e-20) (tests/test_utils.h:142-151)
int ref_poisson(void* h, int correctors, int steps, double* P_out) {
    return guarded([&] {
        using namespace prism::scheme;
        auto m = static_cast<MeshHandle*>(h)->mesh;
        auto P = makeShared<field::Scalar>("P", m, 0.0);
        VectorXd src(static_cast<Eigen::Index>(m->cellCount()));
        for (const auto& cell : m->cells()) {
            double x = cell.center().x();
            double y = cell.center().y();
            src[cell.id()] = 2 * std::pow(prism::PI, 2) * std::sin(prism::PI * x) * std::cos(prism::PI * y);
        }
        auto c = makeShared<field::Tensor>("c", m, Matrix3d::Identity());
        auto S = makeShared<field::Scalar>("S", m, std::move(src));
        auto eqn = eqn::Transport(diffusion::Corrected(c, P), source::ConstantScalar<Sign::Positive>(S));
        solver::BiCGSTAB solver;
        for (int i = 0; i < correctors; ++i) solver.solve(eqn, static_cast<size_t>(steps), 1e-20);
        fromVec(P->values(), P_out);
    });
}

// tests/test_advection_1d.cpp:24-65: Upwind(U, T) + NonCorrected(kappa = 0.1, T) with U the
// inlet velocity, solveWithBiCGSTAB(eqn, 5, 5, 1e-20)
int ref_advection_1d(void* h, double* T_out) {
    return guarded([&] {
        using namespace prism::scheme;
        auto m = static_cast<MeshHandle*>(h)->mesh;
        auto T = makeShared<field::Scalar>("T", m, 0.0);
        const auto& patches = m->boundaryPatches();
        auto it = std::find_if(patches.begin(), patches.end(), [](const auto& p) { return p.name() == "Inlet"; });
        Vector3d u_in = it->getVectorBoundaryCondition("U");
        auto U = makeShared<field::Velocity>("U", m, u_in);
        auto kappa = makeShared<field::Scalar>("kappa", m, 0.1);
        auto eqn = eqn::Transport(convection::Upwind(U, T), diffusion::NonCorrected(kappa, T));
        solver::BiCGSTAB solver;
        for (int i = 0; i < 5; ++i) solver.solve(eqn, 5, 1e-20);
        fromVec(T->values(), T_out);
    });
}

// Steady scalar transport (the C1 / C3 shapes): convection `conv` with a per-cell field::Vector U
// (component-major, may be null for none) + NonCorrected (diffusion 0) or Corrected (1) with a
// uniform scalar kappa, optional ConstantScalar<Positive> source (per cell), optional face values
// of T (Scalar::setFaceValues); `outer` x solve(n_iter, eps) with BiCGSTAB (method 0) or Jacobi
// (1). If cap > 0 the equation is assembled once more at the final state (updateCoeffs) and its
// CSR matrix / rhs are returned (return value = nnz; a larger nnz than cap writes nothing).
int64_t ref_transport(void* h, int conv, const double* U, double kappa, int diffusion, const double* src,
                      const double* face_values, int outer, int n_iter, double eps, int method, double* T_out,
                      int64_t cap, int64_t* rowptr, int64_t* col, double* val, double* rhs) {
    int64_t nnz = 0;
    int rc = guarded([&] {
        using namespace prism::scheme;
        auto m = static_cast<MeshHandle*>(h)->mesh;
        const size_t nc = m->cellCount();
        auto T = makeShared<field::Scalar>("T", m, toVec(T_out, nc));
        if (face_values) T->setFaceValues(toVec(face_values, m->faceCount()));
        auto k = makeShared<field::Scalar>("kappa", m, kappa);
        SharedPtr<field::Vector> Uf;
        if (U) Uf = makeVector<field::Vector, field::Scalar>("U", m, U);
        SharedPtr<field::Scalar> S;
        if (src) S = makeShared<field::Scalar>("S", m, toVec(src, nc));
        auto run = [&](auto& eqn) {
            SharedPtr<solver::ISolver> s;
            if (method == 1) s = makeShared<solver::Jacobi>();
            else s = makeShared<solver::BiCGSTAB>();
            for (int i = 0; i < outer; ++i) s->solve(eqn, static_cast<size_t>(n_iter), eps);
            fromVec(T->values(), T_out);
            if (cap > 0) {
                eqn.updateCoeffs();
                nnz = exportSystem(eqn, cap, rowptr, col, val, rhs);
                eqn.zeroOutCoeffs();
            }
        };
        auto withDiff = [&](auto diff) {
            if (!Uf) {
                if (S) {
                    auto eqn = eqn::Transport(std::move(diff), source::ConstantScalar<Sign::Positive>(S));
                    run(eqn);
                } else {
                    auto eqn = eqn::Transport(std::move(diff));
                    run(eqn);
                }
                return;
            }
            withConv(conv, [&](auto* tag) {
                using C = std::remove_pointer_t<decltype(tag)>;
                if (S) {
                    auto eqn = eqn::Transport(C(Uf, T), std::move(diff), source::ConstantScalar<Sign::Positive>(S));
                    run(eqn);
                } else {
                    auto eqn = eqn::Transport(C(Uf, T), std::move(diff));
                    run(eqn);
                }
            });
        };
        if (diffusion == 0) withDiff(diffusion::NonCorrected(k, T));
        else withDiff(diffusion::Corrected(k, T));
    });
    return rc == 0 ? nnz : -1;
}

// SIMPLE on a case (tests/test_simple_coarse_pipe.cpp:13-50, test_simple_duct_symmetry.cpp:13-54,
// examples/SIMPLESolver/main.cpp): makePressureVelocityFields(nu), MomentumEquations<conv,
// Corrected, Gradient<Negative>>, optional Symmetry<Transport> handlers, `iters` x
// IncompressibleSIMPLE(SIMPLEControls{}).step(...). Outputs U (3 x nc), p, the cell-based face
// flux of U and the stored mass flux of mdot (per face), the reports of the last step
// (initial residual, final residual, iterations; up to 16) and needsPressureReference(p).
// `seconds` receives the wall time of each step (may be null).
int ref_simple(void* h, double nu, int conv, int symmetry, int iters, double* U_out, double* p_out,
               double* flux_out, double* mdot_flux_out, double* report_out, int* n_reports, int* needs_ref,
               double* seconds) {
    return guarded([&] {
        auto m = static_cast<MeshHandle*>(h)->mesh;
        auto U = makeShared<field::Velocity>("U", m, Vector3d {0, 0, 0});
        auto p = makeShared<field::Pressure>("P", m, 0.0);
        auto nuf = makeShared<field::Scalar>("nu", m, nu);
        auto mdot = makeShared<field::Velocity>(U->clone());
        withConv(conv, [&](auto* tag) {
            using C = std::remove_pointer_t<decltype(tag)>;
            auto eqs = momentumPair<C>(U, p, nuf, mdot, symmetry);
            std::vector<eqn::Momentum*> ptrs {&eqs[0], &eqs[1]};
            algo::SIMPLEControls controls;
            std::vector<report::Entry> reps;
            for (int it = 0; it < iters; ++it) {
                auto t0 = std::chrono::steady_clock::now();
                reps = algo::IncompressibleSIMPLE(controls).step(std::span<eqn::Momentum*>(ptrs), U, mdot, p);
                auto t1 = std::chrono::steady_clock::now();
                if (seconds) seconds[it] = std::chrono::duration<double>(t1 - t0).count();
            }
            int nr = 0;
            for (const auto& r : reps) {
                if (nr >= 16) break;
                if (report_out) {
                    report_out[3 * nr] = r.initial_residual;
                    report_out[3 * nr + 1] = r.final_residual;
                    report_out[3 * nr + 2] = static_cast<double>(r.n_iterations);
                }
                ++nr;
            }
            if (n_reports) *n_reports = nr;
        });
        writeSimpleOutputs(m, U, mdot, p, U_out, p_out, flux_out, mdot_flux_out);
        if (needs_ref) *needs_ref = algo::needsPressureReference(p) ? 1 : 0;
    });
}

} // extern "C"
