// prism_b200.hpp -- C++20 mirror of Prism's operator API over the C-ABI.
//
// Header-only. The class names, constructor arguments and method names follow
// the reference (namespace prism_b200 mirrors prism::):
//   mesh::PMesh                    <- UnvToPMeshConverter(...).toPMesh() (mesh/unv.h:21-73)
//   field::Scalar / Vector / Tensor (field/scalar.h, field/vector.h, field/tensor.h)
//   scheme::convection::Upwind ... SMART, scheme::diffusion::NonCorrected / Corrected,
//   scheme::source::ConstantScalar / Divergence / Gradient
//   eqn::Transport(schemes...)     (equation/transport.h:27-97)
//   solver::BiCGSTAB / Jacobi ::solve(eqn, n_iter, eps, ref_cell, ref_value, clear_coeffs)
//                                  (numerics/solver.h:43-49)
//   algo::IncompressibleSIMPLE / PRIME / PISO ::step(momentum, U, mdot, p)
//                                  (algorithm/algorithm.h:11-24)
// Ownership is shared_ptr-based like the reference; failures throw
// std::runtime_error carrying the C-ABI status text, as the reference throws
// std::runtime_error / error::NonImplementedBoundaryCondition / error::InvalidMesh.
#pragma once

#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "prism_b200.h"

namespace prism_b200 {

inline void check(int status) {
    if (status != PRISM_OK)
        throw std::runtime_error(std::string(prism_status_string(status)) + ": " + prism_last_error());
}

namespace mesh {
// Boundary patch as read from fields.json: name, "empty" flag.
struct PatchInfo {
    std::string name;
    bool empty = false;
};
// A mesh as UnvToPMeshConverter reads it (nodes, element list, element groups).
struct UnvMesh {
    std::vector<double> xyz;
    std::vector<int32_t> elem_kind;
    std::vector<int64_t> elem_offsets{0};
    std::vector<int64_t> elem_nodes;
    struct Group {
        std::string name;
        bool vertex = false;
        std::vector<int64_t> elements;
    };
    std::vector<Group> groups;
};

class PMesh {
  public:
    PMesh(const UnvMesh& unv, const std::vector<PatchInfo>& patches) {
        std::vector<const char*> gn, pn;
        std::vector<int32_t> gv, pe;
        std::vector<int64_t> go{0}, ge;
        for (auto& g : unv.groups) {
            gn.push_back(g.name.c_str());
            gv.push_back(g.vertex ? 1 : 0);
            ge.insert(ge.end(), g.elements.begin(), g.elements.end());
            go.push_back((int64_t)ge.size());
        }
        for (auto& p : patches) {
            pn.push_back(p.name.c_str());
            pe.push_back(p.empty ? 1 : 0);
        }
        PrismUnvMesh d{};
        d.n_nodes = (int64_t)unv.xyz.size() / 3;
        d.xyz = unv.xyz.data();
        d.n_elements = (int64_t)unv.elem_kind.size();
        d.elem_kind = unv.elem_kind.data();
        d.elem_offsets = unv.elem_offsets.data();
        d.elem_nodes = unv.elem_nodes.data();
        d.n_groups = (int32_t)gn.size();
        d.group_names = gn.data();
        d.group_is_vertex = gv.data();
        d.group_offsets = go.data();
        d.group_elements = ge.data();
        d.n_patches = (int32_t)pn.size();
        d.patch_names = pn.data();
        d.patch_is_empty = pe.data();
        PrismMesh* h = nullptr;
        check(prism_mesh_from_unv(&d, &h));
        _h.reset(h, [](PrismMesh* m) { prism_mesh_destroy(m); });
        check(prism_mesh_info(h, &_info));
    }
    auto cellCount() const -> size_t { return (size_t)_info.n_cells; }
    auto faceCount() const -> size_t { return (size_t)_info.n_faces; }
    auto boundaryFaceCount() const -> size_t { return (size_t)_info.n_boundary_faces; }
    auto patchCount() const -> size_t { return (size_t)_info.n_patches; }
    auto vertexCount() const -> size_t { return (size_t)_info.n_vertices; }
    // mesh::CuthillMckee(mesh).reorder(reverse) (reorder.cpp:8-130); before any field exists
    void reorder(bool reverse = false) { check(prism_mesh_reorder(_h.get(), reverse ? 1 : 0)); }
    auto handle() const -> PrismMesh* { return _h.get(); }
    // output::cellToPoint (export.cpp:73-111): interleaved cell data -> interleaved vertex data
    auto cellToPoint(const std::vector<double>& cell_data, size_t n_components) const -> std::vector<double> {
        std::vector<double> out(vertexCount() * n_components);
        check(prism_cell_to_point(_h.get(), cell_data.data(), (int32_t)n_components, out.data()));
        return out;
    }

  private:
    std::shared_ptr<PrismMesh> _h;
    PrismMeshInfo _info{};
};
}  // namespace mesh

namespace field {
using BC = PrismBC;

class Scalar {
  public:
    Scalar(const std::string& name, const std::shared_ptr<mesh::PMesh>& mesh, double value,
           const std::vector<BC>& bcs, int grad_scheme = PRISM_GRAD_LEAST_SQUARES)
        : _mesh(mesh), _name(name) {
        std::vector<double> v(mesh->cellCount(), value);
        create(v, bcs, grad_scheme);
    }
    Scalar(const std::string& name, const std::shared_ptr<mesh::PMesh>& mesh, const std::vector<double>& values,
           const std::vector<BC>& bcs, int grad_scheme = PRISM_GRAD_LEAST_SQUARES)
        : _mesh(mesh), _name(name) {
        create(values, bcs, grad_scheme);
    }
    // borrowed component of a Vector
    Scalar(PrismScalar* borrowed, std::shared_ptr<void> owner, std::shared_ptr<mesh::PMesh> mesh, std::string name)
        : _mesh(std::move(mesh)), _name(std::move(name)), _owner(std::move(owner)) {
        _h.reset(borrowed, [](PrismScalar*) {});
    }
    // a scalar the library created (ops::div, monitor::courantNumber): owned
    static auto adopt(PrismScalar* owned, std::shared_ptr<mesh::PMesh> mesh, std::string name) -> Scalar {
        Scalar s(owned, nullptr, std::move(mesh), std::move(name));
        s._h.reset(owned, [](PrismScalar* p) { prism_scalar_destroy(p); });
        return s;
    }
    // cellToPoint of the cell values: one value per mesh vertex
    auto toPoints() const -> std::vector<double> {
        std::vector<double> v(_mesh->vertexCount());
        check(prism_scalar_to_points(_h.get(), v.data()));
        return v;
    }
    auto name() const -> const std::string& { return _name; }
    auto values() const -> std::vector<double> {
        std::vector<double> v(_mesh->cellCount());
        check(prism_scalar_get_values(_h.get(), v.data()));
        return v;
    }
    // Scalar::update (scalar.cpp:311-320): history push, new values, face values cleared
    void update(const std::vector<double>& v) { check(prism_scalar_update(_h.get(), v.data())); }
    // time-step history (field/history.cpp)
    void setHistorySize(size_t n) { check(prism_scalar_set_history_size(_h.get(), (int32_t)n)); }
    void updatePrevTimeSteps() { check(prism_scalar_update_prev_time_steps(_h.get())); }
    auto getHistory(size_t index) const -> std::optional<std::vector<double>> {
        std::vector<double> v(_mesh->cellCount());
        int32_t ok = 0;
        check(prism_scalar_history(_h.get(), (int32_t)index, v.data(), &ok));
        if (!ok) return std::nullopt;
        return v;
    }
    auto prevValues() const { return getHistory(0); }
    auto prevPrevValues() const { return getHistory(1); }
    void setFaceValues(const std::vector<double>& fv) { check(prism_scalar_set_face_values(_h.get(), fv.data())); }
    void clearFaceValues() { check(prism_scalar_set_face_values(_h.get(), nullptr)); }
    // Scalar::setGradScheme (scalar.cpp:252-258) by kind (PRISM_GRAD_*)
    void setGradScheme(int grad_scheme) { check(prism_scalar_set_grad_scheme(_h.get(), grad_scheme)); }
    auto handle() const -> PrismScalar* { return _h.get(); }
    auto mesh() const -> const std::shared_ptr<mesh::PMesh>& { return _mesh; }

  private:
    void create(const std::vector<double>& v, const std::vector<BC>& bcs, int gs) {
        PrismScalar* h = nullptr;
        check(prism_scalar_create(_mesh->handle(), _name.c_str(), v.data(), gs, bcs.data(), &h));
        _h.reset(h, [](PrismScalar* s) { prism_scalar_destroy(s); });
    }
    std::shared_ptr<mesh::PMesh> _mesh;
    std::string _name;
    std::shared_ptr<void> _owner;
    std::shared_ptr<PrismScalar> _h;
};

class Vector : public std::enable_shared_from_this<Vector> {
  public:
    Vector(const std::string& name, const std::shared_ptr<mesh::PMesh>& mesh, const double value[3],
           const std::vector<BC>& bcs, int grad_scheme = PRISM_GRAD_LEAST_SQUARES)
        : _mesh(mesh), _name(name) {
        size_t n = mesh->cellCount();
        std::vector<double> v(3 * n);
        for (int k = 0; k < 3; ++k)
            for (size_t c = 0; c < n; ++c) v[k * n + c] = value[k];
        PrismVector* h = nullptr;
        check(prism_vector_create(mesh->handle(), name.c_str(), v.data(), grad_scheme, bcs.data(), &h));
        _h.reset(h, [](PrismVector* p) { prism_vector_destroy(p); });
    }
    auto clone() const -> std::shared_ptr<Vector> {
        PrismVector* h = nullptr;
        check(prism_vector_clone(_h.get(), &h));
        return std::shared_ptr<Vector>(new Vector(_mesh, _name, h));
    }
    auto x() { return component(0); }
    auto y() { return component(1); }
    auto z() { return component(2); }
    auto name() const -> const std::string& { return _name; }
    auto mesh() const -> const std::shared_ptr<mesh::PMesh>& { return _mesh; }
    auto handle() const -> PrismVector* { return _h.get(); }
    // setFaceFluxValues (vector.h:359-377)
    void setFaceFluxValues(const std::vector<double>& flux) {
        check(prism_vector_set_face_flux(_h.get(), flux.data()));
    }
    // fluxAtFace for every face (empty-patch faces 0)
    auto faceFlux() const -> std::vector<double> {
        std::vector<double> f(_mesh->faceCount());
        check(prism_vector_face_flux(_h.get(), f.data()));
        return f;
    }
    // cellToPoint of the cell values, x,y,z interleaved per vertex
    auto toPoints() const -> std::vector<double> {
        std::vector<double> v(3 * _mesh->vertexCount());
        check(prism_vector_to_points(_h.get(), v.data()));
        return v;
    }

  private:
    Vector(std::shared_ptr<mesh::PMesh> mesh, std::string name, PrismVector* h) : _mesh(std::move(mesh)), _name(std::move(name)) {
        _h.reset(h, [](PrismVector* p) { prism_vector_destroy(p); });
    }
    auto component(int k) -> std::shared_ptr<Scalar> {
        PrismScalar* c = nullptr;
        check(prism_vector_component(_h.get(), k, &c));
        static const char* suf[3] = {"_x", "_y", "_z"};
        return std::make_shared<Scalar>(c, std::static_pointer_cast<void>(_h), _mesh, _name + suf[k]);
    }
    std::shared_ptr<mesh::PMesh> _mesh;
    std::string _name;
    std::shared_ptr<PrismVector> _h;
};
using Velocity = Vector;
using Pressure = Scalar;

class Tensor {
  public:
    // values: 9 blocks of n cell values (block 3i+j = T(i,j)); empty = identity
    Tensor(const std::string& name, const std::shared_ptr<mesh::PMesh>& mesh, const std::vector<double>& values = {}) {
        PrismTensor* h = nullptr;
        check(prism_tensor_create(mesh->handle(), name.c_str(), values.empty() ? nullptr : values.data(), &h));
        _h.reset(h, [](PrismTensor* t) { prism_tensor_destroy(t); });
    }
    auto handle() const -> PrismTensor* { return _h.get(); }

  private:
    std::shared_ptr<PrismTensor> _h;
};
}  // namespace field

namespace ops {
// ops::div (operations/operations.h:84-100): "div(<name>)" = signed flux sum / volume
inline auto div(const field::Vector& U) -> field::Scalar {
    PrismScalar* h = nullptr;
    check(prism_ops_div(U.handle(), &h));
    return field::Scalar::adopt(h, U.mesh(), "div(" + U.name() + ")");
}
// mdot.mapFaceValues(U.valueAtFace); mdot.mapInteriorFaceValues(rhieChowCorrectFace)
// (SIMPLE.cpp:136-138, operations/rhie_chow.h:47-63)
inline void rhieChowFaces(field::Vector& mdot, const field::Vector& U, const field::Tensor& D, field::Scalar& p) {
    check(prism_rhie_chow(mdot.handle(), U.handle(), D.handle(), p.handle()));
}
}  // namespace ops

namespace monitor {
// monitor::courantNumber (monitor/courant.cpp:7-24): "Co" = 0.5 dt sum|flux| / volume
inline auto courantNumber(const field::Vector& mdot, double dt) -> field::Scalar {
    PrismScalar* h = nullptr;
    check(prism_courant_number(mdot.handle(), dt, &h));
    return field::Scalar::adopt(h, mdot.mesh(), "Co");
}
}  // namespace monitor

namespace scheme {
namespace convection {
template <int Code>
struct Scheme {
    Scheme(std::shared_ptr<field::Vector> U, std::shared_ptr<field::Scalar> phi) : U(std::move(U)), phi(std::move(phi)) {}
    std::shared_ptr<field::Vector> U;
    std::shared_ptr<field::Scalar> phi;
    static constexpr int code = Code;
};
using Upwind = Scheme<PRISM_CONV_UPWIND>;
using CentralDifference = Scheme<PRISM_CONV_CENTRAL>;
using LinearUpwind = Scheme<PRISM_CONV_LINEAR_UPWIND>;
using QUICK = Scheme<PRISM_CONV_QUICK>;
using FROMM = Scheme<PRISM_CONV_FROMM>;
using MINMOD = Scheme<PRISM_CONV_MINMOD>;
using MUSCL = Scheme<PRISM_CONV_MUSCL>;
using SMART = Scheme<PRISM_CONV_SMART>;
}  // namespace convection
namespace diffusion {
template <int Corrected>
struct Scheme {
    Scheme(std::shared_ptr<field::Scalar> kappa, std::shared_ptr<field::Scalar> phi, int corrector = PRISM_CORR_OVER_RELAXED)
        : ks(std::move(kappa)), phi(std::move(phi)), corrector(corrector) {}
    Scheme(std::shared_ptr<field::Tensor> kappa, std::shared_ptr<field::Scalar> phi, int corrector = PRISM_CORR_OVER_RELAXED)
        : kt(std::move(kappa)), phi(std::move(phi)), corrector(corrector) {}
    std::shared_ptr<field::Scalar> ks;
    std::shared_ptr<field::Tensor> kt;
    std::shared_ptr<field::Scalar> phi;
    int corrector;
    static constexpr int corrected = Corrected;
};
using NonCorrected = Scheme<0>;
using Corrected = Scheme<1>;
}  // namespace diffusion
namespace source {
template <int Sign = PRISM_SIGN_POSITIVE>
struct ConstantScalar {
    explicit ConstantScalar(std::shared_ptr<field::Scalar> phi) : phi(std::move(phi)) {}
    std::shared_ptr<field::Scalar> phi;
};
template <int Sign = PRISM_SIGN_POSITIVE>
struct Divergence {
    explicit Divergence(std::shared_ptr<field::Vector> U) : U(std::move(U)) {}
    std::shared_ptr<field::Vector> U;
};
template <int Sign = PRISM_SIGN_POSITIVE>
struct Gradient {
    Gradient(std::shared_ptr<field::Scalar> phi, int coord) : phi(std::move(phi)), coord(coord) {}
    std::shared_ptr<field::Scalar> phi;
    int coord;
};
}  // namespace source
namespace temporal {
template <int Kind>
struct Scheme {
    explicit Scheme(std::shared_ptr<field::Scalar> phi, double dt = 1e-5) : phi(std::move(phi)), dt(dt) {
        if (dt <= 0.0) throw std::invalid_argument("prism::scheme::temporal::ITemporal(phi, dt): dt must be positive");
    }
    std::shared_ptr<field::Scalar> phi;
    double dt;
};
using BackwardEuler = Scheme<PRISM_TEMPORAL_BACKWARD_EULER>;
using AdamMoulton = Scheme<PRISM_TEMPORAL_ADAM_MOULTON>;
}  // namespace temporal
}  // namespace scheme

namespace eqn {
class Transport {
  public:
    template <typename Scheme, typename... Schemes>
    explicit Transport(Scheme&& first, Schemes&&... rest) {
        _phi = first.phi;
        PrismTransport* h = nullptr;
        check(prism_transport_create(_phi->handle(), &h));
        _h.reset(h, [](PrismTransport* t) { prism_transport_destroy(t); });
        add(std::forward<Scheme>(first));
        (add(std::forward<Schemes>(rest)), ...);
    }
    void setUnderRelaxFactor(double f) { check(prism_transport_set_urf(_h.get(), f)); }
    void updateCoeffs() { check(prism_transport_update_coeffs(_h.get())); }
    void relax() { check(prism_transport_relax(_h.get())); }
    void zeroOutCoeffs() { check(prism_transport_zero_coeffs(_h.get())); }
    void addSymmetryHandler() { check(prism_transport_add_symmetry_handler(_h.get())); }
    // temporalScheme()->setTimeStep(dt) (temporal.cpp:24-31)
    void setTimeStep(double dt) { check(prism_transport_set_time_step(_h.get(), dt)); }
    auto field() const -> const std::shared_ptr<field::Scalar>& { return _phi; }
    auto handle() const -> PrismTransport* { return _h.get(); }

  private:
    template <int C>
    void add(scheme::convection::Scheme<C> s) {
        check(prism_transport_add_convection(_h.get(), C, s.U->handle()));
        _keep.push_back(s.U);
    }
    template <int C>
    void add(scheme::diffusion::Scheme<C> s) {
        check(prism_transport_add_diffusion(_h.get(), C, s.corrector, s.ks ? s.ks->handle() : nullptr,
                                            s.kt ? s.kt->handle() : nullptr));
        _keep.push_back(s.ks);
        _keep.push_back(s.kt);
    }
    template <int K>
    void add(scheme::temporal::Scheme<K> s) {
        check(prism_transport_add_temporal(_h.get(), K, s.dt));
    }
    template <int S>
    void add(scheme::source::ConstantScalar<S> s) {
        check(prism_transport_add_source(_h.get(), PRISM_SRC_CONSTANT, S, s.phi->handle(), nullptr, 0));
        _keep.push_back(s.phi);
    }
    template <int S>
    void add(scheme::source::Divergence<S> s) {
        check(prism_transport_add_source(_h.get(), PRISM_SRC_DIVERGENCE, S, nullptr, s.U->handle(), 0));
        _keep.push_back(s.U);
    }
    template <int S>
    void add(scheme::source::Gradient<S> s) {
        check(prism_transport_add_source(_h.get(), PRISM_SRC_GRADIENT, S, s.phi->handle(), nullptr, s.coord));
        _keep.push_back(s.phi);
    }
    std::shared_ptr<field::Scalar> _phi;
    std::vector<std::shared_ptr<void>> _keep;
    std::shared_ptr<PrismTransport> _h;
};
using Momentum = Transport;
}  // namespace eqn

namespace solver {
struct SolverResult {
    size_t iteration = 0;
    double initial_residual = 0.0, final_residual = 0.0;
    bool converged = false;
    auto hasConverged() const -> bool { return converged; }
    auto iterations() const -> size_t { return iteration; }
    auto initialResidual() const -> double { return initial_residual; }
    auto finalResidual() const -> double { return final_residual; }
};

class ISolver {
  public:
    explicit ISolver(int method, int precision = PRISM_PREC_FP64) {
        prism_solve_opts_default(&_opts);
        _opts.method = method;
        _opts.precision = precision;
    }
    virtual ~ISolver() = default;
    auto solve(eqn::Transport& eq, size_t n_iter = 10, double eps = 1e-7, std::optional<size_t> ref_cell = std::nullopt,
               double ref_value = 0.0, bool clear_coeffs = true) -> SolverResult {
        PrismSolveOpts o = _opts;
        o.n_iter = (int64_t)n_iter;
        o.eps = eps;
        o.ref_cell = ref_cell ? (int64_t)*ref_cell : -1;
        o.ref_value = ref_value;
        o.clear_coeffs = clear_coeffs ? 1 : 0;
        PrismSolveResult r{};
        check(prism_solve(eq.handle(), &o, &r));
        return {(size_t)r.iterations, r.initial_residual, r.final_residual, r.converged != 0};
    }
    auto options() -> PrismSolveOpts& { return _opts; }

  private:
    PrismSolveOpts _opts{};
};
struct BiCGSTAB : ISolver {
    explicit BiCGSTAB(int precision = PRISM_PREC_FP64) : ISolver(PRISM_SOLVER_BICGSTAB, precision) {}
};
struct Jacobi : ISolver {
    Jacobi() : ISolver(PRISM_SOLVER_JACOBI) {}
};
}  // namespace solver

namespace algo {
struct Entry {
    std::string field_name;
    size_t n_iterations;
    double initial_residual, final_residual;
    bool converged;
};
using SIMPLEControls = PrismSIMPLEControls;
using PISOControls = PrismPISOControls;

namespace detail {
template <typename Controls, typename Fn>
auto step(const Controls& c, std::span<eqn::Momentum*> mom, field::Velocity& U, field::Velocity& mdot,
          field::Pressure& p, const PrismSolveOpts* so, Fn fn) -> std::vector<Entry> {
    std::vector<PrismTransport*> eqs;
    for (auto* e : mom) eqs.push_back(e->handle());
    PrismReport rep[64];
    int32_t n = 0;
    check(fn(&c, eqs.data(), (int32_t)eqs.size(), U.handle(), mdot.handle(), p.handle(), so, rep, 64, &n));
    std::vector<Entry> out;
    for (int32_t i = 0; i < n && i < 64; ++i)
        out.push_back({rep[i].field_name, (size_t)rep[i].n_iterations, rep[i].initial_residual, rep[i].final_residual,
                       rep[i].converged != 0});
    return out;
}
}  // namespace detail

class IncompressibleSIMPLE {
  public:
    explicit IncompressibleSIMPLE(SIMPLEControls c) : _c(c) {}
    IncompressibleSIMPLE() { prism_simple_controls_default(&_c); }
    auto step(std::span<eqn::Momentum*> mom, field::Velocity& U, field::Velocity& mdot, field::Pressure& p,
              const PrismSolveOpts* so = nullptr) -> std::vector<Entry> {
        return detail::step(_c, mom, U, mdot, p, so, prism_simple_step);
    }

  private:
    SIMPLEControls _c{};
};
class PRIME {
  public:
    explicit PRIME(SIMPLEControls c) : _c(c) {}
    auto step(std::span<eqn::Momentum*> mom, field::Velocity& U, field::Velocity& mdot, field::Pressure& p,
              const PrismSolveOpts* so = nullptr) -> std::vector<Entry> {
        return detail::step(_c, mom, U, mdot, p, so, prism_prime_step);
    }

  private:
    SIMPLEControls _c{};
};
class PISO {
  public:
    explicit PISO(PISOControls c) : _c(c) {}
    PISO() { prism_piso_controls_default(&_c); }
    auto step(std::span<eqn::Momentum*> mom, field::Velocity& U, field::Velocity& mdot, field::Pressure& p,
              const PrismSolveOpts* so = nullptr) -> std::vector<Entry> {
        return detail::step(_c, mom, U, mdot, p, so, prism_piso_step);
    }

  private:
    PISOControls _c{};
};
inline auto needsPressureReference(const field::Pressure& p) -> bool {
    int32_t out = 0;
    check(prism_needs_pressure_reference(p.handle(), &out));
    return out != 0;
}
}  // namespace algo

}  // namespace prism_b200
