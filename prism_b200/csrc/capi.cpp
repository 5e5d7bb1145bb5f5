// capi.cpp -- the extern "C" entry points of include/prism_b200.h.
// Every entry point converts library exceptions into a status code and keeps a
// thread-local message for prism_last_error(); nothing throws across the ABI.
// Every entry point is also an NVTX range named after it, so that a profiler's
// timeline (Nsight Systems, ncu --nvtx) shows which library call issued which
// kernels; without a tool attached the NVTX calls return at once.
#include <nvtx3/nvToolsExt.h>

#include <cstring>
#include <new>

#include "gradient.h"
#include "runtime.h"

using namespace pb;

struct PrismMesh {
    std::unique_ptr<Mesh> m;
};
struct PrismScalar {
    std::shared_ptr<Scalar> s;
};
struct PrismVector {
    std::unique_ptr<Vector> v;
    PrismScalar comp[3];
};
struct PrismTensor {
    std::unique_ptr<Tensor> t;
};
struct PrismTransport {
    Transport eq;
};
struct PrismBatch {
    BatchHandle h;
};

namespace {
thread_local std::string g_last_error;

struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

template <typename F>
int guardNamed(const char* name, F&& f) {
    NvtxRange range(name);
    try {
        f();
        return PRISM_OK;
    } catch (const Error& e) {
        g_last_error = e.msg;
        return e.status;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return PRISM_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return PRISM_INTERNAL;
    }
}
// guard([&] { ... }) inside an entry point: the range takes the entry point's name
#define guard(...) guardNamed(__func__, __VA_ARGS__)
#define ARG(cond, msg) \
    if (!(cond)) fail(PRISM_BAD_ARG, msg)

void setBC(Scalar& s, const PrismBC* bcs, int coord) {
    Mesh& m = *s.m;
    int np = std::max(m.npatch, 1);
    s.bc.assign(bcs, bcs + m.npatch);
    std::vector<int> kind(np, PRISM_BC_UNKNOWN);
    std::vector<double> val(np, 0.0), vec(3 * np, 0.0);
    for (int p = 0; p < m.npatch; ++p) {
        kind[p] = bcs[p].kind;
        if (coord >= 0) val[p] = bcs[p].value_kind == PRISM_BCV_VECTOR ? bcs[p].vector[coord] : 0.0;
        else val[p] = bcs[p].value_kind == PRISM_BCV_SCALAR ? bcs[p].value : 0.0;
        for (int k = 0; k < 3; ++k) vec[3 * p + k] = bcs[p].vector[k];
    }
    s.bc_kind.alloc(np);
    s.bc_kind.upload(kind.data(), np, m.stream);
    s.bc_val.alloc(np);
    s.bc_val.upload(val.data(), np, m.stream);
    s.bc_vec.alloc(3 * np);
    s.bc_vec.upload(vec.data(), 3 * np, m.stream);
}

std::shared_ptr<Scalar> newScalar(Mesh& m, const std::string& name, const double* values, int grad, const PrismBC* bcs,
                                  int coord) {
    auto s = std::make_shared<Scalar>();
    s->m = &m;
    s->name = name;
    s->coord = coord;
    s->v.alloc(m.n_pad);
    s->v.zero(m.stream);
    if (values) s->v.upload(values, m.nc, m.stream);
    setBC(*s, bcs, coord);
    s->grad = std::make_shared<GradState>();
    s->grad->type = grad;
    s->grad->g.alloc(3 * (size_t)m.n_pad);
    s->grad->g.zero(m.stream);
    PB_CUDA(cudaStreamSynchronize(m.stream));
    return s;
}

void sync(const Mesh& m) { PB_CUDA(cudaStreamSynchronize(m.stream)); }

std::vector<Transport*> momVec(PrismTransport* const* mom, int32_t n) {
    if (!mom || n <= 0) fail(PRISM_BAD_ARG, "no momentum equations");
    std::vector<Transport*> v;
    for (int32_t i = 0; i < n; ++i) {
        if (!mom[i]) fail(PRISM_BAD_ARG, "null momentum equation");
        v.push_back(&mom[i]->eq);
    }
    return v;
}
void writeReports(const std::vector<Report>& rep, PrismReport* out, int32_t max, int32_t* n) {
    int32_t k = 0;
    for (auto& r : rep) {
        if (out && k < max) {
            std::memset(&out[k], 0, sizeof(PrismReport));
            std::strncpy(out[k].field_name, r.name.c_str(), sizeof(out[k].field_name) - 1);
            out[k].n_iterations = r.n;
            out[k].initial_residual = r.init;
            out[k].final_residual = r.fin;
            out[k].converged = r.conv ? 1 : 0;
        }
        ++k;
    }
    if (n) *n = k;
}
PrismSolveOpts optsOrDefault(const PrismSolveOpts* so) {
    PrismSolveOpts o;
    solveDefaults(&o);
    if (so) o = *so;
    return o;
}
}  // namespace

#define API extern "C" __attribute__((visibility("default")))

API const char* prism_last_error(void) { return g_last_error.c_str(); }
API const char* prism_status_string(int s) {
    static const char* names[] = {"OK", "NOT_CONVERGED", "BREAKDOWN", "NONFINITE", "BAD_ARG", "CUDA_ERROR",
                                  "INVALID_MESH", "NO_BC_HANDLER", "SPIN_TIMEOUT", "INTERNAL", "OUT_OF_MEMORY"};
    return (s >= 0 && s <= 10) ? names[s] : "UNKNOWN";
}

// ---- mesh
API int prism_mesh_from_unv(const PrismUnvMesh* d, PrismMesh** out) {
    return guard([&] {
        ARG(d && out, "null argument");
        auto pm = std::make_unique<PrismMesh>();
        pm->m = createMesh(d);
        *out = pm.release();
    });
}
API int prism_mesh_info(const PrismMesh* pm, PrismMeshInfo* info) {
    return guard([&] {
        ARG(pm && info, "null argument");
        const Mesh& m = *pm->m;
        info->n_cells = m.nc;
        info->n_faces = m.nf;
        info->n_boundary_faces = m.nb;
        info->n_nonempty_boundary_faces = m.nne;
        info->nnz = m.pat.nnz;
        info->n_patches = m.npatch;
        info->n_gs_levels = (int32_t)m.level_off.size() - 1;
        info->n_vertices = m.h->nv;
        info->n_cell_vertices = m.h->cv_off[m.h->nc];
    });
}
API int prism_mesh_export(const PrismMesh* pm, PrismMeshExport* o) {
    return guard([&] {
        ARG(pm && o, "null argument");
        const Mesh& m = *pm->m;
        const HostMesh& h = *m.h;
        const int64_t nf = h.nf, nc = h.nc;
        for (int64_t f = 0; f < nf; ++f) {
            if (o->owner) o->owner[f] = h.owner[f];
            if (o->neighbor) o->neighbor[f] = h.nbr[f];
            if (o->face_patch) o->face_patch[f] = h.nbr[f] >= 0 ? -1 : h.patch[f];
            if (o->face_area) o->face_area[f] = h.area[f];
            for (int k = 0; k < 3; ++k) {
                if (o->face_normal) o->face_normal[k * nf + f] = h.normal[k][f];
                if (o->face_center) o->face_center[k * nf + f] = h.fc[k][f];
            }
        }
        for (int64_t c = 0; c < nc; ++c) {
            if (o->cell_volume) o->cell_volume[c] = h.vol[c];
            for (int k = 0; k < 3; ++k)
                if (o->cell_center) o->cell_center[k * nc + c] = h.cc[k][c];
        }
        for (int64_t c = 0; c <= nc; ++c)
            if (o->cell_face_offsets) o->cell_face_offsets[c] = h.cf_off[c];
        if (o->cell_faces)
            for (size_t q = 0; q < h.cf_face.size(); ++q) o->cell_faces[q] = h.cf_face[q];
        if (o->csr_rowptr || o->csr_col) {
            // the pattern was built on the device: read it back
            std::vector<int> rp(nc + 1), col(m.pat.nnz);
            m.pat.rowptr.download(rp.data(), nc + 1, m.stream);
            m.pat.col.download(col.data(), m.pat.nnz, m.stream);
            sync(m);
            if (o->csr_rowptr)
                for (int64_t i = 0; i <= nc; ++i) o->csr_rowptr[i] = rp[i];
            if (o->csr_col)
                for (int64_t k = 0; k < m.pat.nnz; ++k) o->csr_col[k] = col[k];
        }
        int64_t pos = 0;
        for (size_t p = 0; p < h.patches.size(); ++p) {
            if (o->patch_face_offsets) o->patch_face_offsets[p] = pos;
            for (auto f : h.patches[p].faces) {
                if (o->patch_faces) o->patch_faces[pos] = f;
                ++pos;
            }
        }
        if (o->patch_face_offsets) o->patch_face_offsets[h.patches.size()] = pos;
        for (int k = 0; k < 3; ++k)
            if (o->vertex_coords) std::copy(h.vx[k].begin(), h.vx[k].end(), o->vertex_coords + k * h.nv);
        if (o->cell_vertex_offsets) std::copy(h.cv_off.begin(), h.cv_off.end(), o->cell_vertex_offsets);
        if (o->cell_vertices) std::copy(h.cv_node.begin(), h.cv_node.end(), o->cell_vertices);
        if (o->cell_original) std::copy(h.cell_orig.begin(), h.cell_orig.end(), o->cell_original);
    });
}
API int prism_mesh_destroy(PrismMesh* pm) {
    return guard([&] { delete pm; });
}
API int prism_mesh_reorder(PrismMesh* pm, int32_t reverse) {
    return guard([&] {
        ARG(pm, "null argument");
        reorderMesh(*pm->m, reverse != 0);
    });
}

// ---- scalar
API int prism_scalar_create(PrismMesh* pm, const char* name, const double* values, int32_t grad, const PrismBC* bcs,
                            PrismScalar** out) {
    return guard([&] {
        ARG(pm && name && bcs && out, "null argument");
        pm->m->frozen = true;
        ARG(grad == PRISM_GRAD_LEAST_SQUARES || grad == PRISM_GRAD_GREEN_GAUSS, "bad gradient scheme");
        auto ps = std::make_unique<PrismScalar>();
        ps->s = newScalar(*pm->m, name, values, grad, bcs, -1);
        *out = ps.release();
    });
}
API int prism_scalar_destroy(PrismScalar* s) {
    return guard([&] {
        delete s;  // cudaFree synchronizes; the mesh is not touched
    });
}
API int prism_scalar_set_values(PrismScalar* ps, const double* v) {
    return guard([&] {
        ARG(ps && v, "null argument");
        Scalar& s = *ps->s;
        ++s.event;
        s.v.upload(v, s.m->nc, s.m->stream);
        sync(*s.m);
    });
}
API int prism_scalar_get_values(const PrismScalar* ps, double* v) {
    return guard([&] {
        ARG(ps && v, "null argument");
        const Scalar& s = *ps->s;
        s.v.download(v, s.m->nc, s.m->stream);
        sync(*s.m);
    });
}
API int prism_scalar_set_face_values(PrismScalar* ps, const double* fv) {
    return guard([&] {
        ARG(ps, "null argument");
        Scalar& s = *ps->s;
        if (fv) {
            if (!s.fv) s.fv.alloc(std::max(s.m->nf, 1));
            s.fv.upload(fv, s.m->nf, s.m->stream);
            s.has_fv = true;
            sync(*s.m);
        } else {
            s.has_fv = false;
        }
    });
}
API int prism_scalar_face_values(PrismScalar* ps, double* out) {
    return guard([&] {
        ARG(ps && out, "null argument");
        Scalar& s = *ps->s;
        Mesh& m = *s.m;
        // every non-empty boundary face is evaluated through its handler
        if (!s.has_fv)
            for (int p = 0; p < m.npatch; ++p)
                if (!m.h->patches[p].empty && !m.h->patches[p].faces.empty()) {
                    int k = s.bc[p].kind;
                    if (!(k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP || k == PRISM_BC_SYMMETRY ||
                          k == PRISM_BC_OUTLET || k == PRISM_BC_ZERO_GRADIENT))
                        fail(PRISM_NO_BC_HANDLER, "Scalar::valueAtBoundaryFace(): no handler on patch '" +
                                                      m.h->patches[p].name + "'");
                }
        launchScalarFaces(m.view(), s.view(), m.scratch.p, m.stream);
        m.scratch.download(out, m.nf, m.stream);
        sync(m);
    });
}
API int prism_scalar_grad(PrismScalar* ps, double* out) {
    return guard([&] {
        ARG(ps && out, "null argument");
        Scalar& s = *ps->s;
        ensureGradient(s);
        for (int k = 0; k < 3; ++k)
            PB_CUDA(cudaMemcpyAsync(out + (size_t)k * s.m->nc, s.grad->g.p + (size_t)k * s.m->n_pad,
                                    s.m->nc * sizeof(double), cudaMemcpyDeviceToHost, s.m->stream));
        sync(*s.m);
    });
}
API int prism_scalar_compute_gradients(PrismScalar* ps) {
    return guard([&] {
        ARG(ps, "null argument");
        computeGradient(*ps->s);
        sync(*ps->s->m);
    });
}
API int prism_scalar_set_grad_scheme(PrismScalar* ps, int32_t grad) {
    return guard([&] {
        ARG(ps, "null argument");
        ARG(grad == PRISM_GRAD_LEAST_SQUARES || grad == PRISM_GRAD_GREEN_GAUSS, "bad gradient scheme");
        Scalar& s = *ps->s;
        auto g = std::make_shared<GradState>();
        g->type = grad;
        g->g.alloc(3 * (size_t)s.m->n_pad);
        g->g.zero(s.m->stream);
        s.grad = std::move(g);
        sync(*s.m);
    });
}
API int prism_rhie_chow(PrismVector* pmdot, PrismVector* pU, PrismTensor* pD, PrismScalar* pp) {
    return guard([&] {
        ARG(pmdot && pU && pD && pp, "null argument");
        Mesh& m = *pp->s->m;
        ARG(pmdot->v->m == &m && pU->v->m == &m && pD->t->m == &m, "fields on different meshes");
        rhieChowFaces(*pmdot->v, *pU->v, *pD->t, *pp->s);
        sync(m);
    });
}
API int prism_scalar_set_history_size(PrismScalar* ps, int32_t n) {
    return guard([&] {
        ARG(ps && n >= 0, "bad argument");
        setHistorySize(*ps->s, (size_t)n);
    });
}
API int prism_scalar_update_prev_time_steps(PrismScalar* ps) {
    return guard([&] {
        ARG(ps, "null argument");
        updatePrevTimeSteps(*ps->s);
        sync(*ps->s->m);
    });
}
API int prism_scalar_update(PrismScalar* ps, const double* values) {
    return guard([&] {
        ARG(ps && values, "null argument");
        Scalar& s = *ps->s;
        updatePrevTimeSteps(s);
        s.v.upload(values, s.m->nc, s.m->stream);
        ++s.event;
        s.has_fv = false;
        sync(*s.m);
    });
}
API int prism_scalar_history(const PrismScalar* ps, int32_t index, double* out, int32_t* available) {
    return guard([&] {
        ARG(ps && out && available && index >= 0, "bad argument");
        const Scalar& s = *ps->s;
        *available = (size_t)index < s.hist.size() ? 1 : 0;
        if (*available) {
            s.hist[index].download(out, s.m->nc, s.m->stream);
            sync(*s.m);
        }
    });
}

// ---- vector
API int prism_vector_create(PrismMesh* pm, const char* name, const double* values, int32_t grad, const PrismBC* bcs,
                            PrismVector** out) {
    return guard([&] {
        ARG(pm && name && bcs && out, "null argument");
        pm->m->frozen = true;
        ARG(grad == PRISM_GRAD_LEAST_SQUARES || grad == PRISM_GRAD_GREEN_GAUSS, "bad gradient scheme");
        Mesh& m = *pm->m;
        auto pv = std::make_unique<PrismVector>();
        pv->v = std::make_unique<Vector>();
        Vector& U = *pv->v;
        U.m = &m;
        U.name = name;
        U.bc.assign(bcs, bcs + m.npatch);
        int np = std::max(m.npatch, 1);
        std::vector<int> kind(np, PRISM_BC_UNKNOWN);
        std::vector<double> vec(3 * np, 0.0);
        for (int p = 0; p < m.npatch; ++p) {
            kind[p] = bcs[p].kind;
            for (int k = 0; k < 3; ++k) vec[3 * p + k] = bcs[p].vector[k];
        }
        U.bc_kind.alloc(np);
        U.bc_kind.upload(kind.data(), np, m.stream);
        U.bc_vec.alloc(3 * np);
        U.bc_vec.upload(vec.data(), 3 * np, m.stream);
        const char* suf[3] = {"_x", "_y", "_z"};
        for (int k = 0; k < 3; ++k) {
            U.c[k] = newScalar(m, std::string(name) + suf[k], values ? values + (size_t)k * m.nc : nullptr, grad, bcs,
                               k);
            pv->comp[k].s = U.c[k];
        }
        *out = pv.release();
    });
}
API int prism_vector_clone(const PrismVector* src, PrismVector** out) {
    return guard([&] {
        ARG(src && out, "null argument");
        const Vector& S = *src->v;
        Mesh& m = *S.m;
        auto pv = std::make_unique<PrismVector>();
        pv->v = std::make_unique<Vector>();
        Vector& U = *pv->v;
        U.m = &m;
        U.name = S.name;
        U.bc = S.bc;
        int np = std::max(m.npatch, 1);
        U.bc_kind.alloc(np);
        U.bc_vec.alloc(3 * np);
        PB_CUDA(cudaMemcpyAsync(U.bc_kind.p, S.bc_kind.p, np * sizeof(int), cudaMemcpyDeviceToDevice, m.stream));
        PB_CUDA(cudaMemcpyAsync(U.bc_vec.p, S.bc_vec.p, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
        if (S.has_fd) {
            U.fd.alloc(S.fd.n);
            PB_CUDA(cudaMemcpyAsync(U.fd.p, S.fd.p, S.fd.n * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
            U.has_fd = true;
        }
        if (S.has_ff) {
            U.ff.alloc(S.ff.n);
            PB_CUDA(cudaMemcpyAsync(U.ff.p, S.ff.p, S.ff.n * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
            U.has_ff = true;
        }
        for (int k = 0; k < 3; ++k) {
            // Scalar copy: values copied, gradient scheme shared (vector.h:318-336)
            const Scalar& cs = *S.c[k];
            auto s = std::make_shared<Scalar>();
            s->m = &m;
            s->name = cs.name;
            s->coord = cs.coord;
            s->v.alloc(m.n_pad);
            PB_CUDA(cudaMemcpyAsync(s->v.p, cs.v.p, m.n_pad * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
            if (cs.has_fv) {
                s->fv.alloc(cs.fv.n);
                PB_CUDA(cudaMemcpyAsync(s->fv.p, cs.fv.p, cs.fv.n * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
                s->has_fv = true;
            }
            setBC(*s, cs.bc.data(), cs.coord);
            s->grad = cs.grad;
            s->event = cs.event;
            U.c[k] = s;
            pv->comp[k].s = s;
        }
        sync(m);
        *out = pv.release();
    });
}
API int prism_vector_destroy(PrismVector* v) {
    return guard([&] {
        delete v;  // cudaFree synchronizes; the mesh is not touched
    });
}
API int prism_vector_component(PrismVector* pv, int32_t coord, PrismScalar** out) {
    return guard([&] {
        ARG(pv && out && coord >= 0 && coord < 3, "bad argument");
        *out = &pv->comp[coord];
    });
}
API int prism_vector_set_values(PrismVector* pv, const double* v) {
    return guard([&] {
        ARG(pv && v, "null argument");
        Vector& U = *pv->v;
        for (int k = 0; k < 3; ++k) {
            ++U.c[k]->event;
            U.c[k]->v.upload(v + (size_t)k * U.m->nc, U.m->nc, U.m->stream);
        }
        sync(*U.m);
    });
}
API int prism_vector_get_values(const PrismVector* pv, double* v) {
    return guard([&] {
        ARG(pv && v, "null argument");
        const Vector& U = *pv->v;
        for (int k = 0; k < 3; ++k) U.c[k]->v.download(v + (size_t)k * U.m->nc, U.m->nc, U.m->stream);
        sync(*U.m);
    });
}
API int prism_vector_face_flux(PrismVector* pv, double* out) {
    return guard([&] {
        ARG(pv && out, "null argument");
        Vector& U = *pv->v;
        Mesh& m = *U.m;
        if (!U.has_ff)
            for (int p = 0; p < m.npatch; ++p)
                if (!m.h->patches[p].empty && !m.h->patches[p].faces.empty()) {
                    int k = U.bc[p].kind;
                    if (!(k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP || k == PRISM_BC_SYMMETRY ||
                          k == PRISM_BC_OUTLET || k == PRISM_BC_ZERO_GRADIENT))
                        fail(PRISM_NO_BC_HANDLER, "GeneralVector::fluxAtBoundaryFace(): no handler on patch '" +
                                                      m.h->patches[p].name + "'");
                }
        launchVectorFlux(m.view(), U.view(), m.scratch.p, m.stream);
        m.scratch.download(out, m.nf, m.stream);
        sync(m);
    });
}

// ---- diagnostics and point data
namespace {
PrismScalar* diagnosticScalar(Mesh& m, const std::string& name) {
    // field::Scalar(name, mesh, data): no boundary handlers, least-squares gradient
    std::vector<PrismBC> none(std::max(m.npatch, 1));
    for (auto& b : none) {
        std::memset(&b, 0, sizeof(PrismBC));
        b.kind = PRISM_BC_UNKNOWN;
    }
    auto ps = std::make_unique<PrismScalar>();
    ps->s = newScalar(m, name, nullptr, PRISM_GRAD_LEAST_SQUARES, none.data(), -1);
    return ps.release();
}
void downloadPoints(Mesh& m, int ncomp, const double* const* comp, int64_t stride, double* out) {
    DevBuf<double> pts((size_t)m.h->nv * ncomp);
    cellToPoint(m, comp, ncomp, stride, pts.p);
    pts.download(out, pts.n, m.stream);
    sync(m);
}
}  // namespace

API int prism_ops_div(PrismVector* pv, PrismScalar** out) {
    return guard([&] {
        ARG(pv && out, "null argument");
        Vector& U = *pv->v;
        std::unique_ptr<PrismScalar> ps(diagnosticScalar(*U.m, "div(" + U.name + ")"));
        opsDiv(U, ps->s->v.p);
        sync(*U.m);
        *out = ps.release();
    });
}
API int prism_courant_number(PrismVector* pv, double dt, PrismScalar** out) {
    return guard([&] {
        ARG(pv && out, "null argument");
        Vector& U = *pv->v;
        std::unique_ptr<PrismScalar> ps(diagnosticScalar(*U.m, "Co"));
        courantNumber(U, dt, ps->s->v.p);
        sync(*U.m);
        *out = ps.release();
    });
}
API int prism_cell_to_point(PrismMesh* pm, const double* cell_data, int32_t ncomp, double* point_data) {
    return guard([&] {
        ARG(pm && cell_data && point_data, "null argument");
        ARG(ncomp >= 1 && ncomp <= 9, "n_components must be 1..9");
        Mesh& m = *pm->m;
        DevBuf<double> cells((size_t)m.nc * ncomp);
        cells.upload(cell_data, cells.n, m.stream);
        const double* comp[9];
        for (int k = 0; k < ncomp; ++k) comp[k] = cells.p + k;
        downloadPoints(m, ncomp, comp, ncomp, point_data);
    });
}
API int prism_scalar_to_points(PrismScalar* ps, double* point_data) {
    return guard([&] {
        ARG(ps && point_data, "null argument");
        const double* comp[1] = {ps->s->v.p};
        downloadPoints(*ps->s->m, 1, comp, 1, point_data);
    });
}
API int prism_vector_to_points(PrismVector* pv, double* point_data) {
    return guard([&] {
        ARG(pv && point_data, "null argument");
        Vector& U = *pv->v;
        const double* comp[3] = {U.c[0]->v.p, U.c[1]->v.p, U.c[2]->v.p};
        downloadPoints(*U.m, 3, comp, 1, point_data);
    });
}

API int prism_vector_set_face_flux(PrismVector* pv, const double* flux) {
    return guard([&] {
        ARG(pv && flux, "null argument");
        Vector& U = *pv->v;
        Mesh& m = *U.m;
        if (U.ff.n < (size_t)m.nf) U.ff.alloc(std::max(m.nf, 1));
        U.ff.upload(flux, m.nf, m.stream);
        U.has_ff = true;
        sync(m);
    });
}

// ---- tensor
API int prism_tensor_create(PrismMesh* pm, const char* name, const double* values, PrismTensor** out) {
    return guard([&] {
        ARG(pm && out, "null argument");
        pm->m->frozen = true;
        (void)name;
        Mesh& m = *pm->m;
        auto pt = std::make_unique<PrismTensor>();
        pt->t = std::make_unique<Tensor>();
        Tensor& T = *pt->t;
        T.m = &m;
        T.diag = 0;
        std::vector<double> h(9 * (size_t)m.n_pad, 0.0);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int c = 0; c < m.nc; ++c)
                    h[(3 * i + j) * (size_t)m.n_pad + c] = values ? values[(3 * i + j) * (size_t)m.nc + c] : (i == j ? 1.0 : 0.0);
        T.d.alloc(h.size());
        T.d.upload(h.data(), h.size(), m.stream);
        sync(m);
        *out = pt.release();
    });
}
API int prism_tensor_destroy(PrismTensor* t) {
    return guard([&] {
        delete t;  // cudaFree synchronizes; the mesh is not touched
    });
}

// ---- transport
API int prism_transport_create(PrismScalar* phi, PrismTransport** out) {
    return guard([&] {
        ARG(phi && out, "null argument");
        auto pt = std::make_unique<PrismTransport>();
        pt->eq.phi = phi->s.get();
        *out = pt.release();
    });
}
API int prism_transport_destroy(PrismTransport* eq) {
    return guard([&] {
        delete eq;  // cudaFree synchronizes; the mesh is not touched
    });
}
API int prism_transport_add_convection(PrismTransport* pt, int32_t scheme, PrismVector* U) {
    return guard([&] {
        ARG(pt && U && scheme >= PRISM_CONV_UPWIND && scheme <= PRISM_CONV_SMART, "bad argument");
        ARG(!pt->eq.has_conv, "equation already has a convection scheme");
        pt->eq.has_conv = 1;
        pt->eq.conv_scheme = scheme;
        pt->eq.U = U->v.get();
        if (!pt->eq.has_diff) pt->eq.conv_first = 1;
        pt->eq.order[pt->eq.nsch++] = SCH_CONV;
    });
}
API int prism_transport_add_diffusion(PrismTransport* pt, int32_t corrected, int32_t corrector, PrismScalar* ks,
                                      PrismTensor* kt) {
    return guard([&] {
        ARG(pt && ((ks != nullptr) != (kt != nullptr)), "exactly one diffusion coefficient");
        ARG(corrector >= 0 && corrector <= 2, "bad corrector");
        ARG(!pt->eq.has_diff, "equation already has a diffusion scheme");
        pt->eq.has_diff = 1;
        pt->eq.corrected = corrected ? 1 : 0;
        pt->eq.corrector = corrector;
        pt->eq.ks = ks ? ks->s.get() : nullptr;
        pt->eq.kt = kt ? kt->t.get() : nullptr;
        if (!pt->eq.has_conv) pt->eq.conv_first = 0;
        pt->eq.order[pt->eq.nsch++] = SCH_DIFF;
    });
}
API int prism_transport_add_temporal(PrismTransport* pt, int32_t kind, double dt) {
    return guard([&] {
        ARG(pt, "null argument");
        ARG(kind == PRISM_TEMPORAL_BACKWARD_EULER || kind == PRISM_TEMPORAL_ADAM_MOULTON, "bad temporal scheme");
        ARG(dt > 0.0, "prism::scheme::temporal::ITemporal(phi, dt): dt must be positive");
        ARG(!pt->eq.has_temporal, "equation already has a temporal scheme");
        pt->eq.has_temporal = 1;
        pt->eq.temporal_kind = kind;
        pt->eq.dt = dt;
        pt->eq.order[pt->eq.nsch++] = SCH_TEMPORAL;
    });
}
API int prism_transport_set_time_step(PrismTransport* pt, double dt) {
    return guard([&] {
        ARG(pt, "null argument");
        ARG(dt > 0.0, "prism::scheme::temporal::ITemporal::setTimeStep(): dt must be positive");
        ARG(pt->eq.has_temporal, "equation has no temporal scheme");
        pt->eq.dt = dt;
    });
}
API int prism_transport_add_source(PrismTransport* pt, int32_t kind, int32_t sign, PrismScalar* ss, PrismVector* sv,
                                   int32_t coord) {
    return guard([&] {
        ARG(pt, "null argument");
        ARG(kind >= PRISM_SRC_CONSTANT && kind <= PRISM_SRC_GRADIENT, "bad source kind");
        ARG((int)pt->eq.sources.size() < MAX_SOURCES, "too many sources");
        Source s{kind, sign, coord, nullptr, nullptr};
        if (kind == PRISM_SRC_DIVERGENCE) {
            ARG(sv, "divergence needs a vector");
            s.U = sv->v.get();
        } else {
            ARG(ss, "source needs a scalar");
            s.s = ss->s.get();
        }
        ARG(kind != PRISM_SRC_GRADIENT || (coord >= 0 && coord < 3), "bad coord");
        pt->eq.sources.push_back(s);
    });
}
API int prism_transport_add_symmetry_handler(PrismTransport* pt) {
    return guard([&] {
        ARG(pt, "null argument");
        pt->eq.symmetry = true;
    });
}
API int prism_transport_set_urf(PrismTransport* pt, double f) {
    return guard([&] {
        ARG(pt, "null argument");
        if (f < 0.0 || f > 1.0) return;  // transport.cpp:38-52 keeps the old value
        pt->eq.urf = f;
    });
}
API int prism_transport_update_coeffs(PrismTransport* pt) {
    return guard([&] {
        ARG(pt, "null argument");
        updateCoeffs(pt->eq);
        sync(*pt->eq.phi->m);
    });
}
API int prism_transport_relax(PrismTransport* pt) {
    return guard([&] {
        ARG(pt, "null argument");
        relax(pt->eq);
        sync(*pt->eq.phi->m);
    });
}
API int prism_transport_zero_coeffs(PrismTransport* pt) {
    return guard([&] {
        ARG(pt, "null argument");
        zeroOutCoeffs(pt->eq);
        sync(*pt->eq.phi->m);
    });
}
API int prism_transport_get_system(const PrismTransport* pt, double* vals, double* rhs) {
    return guard([&] {
        ARG(pt, "null argument");
        Transport& eq = const_cast<Transport&>(pt->eq);
        Mesh& m = *eq.phi->m;
        eq.ensure();
        if (vals) {
            // SELL -> CSR order: entry j of row r is at sl_off[r/32] + 32 j + r%32
            std::vector<double> sv(m.pat.sell_nnz);
            std::vector<int> slo(m.pat.nslices + 1), rp(m.nc + 1);
            eq.A.download(sv.data(), sv.size(), m.stream);
            m.pat.sl_off.download(slo.data(), slo.size(), m.stream);
            m.pat.rowptr.download(rp.data(), rp.size(), m.stream);
            sync(m);
            for (int r = 0; r < m.nc; ++r)
                for (int j = 0; j < rp[r + 1] - rp[r]; ++j) vals[rp[r] + j] = sv[slo[r >> 5] + 32 * j + (r & 31)];
        }
        if (rhs) {
            eq.b.download(rhs, m.nc, m.stream);
            sync(m);
        }
    });
}

// ---- solvers
API void prism_solve_opts_default(PrismSolveOpts* o) {
    if (o) solveDefaults(o);
}
API int prism_solve(PrismTransport* pt, const PrismSolveOpts* o, PrismSolveResult* r) {
    return guard([&] {
        ARG(pt && o && r, "null argument");
        if (o->graph && graphReady(pt->eq, *o)) *r = solveAsGraph(pt->eq, *o);
        else *r = solve(pt->eq, *o);
        sync(*pt->eq.phi->m);
    });
}
API int prism_solve_csr(int64_t n, const int64_t* rowptr, const int64_t* col, const double* values, const double* b,
                        double* x, const PrismSolveOpts* o, PrismSolveResult* r) {
    return guard([&] {
        ARG(n > 0 && rowptr && col && values && b && x && o, "bad argument");
        ARG(n < (int64_t(1) << 31), "matrix too large");
        ARG(rowptr[0] == 0 && rowptr[n] < (int64_t(1) << 31), "bad row pointers");
        for (int64_t i = 0; i < n; ++i) ARG(rowptr[i + 1] >= rowptr[i], "bad row pointers");
        // host-side SELL-32 layout of the caller's CSR matrix
        int nslices = ceil_div(n, 32);
        std::vector<int> slo(nslices + 1, 0), dpos(n, -1);
        for (int s = 0; s < nslices; ++s) {
            int64_t w = 0;
            for (int l = 0; l < 32 && s * 32 + l < n; ++l) w = std::max(w, rowptr[s * 32 + l + 1] - rowptr[s * 32 + l]);
            slo[s + 1] = slo[s] + 32 * (int)w;
        }
        std::vector<int> sc(slo[nslices], 0);
        std::vector<double> sv(slo[nslices], 0.0);
        for (int64_t i = 0; i < n; ++i) {
            int s = (int)(i >> 5), lane = (int)(i & 31);
            int w = (slo[s + 1] - slo[s]) >> 5;
            int64_t len = rowptr[i + 1] - rowptr[i];
            for (int j = 0; j < w; ++j) {
                int pos = slo[s] + 32 * j + lane;
                if (j < len) {
                    ARG(col[rowptr[i] + j] >= 0 && col[rowptr[i] + j] < n, "column out of range");
                    sc[pos] = (int)col[rowptr[i] + j];
                    sv[pos] = values[rowptr[i] + j];
                    if (sc[pos] == i) dpos[i] = pos;
                } else {
                    sc[pos] = (int)i;
                }
            }
            ARG(dpos[i] >= 0, "matrix row without a diagonal entry");
        }
        cudaStream_t s;
        PB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
        } sg{s};
        DevBuf<int> d_slo, d_sc, d_dpos;
        DevBuf<double> d_sv, d_b, d_x;
        d_slo.upload(slo, s);
        d_sc.upload(sc, s);
        d_dpos.upload(dpos, s);
        d_sv.upload(sv, s);
        int n_pad = nslices * 32;
        d_b.alloc(n_pad);
        d_b.zero(s);
        d_b.upload(b, n, s);
        d_x.alloc(n_pad);
        d_x.zero(s);
        d_x.upload(x, n, s);
        SellMatrix A;
        A.n = (int)n;
        A.nslices = nslices;
        A.nnz_padded = slo[nslices];
        A.sl_off = d_slo.p;
        A.col = d_sc.p;
        A.diag_pos = d_dpos.p;
        A.vals = d_sv.p;
        A.nnz_csr = rowptr[n];
        KrylovWork kw;
        KrylovOut k;
        if (o->method == PRISM_SOLVER_JACOBI) {
            jacobiStep(A, d_b.p, d_x.p, kw, s);
        } else {
            Amg amg;
            DevBuf<int> d_rp, d_col;
            const bool fcg = o->method == PRISM_SOLVER_FCG;
            if (fcg && (o->precision != PRISM_PREC_FP64 || o->preconditioner == PRISM_PC_JACOBI))
                fail(PRISM_BAD_ARG, "flexible CG runs in FP64 with the AMG preconditioner");
            const bool use_amg = fcg || choosePreconditioner(o->preconditioner, n) == PRISM_PC_AMG;
            if (use_amg) {
                std::vector<int> rp32(rowptr, rowptr + n + 1), col32(col, col + rowptr[n]);
                d_rp.upload(rp32, s);
                d_col.upload(col32, s);
            }
            k = bicgstab(A, d_b.p, d_x.p, o->krylov_tol > 0 ? o->krylov_tol : 1e-12,
                         o->krylov_max_iter > 0 ? o->krylov_max_iter : 2 * n, o->precision,
                         o->inner_tol > 0 ? o->inner_tol : 0.1, kw, s, use_amg ? &amg : nullptr, d_rp.p, d_col.p,
                         fcg);
        }
        double res = scaledResidual(A, d_b.p, d_x.p, kw, s);
        d_x.download(x, n, s);
        PB_CUDA(cudaStreamSynchronize(s));
        if (r) {
            std::memset(r, 0, sizeof(*r));
            r->iterations = 1;
            r->krylov_iterations = k.iterations;
            r->krylov_rel_residual = k.rel_residual;
            r->status = k.status;
            r->final_residual = res;
        }
    });
}

// ---- pressure-velocity coupling
API void prism_simple_controls_default(PrismSIMPLEControls* c) {
    if (c) simpleDefaults(c);
}
API void prism_piso_controls_default(PrismPISOControls* c) {
    if (c) pisoDefaults(c);
}
API int prism_simple_step(const PrismSIMPLEControls* c, PrismTransport* const* mom, int32_t n_mom, PrismVector* U,
                          PrismVector* mdot, PrismScalar* p, const PrismSolveOpts* so, PrismReport* rep, int32_t max,
                          int32_t* n) {
    return guard([&] {
        ARG(c && U && mdot && p, "null argument");
        auto v = momVec(mom, n_mom);
        std::vector<Report> r;
        const PrismSolveOpts opts = optsOrDefault(so);
        if (opts.graph && !c->batched_momentum && stepGraphReady(v, *U->v, *p->s, opts, true))
            stepAsGraph(*p->s->m, [&] { simpleStep(*c, v, *U->v, *mdot->v, *p->s, opts, r); }, r);
        else
            simpleStep(*c, v, *U->v, *mdot->v, *p->s, opts, r);
        sync(*p->s->m);
        writeReports(r, rep, max, n);
    });
}
API int prism_prime_step(const PrismSIMPLEControls* c, PrismTransport* const* mom, int32_t n_mom, PrismVector* U,
                         PrismVector* mdot, PrismScalar* p, const PrismSolveOpts* so, PrismReport* rep, int32_t max,
                         int32_t* n) {
    return guard([&] {
        ARG(c && U && mdot && p, "null argument");
        auto v = momVec(mom, n_mom);
        std::vector<Report> r;
        const PrismSolveOpts opts = optsOrDefault(so);
        if (opts.graph && stepGraphReady(v, *U->v, *p->s, opts, false))
            stepAsGraph(*p->s->m, [&] { primeStep(*c, v, *U->v, *mdot->v, *p->s, opts, r); }, r);
        else
            primeStep(*c, v, *U->v, *mdot->v, *p->s, opts, r);
        sync(*p->s->m);
        writeReports(r, rep, max, n);
    });
}
API int prism_piso_step(const PrismPISOControls* c, PrismTransport* const* mom, int32_t n_mom, PrismVector* U,
                        PrismVector* mdot, PrismScalar* p, const PrismSolveOpts* so, PrismReport* rep, int32_t max,
                        int32_t* n) {
    return guard([&] {
        ARG(c && U && mdot && p, "null argument");
        auto v = momVec(mom, n_mom);
        std::vector<Report> r;
        const PrismSolveOpts opts = optsOrDefault(so);
        if (opts.graph && !c->batched_momentum && stepGraphReady(v, *U->v, *p->s, opts, true))
            stepAsGraph(*p->s->m, [&] { pisoStep(*c, v, *U->v, *mdot->v, *p->s, opts, r); }, r);
        else
            pisoStep(*c, v, *U->v, *mdot->v, *p->s, opts, r);
        sync(*p->s->m);
        writeReports(r, rep, max, n);
    });
}
API int prism_needs_pressure_reference(PrismScalar* p, int32_t* out) {
    return guard([&] {
        ARG(p && out, "null argument");
        *out = needsPressureReference(*p->s) ? 1 : 0;
    });
}

// ---- measurement
API int prism_profile_start(int32_t max_samples) {
    return guard([&] { profileStart(max_samples); });
}
API int prism_profile_stop(PrismProfile* out) {
    return guard([&] {
        ARG(out, "null argument");
        profileStop(out);
    });
}

// ---- allocation-free Jacobi sweep (see include/prism_b200.h)
API int prism_jacobi_step_noalloc(int64_t n, const int32_t* rowptr, const int32_t* col, const double* values,
                                  const double* b, double* x, void* stream) {
    return guard([&] { jacobiStepNoAlloc(n, rowptr, col, values, b, x, static_cast<cudaStream_t>(stream)); });
}

// ---- steady fixed point and discrete adjoint (see include/prism_b200.h)
namespace {
void writeFixedPoint(const FixedPointOut& f, PrismFixedPointResult* r) {
    if (!r) return;
    r->outer_iterations = f.outer;
    r->krylov_iterations = f.krylov;
    r->final_change = f.change;
    r->converged = f.converged ? 1 : 0;
    r->status = f.status;
}
}  // namespace
API int prism_adjoint_forward(PrismTransport* pt, const PrismSolveOpts* o, int32_t max_outer, double outer_tol,
                              PrismFixedPointResult* r) {
    return guard([&] {
        ARG(pt && max_outer > 0 && outer_tol >= 0.0, "bad argument");
        FixedPointOut f = steadySolve(pt->eq, optsOrDefault(o), max_outer, outer_tol);
        sync(*pt->eq.phi->m);
        writeFixedPoint(f, r);
    });
}
API int prism_adjoint_backward(PrismTransport* pt, const double* dJ, double* gk, double* gv, const PrismSolveOpts* o,
                               int32_t max_outer, double outer_tol, PrismFixedPointResult* r) {
    return guard([&] {
        ARG(pt && dJ && gk && max_outer > 0 && outer_tol >= 0.0, "bad argument");
        FixedPointOut f = adjointBackward(pt->eq, dJ, gk, gv, optsOrDefault(o), max_outer, outer_tol);
        sync(*pt->eq.phi->m);
        writeFixedPoint(f, r);
    });
}

// ---- batched solves (see include/prism_b200.h)
API int prism_batch_create(PrismBatch** out) {
    return guard([&] {
        ARG(out, "null argument");
        *out = new PrismBatch();
    });
}
API void prism_batch_destroy(PrismBatch* b) { delete b; }
API int prism_batch_solve(PrismBatch* b, PrismTransport* const* eqs, int32_t n, const PrismSolveOpts* o,
                          PrismSolveResult* results) {
    return guard([&] {
        ARG(b && eqs && n > 0 && results, "bad argument");
        std::vector<Transport*> v;
        for (int32_t i = 0; i < n; ++i) {
            ARG(eqs[i], "null equation");
            v.push_back(&eqs[i]->eq);
        }
        auto r = solveBatch(b->h, v, optsOrDefault(o));
        for (int32_t i = 0; i < n; ++i) results[i] = r[i];
        for (auto* e : v) sync(*e->phi->m);
    });
}
