// runtime.cpp -- host side of the sm_100a path: mesh upload, gradient caches,
// eqn::Transport assembly / relax / solve and the SIMPLE, PRIME and PISO
// drivers. The control flow follows the reference call by call (file:line
// cited per function); every cell/face loop is a kernel on the mesh's stream.
#include "runtime.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "adjoint.h"
#include "coupling.h"
#include "diag.h"
#include "gradient.h"

namespace pb {

namespace {

struct H3 {
    double x, y, z;
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline H3 hsub(H3 a, H3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double hdot(H3 a, H3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

template <typename T>
void upload(DevBuf<T>& d, const std::vector<T>& h, cudaStream_t s) {
    d.alloc(h.size());
    d.upload(h.data(), h.size(), s);
}

bool scalarHasHandler(int k) {
    return k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP || k == PRISM_BC_SYMMETRY || k == PRISM_BC_OUTLET ||
           k == PRISM_BC_ZERO_GRADIENT;
}
bool vectorHasHandler(int k) { return scalarHasHandler(k); }
bool isDirichlet(int k) { return k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP; }

[[noreturn]] void noHandler(const Mesh& m, int p, const std::string& who) {
    fail(PRISM_NO_BC_HANDLER, who + ": no boundary handler for patch '" + m.h->patches[p].name + "'");
}

// patches whose faces a boundary loop visits
bool visited(const Mesh& m, int p) { return !m.h->patches[p].empty && !m.h->patches[p].faces.empty(); }

// Scalar::valueAtBoundaryFace would succeed on every visited patch (or on patch `only`)
void checkScalarValues(const Scalar& s, const std::string& who, int only = -1) {
    if (s.has_fv) return;
    const Mesh& m = *s.m;
    for (int p = 0; p < m.npatch; ++p) {
        if (!visited(m, p) || (only >= 0 && p != only)) continue;
        int k = s.bc[p].kind;
        if (!scalarHasHandler(k)) noHandler(m, p, who + " (field " + s.name + ")");
        if (isDirichlet(k)) {
            int want = s.coord >= 0 ? PRISM_BCV_VECTOR : PRISM_BCV_SCALAR;
            if (s.bc[p].value_kind != want)
                fail(PRISM_BAD_ARG, "patch '" + m.h->patches[p].name + "' field '" + s.name + "' value kind mismatch");
        }
    }
}
void checkVectorValues(const Vector& U, const std::string& who, int only = -1) {
    if (U.has_fd) return;
    const Mesh& m = *U.m;
    for (int p = 0; p < m.npatch; ++p) {
        if (!visited(m, p) || (only >= 0 && p != only)) continue;
        int k = U.bc[p].kind;
        if (!vectorHasHandler(k)) noHandler(m, p, who + " (field " + U.name + ")");
        if (isDirichlet(k) && U.bc[p].value_kind != PRISM_BCV_VECTOR)
            fail(PRISM_BAD_ARG, "patch '" + m.h->patches[p].name + "' field '" + U.name + "' is not a vector");
    }
}
void checkVectorFlux(const Vector& U, const std::string& who, int only = -1) {
    if (U.has_ff) return;
    const Mesh& m = *U.m;
    for (int p = 0; p < m.npatch; ++p) {
        if (!visited(m, p) || (only >= 0 && p != only)) continue;
        int k = U.bc[p].kind;
        if (k == PRISM_BC_NOSLIP || k == PRISM_BC_SYMMETRY) continue;
        if (!vectorHasHandler(k)) noHandler(m, p, who + " (field " + U.name + ")");
    }
    checkVectorValues(U, who, only);
}

}  // namespace

// ------------------------------------------------------------------ mesh
Mesh::~Mesh() {
    if (stream) cudaStreamSynchronize(stream);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph_host) cudaFreeHost(graph_host);
    if (stream) cudaStreamDestroy(stream);
}

MeshView Mesh::view() const {
    MeshView v;
    v.nc = nc;
    v.nf = nf;
    v.nb = nb;
    v.nne = nne;
    v.npatch = npatch;
    v.nslices = pat.nslices;
    v.owner = owner.p;
    v.nbr = nbr.p;
    v.bpatch = bpatch.p;
    v.patch_empty = patch_empty.p;
    v.area = area.p;
    v.nx = nx.p;
    v.ny = ny.p;
    v.nz = nz.p;
    v.fx = fx.p;
    v.fy = fy.p;
    v.fz = fz.p;
    v.cx = cx.p;
    v.cy = cy.p;
    v.cz = cz.p;
    v.vol = vol.p;
    v.gcw = gcw.p;
    v.cf_off = cf_off.p;
    v.cf_face = cf_face.p;
    v.cf_pos = nullptr;
    v.diag_pos = pat.diag_pos.p;
    v.sl_off = pat.sl_off.p;
    v.sl_col = pat.sl_col.p;
    return v;
}

SellMatrix Mesh::matrix(const double* vals) const {
    SellMatrix A;
    A.n = nc;
    A.nslices = pat.nslices;
    A.nnz_padded = pat.sell_nnz;
    A.sl_off = pat.sl_off.p;
    A.col = pat.sl_col.p;
    A.diag_pos = pat.diag_pos.p;
    A.vals = vals;
    A.nnz_csr = pat.nnz;
    return A;
}

namespace {
// device copy of the host mesh, the matrix pattern and the Green-Gauss schedule
void setupDevice(Mesh& m) {
    HostMesh& h = *m.h;
    cudaStream_t s = m.stream;
    m.nc = (int)h.nc;
    m.nf = (int)h.nf;
    m.nb = (int)h.nb;
    m.nne = (int)h.nne;
    m.npatch = (int)h.patches.size();
    m.n_pad = ceil_div(m.nc, 32) * 32;
    upload(m.owner, h.owner, s);
    upload(m.nbr, h.nbr, s);
    std::vector<int> bp(h.patch.begin(), h.patch.begin() + h.nb), ppos(h.nb, 0);
    for (auto& pa : h.patches)
        for (size_t i = 0; i < pa.faces.size(); ++i) ppos[pa.faces[i]] = (int)i;
    upload(m.bpatch, bp.empty() ? std::vector<int>{0} : bp, s);
    upload(m.ppos, ppos.empty() ? std::vector<int>{0} : ppos, s);
    std::vector<unsigned char> pe(std::max(1, m.npatch), 0);
    for (int p = 0; p < m.npatch; ++p) pe[p] = h.patches[p].empty ? 1 : 0;
    upload(m.patch_empty, pe, s);
    upload(m.area, h.area, s);
    upload(m.nx, h.normal[0], s);
    upload(m.ny, h.normal[1], s);
    upload(m.nz, h.normal[2], s);
    upload(m.fx, h.fc[0], s);
    upload(m.fy, h.fc[1], s);
    upload(m.fz, h.fc[2], s);
    upload(m.cx, h.cc[0], s);
    upload(m.cy, h.cc[1], s);
    upload(m.cz, h.cc[2], s);
    upload(m.vol, h.vol, s);
    upload(m.gcw, h.gc.empty() ? std::vector<double>{0.0} : h.gc, s);
    std::vector<int> cfo(h.cf_off.begin(), h.cf_off.end());
    upload(m.cf_off, cfo, s);
    upload(m.cf_face, h.cf_face, s);

    PatternInput pin{m.nc, m.nb, m.npatch, (int64_t)h.cf_face.size(), m.cf_off.p, m.cf_face.p,
                     m.owner.p, m.nbr.p, m.bpatch.p, m.ppos.p, m.nf};
    buildPattern(pin, m.pat, s);

    // Green-Gauss schedule: level[c] = 1 + max(level of lower-numbered neighbours)
    std::vector<int> level(m.nc, 0);
    int nl = 0;
    for (int c = 0; c < m.nc; ++c) {
        int l = 0;
        for (int64_t q = h.cf_off[c]; q < h.cf_off[c + 1]; ++q) {
            int f = h.cf_face[q];
            if (f < m.nb) continue;
            int o = h.owner[f];
            int n = (o == c) ? h.nbr[f] : o;
            if (n < c) l = std::max(l, level[n] + 1);
        }
        level[c] = l;
        nl = std::max(nl, l + 1);
    }
    m.level_off.assign(nl + 1, 0);
    for (int c = 0; c < m.nc; ++c) m.level_off[level[c] + 1]++;
    for (int l = 0; l < nl; ++l) m.level_off[l + 1] += m.level_off[l];
    std::vector<int> lc(m.nc), fill(m.level_off.begin(), m.level_off.end() - 1);
    for (int c = 0; c < m.nc; ++c) lc[fill[level[c]]++] = c;
    upload(m.level_cells, lc, s);
    m.scratch.alloc(std::max(3 * m.nf, 1));
    m.ls_ready = false;
    m.points_ready = false;
    PB_CUDA(cudaStreamSynchronize(s));
}
}  // namespace

// The CSR and SELL-32 patterns number their entries with 32-bit ints: bound both for the
// current cell numbering (a row holds the cell and at most one entry per interior face of
// the cell; SELL pads every 32-row slice to its longest row, so the count depends on the
// numbering and is checked again after a renumbering).
void checkPatternBounds(const HostMesh& h) {
    constexpr int64_t LIMIT = int64_t(1) << 31;
    int64_t nnz = 0, sell = 0;
    for (int64_t s0 = 0; s0 < h.nc; s0 += 32) {
        int64_t width = 0;
        for (int64_t c = s0; c < std::min(s0 + 32, h.nc); ++c) {
            int64_t len = 1;
            for (int64_t k = h.cf_off[c]; k < h.cf_off[c + 1]; ++k) len += h.cf_face[k] >= h.nb;
            nnz += len;
            width = std::max(width, len);
        }
        sell += 32 * width;
    }
    if (nnz >= LIMIT || sell >= LIMIT) fail(PRISM_INVALID_MESH, "matrix pattern too large for 32-bit indices");
}

std::unique_ptr<Mesh> createMesh(const PrismUnvMesh* d) {
    auto mesh = std::make_unique<Mesh>();
    mesh->h = buildHostMesh(d);
    const HostMesh& h = *mesh->h;
    constexpr int64_t LIMIT = int64_t(1) << 31;
    if (h.nc >= LIMIT || h.nf >= LIMIT || (int64_t)h.cf_face.size() >= LIMIT)
        fail(PRISM_INVALID_MESH, "mesh too large for 32-bit indices");
    checkPatternBounds(h);
    PB_CUDA(cudaStreamCreateWithFlags(&mesh->stream, cudaStreamNonBlocking));
    setupDevice(*mesh);
    return mesh;
}

// CuthillMckee(mesh).reorder(reverse) (reorder.cpp:89-129); nothing on the
// device refers to the old numbering yet (no fields exist), so the device copy
// is rebuilt from the permuted host mesh
void reorderMesh(Mesh& m, bool reverse) {
    if (m.frozen) fail(PRISM_BAD_ARG, "reorder the mesh before creating fields on it");
    std::vector<int64_t> perm = cuthillMckee(*m.h);
    if (reverse) std::reverse(perm.begin(), perm.end());
    permuteCells(*m.h, perm);
    checkPatternBounds(*m.h);
    setupDevice(m);
}

// LeastSquares::setPseudoInvMatrices (least_squares.cpp:12-61): pinv = (D^T D)^-1 D^T
void Mesh::ensureLeastSquares() {
    if (ls_ready) return;
    const HostMesh& H = *h;
    const int64_t nk = (int64_t)H.cf_face.size();
    std::vector<double> pinv(9 * (size_t)nc), w(3 * (size_t)nk, 0.0);
    for (int c = 0; c < nc; ++c) {
        double D[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        H3 xc{H.cc[0][c], H.cc[1][c], H.cc[2][c]};
        for (int64_t q = H.cf_off[c]; q < H.cf_off[c + 1]; ++q) {
            int f = H.cf_face[q];
            H3 r;
            if (f >= nb) {
                int o = H.owner[f];
                int n = (o == c) ? H.nbr[f] : o;
                r = hsub(H3{H.cc[0][n], H.cc[1][n], H.cc[2][n]}, xc);
            } else {
                r = hsub(H3{H.fc[0][f], H.fc[1][f], H.fc[2][f]}, xc);
            }
            double wk = 1 / (std::sqrt(hdot(r, r)) + EPSILON);
            H3 wd{r.x * wk, r.y * wk, r.z * wk};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) D[i][j] += wd[i] * r[j];
            w[q] = wd.x;
            w[nk + q] = wd.y;
            w[2 * nk + q] = wd.z;
        }
        double P[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) P[i][j] = (D[0][i] * D[0][j] + D[1][i] * D[1][j]) + D[2][i] * D[2][j];
        double c00 = P[1][1] * P[2][2] - P[1][2] * P[2][1];
        double c10 = P[1][2] * P[2][0] - P[1][0] * P[2][2];
        double c20 = P[1][0] * P[2][1] - P[1][1] * P[2][0];
        double det = (P[0][0] * c00 + P[0][1] * c10) + P[0][2] * c20;
        double I[3][3];
        I[0][0] = c00 / det;
        I[1][0] = c10 / det;
        I[2][0] = c20 / det;
        I[0][1] = (P[0][2] * P[2][1] - P[0][1] * P[2][2]) / det;
        I[1][1] = (P[0][0] * P[2][2] - P[0][2] * P[2][0]) / det;
        I[2][1] = (P[0][1] * P[2][0] - P[0][0] * P[2][1]) / det;
        I[0][2] = (P[0][1] * P[1][2] - P[0][2] * P[1][1]) / det;
        I[1][2] = (P[0][2] * P[1][0] - P[0][0] * P[1][2]) / det;
        I[2][2] = (P[0][0] * P[1][1] - P[0][1] * P[1][0]) / det;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)  // (I * D^T)(i,j) = sum_k I(i,k) D(j,k)
                pinv[(3 * i + j) * (size_t)nc + c] = (I[i][0] * D[j][0] + I[i][1] * D[j][1]) + I[i][2] * D[j][2];
    }
    upload(ls_pinv, pinv, stream);
    upload(ls_w, w, stream);
    PB_CUDA(cudaStreamSynchronize(stream));
    ls_ready = true;
}

// ------------------------------------------------------------------ fields
ScalarView Scalar::view() const {
    ScalarView v;
    v.v = this->v.p;
    v.fv = has_fv ? fv.p : nullptr;
    v.g = grad->g.p;
    v.gstride = m->n_pad;
    v.bc_kind = bc_kind.p;
    v.bc_val = bc_val.p;
    v.bc_vec = bc_vec.p;
    return v;
}
VectorView Vector::view() const {
    VectorView v;
    for (int k = 0; k < 3; ++k) v.c[k] = c[k]->view();
    v.fd = has_fd ? fd.p : nullptr;
    v.ff = has_ff ? ff.p : nullptr;
    v.bc_kind = bc_kind.p;
    v.bc_vec = bc_vec.p;
    return v;
}

// IGradient::computeAllCellGradients (green_gauss.cpp:40-45, least_squares.cpp:71-76)
void computeGradient(Scalar& s) {
    Mesh& m = *s.m;
    checkScalarValues(s, "IGradient::computeAllCellGradients()");
    if (s.grad->type == PRISM_GRAD_LEAST_SQUARES) {
        m.ensureLeastSquares();
        launchLeastSquares(m.view(), s.view(), m.ls_pinv.p, m.ls_w.p, (int64_t)m.h->cf_face.size(), m.stream);
    } else {
        launchGreenGauss(m.view(), s.view(), m.level_cells.p, m.level_off, m.stream);
    }
    s.grad->computed = s.event;
}
// gradAtCell lazy cache by event number (green_gauss.cpp:32-38)
void ensureGradient(Scalar& s) {
    if (s.event != s.grad->computed) computeGradient(s);
}

// ------------------------------------------------------------------ time-step history
// HistoryManager::resize (history.cpp:48-60)
void setHistorySize(Scalar& s, size_t n) {
    if (n == s.hist_max) return;
    if (n < s.hist.size()) s.hist.resize(n);
    s.hist_max = n;
}
// HistoryManager::update (history.cpp:28-46): the current values become step 0;
// the oldest buffer is reused once the history is full
void updatePrevTimeSteps(Scalar& s) {
    if (s.hist_max == 0) return;
    Mesh& m = *s.m;
    DevBuf<double> front;
    if (s.hist.size() == s.hist_max) {
        front = std::move(s.hist.back());
        s.hist.pop_back();
    } else {
        front.alloc(m.n_pad);
        front.zero(m.stream);
    }
    PB_CUDA(cudaMemcpyAsync(front.p, s.v.p, m.nc * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
    s.hist.insert(s.hist.begin(), std::move(front));
}

// ------------------------------------------------------------------ transport
void Transport::ensure() {
    Mesh& m = *phi->m;
    if (!A) {
        // each array starts on a 256-byte boundary
        auto up = [](size_t k) { return (k + 31) / 32 * 32; };
        const size_t na = up(m.pat.sell_nnz), nv = up(m.n_pad);
        store.alloc(na + 3 * nv);
        store.zero(m.stream);
        A = {store.p, (size_t)m.pat.sell_nnz};
        b = {store.p + na, (size_t)m.n_pad};
        bconv = {store.p + na + nv, (size_t)m.n_pad};
        bdiff = {store.p + na + 2 * nv, (size_t)m.n_pad};
    }
}

// Transport::updateCoeffs (transport.cpp:4-21)
void updateCoeffs(Transport& eq) {
    Scalar& phi = *eq.phi;
    Mesh& m = *phi.m;
    eq.ensure();
    const bool has_interior = m.nf > m.nb;
    bool need_grad = false;
    // boundary handlers of the schemes (convection_boundary.cpp, diffusion_boundary.h)
    for (int p = 0; p < m.npatch; ++p) {
        if (!visited(m, p)) continue;
        const int k = phi.bc[p].kind;
        if (eq.has_conv) {
            if (k == PRISM_BC_FIXED) {
                int want = phi.coord >= 0 ? PRISM_BCV_VECTOR : PRISM_BCV_SCALAR;
                if (phi.bc[p].value_kind != want)
                    fail(PRISM_BAD_ARG, "patch '" + m.h->patches[p].name + "' value kind mismatch for " + phi.name);
                checkVectorFlux(*eq.U, "IConvection Fixed handler", p);
            } else if (k == PRISM_BC_OUTLET || k == PRISM_BC_ZERO_GRADIENT) {
                checkVectorValues(*eq.U, "IConvection Outlet handler", p);
            } else if (k != PRISM_BC_NOSLIP && k != PRISM_BC_SYMMETRY) {
                noHandler(m, p, "applyBoundary() applied by IConvection");
            }
        }
        if (eq.has_diff) {
            if (k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP) {
                checkScalarValues(phi, "diffusion Fixed handler", p);
                if (eq.corrected) need_grad = true;
            } else if (k == PRISM_BC_FIXED_GRADIENT) {
                if (phi.coord >= 0)
                    fail(PRISM_BAD_ARG, "patch '" + m.h->patches[p].name + "' does not have a field named '" + phi.name + "'");
                if (phi.bc[p].value_kind != PRISM_BCV_VECTOR)
                    fail(PRISM_BAD_ARG, "patch '" + m.h->patches[p].name + "' field is not a vector");
            } else if (k != PRISM_BC_SYMMETRY && k != PRISM_BC_OUTLET && k != PRISM_BC_ZERO_GRADIENT) {
                noHandler(m, p, "applyBoundary() applied by a diffusion scheme");
            }
        }
    }
    if (has_interior && (eq.has_conv || (eq.has_diff && eq.corrected))) need_grad = true;
    if (need_grad) ensureGradient(phi);
    if (eq.symmetry && (!eq.has_conv || !eq.has_diff || phi.coord < 0))
        fail(PRISM_BAD_ARG, "Symmetry<Transport> needs a convection and a diffusion scheme on a vector component");
    AssembleParams P{};
    P.m = m.view();
    P.phi = phi.view();
    P.phi_coord = phi.coord;
    P.has_conv = eq.has_conv;
    P.has_diff = eq.has_diff;
    P.conv_first = eq.conv_first;
    P.nsch = eq.nsch;
    for (int k = 0; k < eq.nsch; ++k) P.order[k] = eq.order[k];
    if (eq.has_temporal) {
        // BackwardEuler::applyIncompressible (backward_euler.cpp:62-76), AdamMoulton (adam_moulton.cpp:62-91)
        if (phi.hist.empty())
            fail(PRISM_BAD_ARG, std::string("prism::scheme::temporal::") +
                                    (eq.temporal_kind == PRISM_TEMPORAL_BACKWARD_EULER ? "BackwardEuler" : "AdamMoulton") +
                                    "::apply() was called for field `" + phi.name +
                                    "`, but the field does not have any previous time step values stored.");
        P.has_temporal = 1;
        P.tm.dt = eq.dt;
        P.tm.prev = phi.hist[0].p;
        P.tm.second_order = (eq.temporal_kind == PRISM_TEMPORAL_ADAM_MOULTON && phi.hist.size() >= 2) ? 1 : 0;
        P.tm.prev2 = P.tm.second_order ? phi.hist[1].p : nullptr;
    }
    P.need_grad = need_grad ? 1 : 0;
    if (eq.has_conv) {
        P.conv.scheme = eq.conv_scheme;
        P.conv.U = eq.U->view();  // interior faces interpolate cell values: no handler needed
    }
    if (eq.has_diff) {
        P.diff.corrected = eq.corrected;
        P.diff.corrector = eq.corrector;
        P.diff.kappa_tensor = eq.kt ? 1 : 0;
        if (eq.ks) P.diff.ks = eq.ks->view();  // kappa is read at cells and interior faces only
        if (eq.kt) P.diff.kt = eq.kt->view();
    }
    if ((int)eq.sources.size() > MAX_SOURCES) fail(PRISM_BAD_ARG, "too many sources");
    P.nsrc = (int)eq.sources.size();
    for (size_t i = 0; i < eq.sources.size(); ++i) {
        Source& src = eq.sources[i];
        SourceDesc& S = P.src[i];
        S.kind = src.kind;
        S.sign = src.sign;
        S.coord = src.coord;
        if (src.kind == PRISM_SRC_CONSTANT) {
            ++src.s->event;  // values() non-const (constant_scalar.h:31)
            S.s = src.s->view();
        } else if (src.kind == PRISM_SRC_GRADIENT) {
            ensureGradient(*src.s);
            S.s = src.s->view();
        } else {
            checkVectorFlux(*src.U, "ops::div()");
            S.U = src.U->view();
        }
    }
    P.symmetry = eq.symmetry ? 1 : 0;
    P.accumulate = eq.clean ? 0 : 1;
    P.ca_off = m.cf_off.p;
    P.ca_face = m.pat.ca_face.p;
    P.ca_pos = m.pat.ca_pos.p;
    P.face_slot = m.pat.face_slot.p;
    P.face_pos = m.pat.face_pos.p;
    if (!m.asm_rec.p) {
        // records of empty-patch faces are never written and stay zero
        m.asm_rec.alloc(4 * std::max<size_t>(m.h->cf_face.size(), 1));
        m.asm_rec.zero(m.stream);
    }
    P.rec = m.asm_rec.p;
    P.A = eq.A.p;
    P.b = eq.b.p;
    P.bconv = eq.bconv.p;
    P.bdiff = eq.bdiff.p;
    launchAssemble(P, m.stream);
    eq.clean = false;
}

// Transport::relax (transport.cpp:54-64)
void relax(Transport& eq) {
    Mesh& m = *eq.phi->m;
    eq.ensure();
    ++eq.phi->event;
    launchRelax(eq.A.p, eq.b.p, m.pat.diag_pos.p, eq.phi->v.p, eq.urf, m.nc, m.stream);
}

// Transport::zeroOutCoeffs (transport.cpp:23-36)
void zeroOutCoeffs(Transport& eq) {
    Mesh& m = *eq.phi->m;
    eq.ensure();
    eq.A.zero(m.stream);
    eq.b.zero(m.stream);
    eq.bconv.zero(m.stream);
    eq.bdiff.zero(m.stream);
    eq.clean = true;
}

void solveDefaults(PrismSolveOpts* o) {
    std::memset(o, 0, sizeof(*o));
    o->method = PRISM_SOLVER_BICGSTAB;
    o->precision = PRISM_PREC_FP64;
    o->n_iter = 10;
    o->eps = 1e-7;
    o->ref_cell = -1;
    o->clear_coeffs = 1;
}

int choosePreconditioner(int pc, int64_t n) {
    if (pc == PRISM_PC_AUTO) return n >= PRISM_PC_AUTO_MIN_ROWS ? PRISM_PC_AMG : PRISM_PC_JACOBI;
    if (pc != PRISM_PC_JACOBI && pc != PRISM_PC_AMG) fail(PRISM_BAD_ARG, "unknown preconditioner");
    return pc;
}

// Amg::values_current for one solve (cleared however the solve ends)
struct HoldAmgValues {
    Amg* a;
    HoldAmgValues(Amg* amg, bool on) : a(amg) {
        if (a) a->values_current = on;
    }
    ~HoldAmgValues() {
        if (a) a->values_current = false;
    }
};

// PRISM_PC_AUTO at AMG sizes: an equation whose off-diagonal row sums stay below this
// fraction of the diagonal (an under-relaxed momentum predictor: about the relaxation
// factor) is solved with Jacobi, whose iteration then converges fast and costs a third
// of an AMG one; PRISM_PC_AUTO_JACOBI overrides it (0: always AMG). The spd pressure
// correction keeps AMG.
static double autoJacobiRatio() {
    static const double v = [] {
        const char* e = std::getenv("PRISM_PC_AUTO_JACOBI");
        return e && e[0] ? std::atof(e) : 0.8;
    }();
    return v;
}

// preconditioner of a solve of eq (A: its assembled matrix); measures and records the
// automatic choice on the first solve (a host round trip, never inside a capture)
static int pcFor(Transport& eq, const PrismSolveOpts& o, const SellMatrix& A) {
    const int c = choosePreconditioner(o.preconditioner, A.n);
    if (o.preconditioner != PRISM_PC_AUTO || c != PRISM_PC_AMG || eq.spd || autoJacobiRatio() <= 0.0) return c;
    if (eq.auto_pc == 0) {
        Mesh& m = *eq.phi->m;
        if (capturing(m.stream)) fail(PRISM_INTERNAL, "automatic preconditioner not chosen before capture");
        const double t = offDiagonalRatio(A, m.kw, m.stream);
        eq.auto_pc = t <= autoJacobiRatio() ? PRISM_PC_JACOBI : PRISM_PC_AMG;
        if (verbose())
            std::fprintf(stderr, "[prism] automatic preconditioner of %s: %s (off-diagonal ratio %.3f)\n",
                         eq.phi->name.c_str(), eq.auto_pc == PRISM_PC_AMG ? "AMG" : "Jacobi", t);
    }
    return eq.auto_pc;
}

// FP64 AMG solves of an spd equation run flexible CG; PRISM_PRESSURE_SOLVER=bicgstab
// keeps BiCGSTAB with the V-cycle for them
static bool flexibleFor(const Transport& eq, const PrismSolveOpts& o, const Amg* amg) {
    static const bool on = [] {
        const char* e = std::getenv("PRISM_PRESSURE_SOLVER");
        return !(e && std::strcmp(e, "bicgstab") == 0);
    }();
    if (o.method == PRISM_SOLVER_FCG) return true;
    return on && eq.spd && amg && o.method == PRISM_SOLVER_BICGSTAB && o.precision == PRISM_PREC_FP64;
}

// PRISM_SOLVER_FCG's requirements: FP64, and the AMG preconditioner (its own choice
// under PRISM_PC_AUTO)
static void checkFcg(const PrismSolveOpts& o) {
    if (o.method != PRISM_SOLVER_FCG) return;
    if (o.precision != PRISM_PREC_FP64) fail(PRISM_BAD_ARG, "flexible CG runs in FP64 (precision PRISM_PREC_FP64)");
    if (o.preconditioner == PRISM_PC_JACOBI) fail(PRISM_BAD_ARG, "flexible CG needs the AMG preconditioner");
}

namespace {
// set while a solve or step is being captured into a graph (graph_capture below)
struct GraphCapture {
    Mesh* m = nullptr;
    int used = 0;
};
thread_local GraphCapture* g_capture = nullptr;
constexpr int GRAPH_SLOTS = 256;  // captured solves per graph
PrismSolveResult solveCaptured(Transport& eq, const PrismSolveOpts& o);
}  // namespace

// ISolver::solve (numerics/solver.cpp:27-82)
PrismSolveResult solve(Transport& eq, const PrismSolveOpts& o) {
    checkFcg(o);
    if (g_capture) return solveCaptured(eq, o);
    Scalar& phi = *eq.phi;
    Mesh& m = *phi.m;
    updateCoeffs(eq);
    relax(eq);
    if (o.ref_cell >= 0 && o.ref_cell < m.nc) {
        int pos = 0;
        PB_CUDA(cudaMemcpyAsync(&pos, m.pat.diag_pos.p + o.ref_cell, sizeof(int), cudaMemcpyDeviceToHost, m.stream));
        PB_CUDA(cudaStreamSynchronize(m.stream));
        launchPin(eq.A.p, eq.b.p, pos, (int)o.ref_cell, o.ref_value, m.stream);
    }
    SellMatrix A = m.matrix(eq.A.p);
    const double ktol = o.krylov_tol > 0 ? o.krylov_tol : 1e-12;
    const long long kmax = o.krylov_max_iter > 0 ? o.krylov_max_iter : 2LL * m.nc;
    const double itol = o.inner_tol > 0 ? o.inner_tol : 0.1;
    Amg* amg = nullptr;
    if (o.method == PRISM_SOLVER_FCG || (o.method != PRISM_SOLVER_JACOBI && pcFor(eq, o, A) == PRISM_PC_AMG)) {
        if (!eq.amg) eq.amg = std::make_shared<Amg>();
        amg = eq.amg.get();
    }
    PrismSolveResult r{};
    r.status = PRISM_OK;
    double init_res = 0.0, cur = 0.0;
    bool conv = false;
    int64_t iter = 0;
    for (; iter < o.n_iter; ++iter) {
        if (iter == 0) {
            ++phi.event;
            init_res = scaledResidual(A, eq.b.p, phi.v.p, m.kw, m.stream);
        }
        phi.event += 2;
        if (o.method == PRISM_SOLVER_JACOBI) {
            jacobiStep(A, eq.b.p, phi.v.p, m.kw, m.stream);
        } else {
            const HoldAmgValues hold(amg, eq.matrix_unchanged || iter > 0);  // A is fixed within one solve
            KrylovOut k = bicgstab(A, eq.b.p, phi.v.p, ktol, kmax, o.precision, itol, m.kw, m.stream, amg,
                                   m.pat.rowptr.p, m.pat.col.p, flexibleFor(eq, o, amg));
            r.krylov_iterations += k.iterations;
            r.krylov_rel_residual = k.rel_residual;
            if (k.status != PRISM_OK && r.status == PRISM_OK) r.status = k.status;
        }
        ++phi.event;
        cur = scaledResidual(A, eq.b.p, phi.v.p, m.kw, m.stream);
        if (std::isnan(cur)) r.status = PRISM_NONFINITE;
        if (cur < o.eps) {
            conv = true;
            ++iter;
            break;
        }
    }
    if (o.clear_coeffs) zeroOutCoeffs(eq);
    r.iterations = iter;
    r.initial_residual = init_res;
    r.final_residual = cur;
    r.converged = conv ? 1 : 0;
    return r;
}

// ------------------------------------------------------------------ SIMPLE / PRIME / PISO
void simpleDefaults(PrismSIMPLEControls* c) {  // SIMPLEControls, SIMPLE.h:14-43
    c->momentum_urf = 0.7;
    c->momentum_max_iter = 3;
    c->momentum_residual = 1e-7;
    c->momentum_residual_stop = 1e-5;
    c->non_ortho_correctors = 2;
    c->pressure_urf = 0.3;
    c->pressure_max_iter = 5;
    c->pressure_residual = 1e-7;
    c->p_ref_cell = -1;
    c->p_ref_value = 0.0;
    c->batched_momentum = 0;
}
void pisoDefaults(PrismPISOControls* c) {  // PISOControls, PISO.h:11-49
    c->outer_iterations = 1;
    c->momentum_implicit_steps = 1;
    c->pressure_correction_steps = 2;
    c->momentum_urf = 1.0;
    c->momentum_max_iter = 3;
    c->momentum_residual = 1e-4;
    c->momentum_residual_stop = 1e-5;
    c->non_ortho_correctors = 2;
    c->pressure_urf = 1.0;
    c->pressure_max_iter = 5;
    c->pressure_residual = 1e-4;
    c->p_ref_cell = -1;
    c->p_ref_value = 0.0;
    c->batched_momentum = 0;
}

// mdot.mapFaceValues(U.valueAtFace); mdot.mapInteriorFaceValues(rhieChowCorrectFace)
// (SIMPLE.cpp:136-138, operations/rhie_chow.h:47-63)
void rhieChowFaces(Vector& mdot, Vector& U, const Tensor& D, Scalar& p) {
    Mesh& m = *p.m;
    checkVectorFlux(mdot, "GeneralVector::initFaceData()");
    checkVectorValues(U, "GeneralVector::valueAtFace()");
    if (m.nf > m.nb) ensureGradient(p);
    if (!mdot.fd) mdot.fd.alloc(3 * (size_t)std::max(m.nf, 1));
    if (!mdot.ff) mdot.ff.alloc(std::max(m.nf, 1));
    launchRhieChow(m.view(), U.view(), D.view(), p.view(), mdot.fd.p, mdot.ff.p, m.stream);
    mdot.has_fd = mdot.has_ff = true;
}

namespace {

PrismSolveOpts inner(const PrismSolveOpts& so, int64_t n_iter, double eps, int64_t ref, double refv, bool clear) {
    PrismSolveOpts o = so;
    o.method = PRISM_SOLVER_BICGSTAB;
    o.n_iter = n_iter;
    o.eps = eps;
    o.ref_cell = ref;
    o.ref_value = refv;
    o.clear_coeffs = clear ? 1 : 0;
    return o;
}

// PRISM_VERBOSE: wall time of a scope, the stream drained at both ends
struct PhaseTimer {
    std::string what;
    cudaStream_t s;
    std::chrono::steady_clock::time_point t0;
    bool on = false;
    PhaseTimer(std::string w, cudaStream_t st) : what(std::move(w)), s(st) {
        on = verbose() && !capturing(st);
        if (!on) return;
        cudaStreamSynchronize(s);
        t0 = std::chrono::steady_clock::now();
    }
    ~PhaseTimer() {
        if (!on) return;
        cudaStreamSynchronize(s);
        std::fprintf(stderr, "[prism] phase %s: %.3f ms\n", what.c_str(),
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
};

void setURF(Transport& eq, double f) {  // transport.cpp:38-52: out-of-range values are ignored
    if (f < 0.0 || f > 1.0) return;
    eq.urf = f;
}

// solveImplicitMomentum, SIMPLE.cpp:19-41. With batched_momentum every component
// is assembled and relaxed as usual and the systems are then solved together in
// one persistent launch (one step each, to the Krylov tolerance).
void solveImplicitMomentum(const PrismSIMPLEControls& c, std::vector<Transport*>& mom, const PrismSolveOpts& so,
                           std::vector<Report>& rep) {
    if (c.batched_momentum) {
        for (auto* eq : mom) setURF(*eq, c.momentum_urf);
        Mesh& m = *mom[0]->phi->m;
        if (!m.mom_batch) m.mom_batch = std::make_unique<BatchHandle>();
        PhaseTimer pt("momentum (batched)", m.stream);
        auto res = solveBatch(*m.mom_batch, mom, inner(so, c.momentum_max_iter, c.momentum_residual, -1, 0.0, false));
        for (size_t i = 0; i < mom.size(); ++i)
            rep.push_back({mom[i]->phi->name, res[i].iterations, res[i].initial_residual, res[i].final_residual,
                           res[i].converged != 0});
        return;
    }
    for (auto* eq : mom) {
        setURF(*eq, c.momentum_urf);
        PhaseTimer pt("momentum " + eq->phi->name, eq->phi->m->stream);
        auto r = solve(*eq, inner(so, c.momentum_max_iter, c.momentum_residual, -1, 0.0, false));
        rep.push_back({eq->phi->name, r.iterations, r.initial_residual, r.final_residual, r.converged != 0});
    }
}

struct PressureResult {
    Scalar* pp;
    Tensor* D;
};

// solvePressureEquation, SIMPLE.cpp:124-196. The reference builds p', the D
// tensor and the pressure equation afresh on every call; here they live in the
// mesh and are reset to exactly that fresh state (zero values, p's boundary
// conditions, a new gradient cache, cleared coefficients), which keeps their
// device buffers -- and the solver's captured iteration graphs -- across steps.
PressureResult solvePressureEquation(PrismSIMPLEControls c, std::vector<Transport*>& mom, Vector& U, Vector& mdot,
                                     Scalar& p, const PrismSolveOpts& so, std::vector<Report>& rep) {
    Mesh& m = *p.m;
    for (auto* eq : mom) eq->ensure();
    // pressureEquationCoeffsTensor, SIMPLE.cpp:77-108
    if (!m.p_D) {
        m.p_D = std::make_unique<Tensor>();
        m.p_D->m = &m;
        m.p_D->diag = 1;
        m.p_D->d.alloc(3 * (size_t)m.n_pad);
    }
    Tensor* D = m.p_D.get();
    D->d.zero(m.stream);
    launchDTensor(m.nc, m.pat.diag_pos.p, m.vol.p, mom[0]->A.p, mom[1]->A.p, mom.size() == 3 ? mom[2]->A.p : nullptr,
                  D->d.p, m.n_pad, m.stream);
    for (auto* eq : mom) zeroOutCoeffs(*eq);
    rhieChowFaces(mdot, U, *D, p);
    // p' named like p, zero valued, with a fresh gradient scheme (scalar.cpp:260-304)
    if (!m.p_corr) {
        m.p_corr = std::make_unique<Scalar>();
        Scalar& q = *m.p_corr;
        q.m = &m;
        q.coord = -1;
        q.v.alloc(m.n_pad);
        q.bc_kind.alloc(std::max(m.npatch, 1));
        q.bc_val.alloc(std::max(m.npatch, 1));
        q.bc_vec.alloc(3 * std::max(m.npatch, 1));
        q.grad = std::make_shared<GradState>();
        q.grad->g.alloc(3 * (size_t)m.n_pad);
        q.fv.alloc(std::max(m.nf, 1));
    }
    Scalar* pp = m.p_corr.get();
    pp->name = p.name;
    pp->bc = p.bc;
    pp->event = 0;
    pp->v.zero(m.stream);
    PB_CUDA(cudaMemcpyAsync(pp->bc_kind.p, p.bc_kind.p, pp->bc_kind.n * sizeof(int), cudaMemcpyDeviceToDevice, m.stream));
    PB_CUDA(cudaMemcpyAsync(pp->bc_val.p, p.bc_val.p, pp->bc_val.n * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
    PB_CUDA(cudaMemcpyAsync(pp->bc_vec.p, p.bc_vec.p, pp->bc_vec.n * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
    pp->grad->type = p.grad->type;
    pp->grad->computed = std::numeric_limits<uint64_t>::max();
    pp->grad->g.zero(m.stream);
    // constrainPPrime, SIMPLE.cpp:43-75: every face value is 0 (Dirichlet/symmetry patches
    // are zeroed, the others take the owner value of the zero field)
    for (int q = 0; q < m.npatch; ++q)
        if (!m.h->patches[q].empty && !scalarHasHandler(pp->bc[q].kind)) noHandler(m, q, "prism::algo::constrainPPrime()");
    pp->fv.zero(m.stream);
    pp->has_fv = true;
    if (c.p_ref_cell < 0 && needsPressureReference(*pp)) c.p_ref_cell = 0;
    if (!m.p_eq) m.p_eq = std::make_unique<Transport>();
    Transport& pEqn = *m.p_eq;
    pEqn.phi = pp;
    pEqn.has_conv = 0;
    pEqn.conv_scheme = 0;
    pEqn.conv_first = 1;
    pEqn.has_temporal = 0;
    pEqn.nsch = 1;
    pEqn.order[0] = SCH_DIFF;
    pEqn.has_diff = 1;
    pEqn.corrected = 1;
    pEqn.corrector = PRISM_CORR_OVER_RELAXED;
    pEqn.U = nullptr;
    pEqn.ks = nullptr;
    pEqn.kt = D;
    pEqn.sources.clear();
    pEqn.sources.push_back({PRISM_SRC_DIVERGENCE, PRISM_SIGN_NEGATIVE, 0, nullptr, &mdot});
    pEqn.symmetry = false;
    pEqn.urf = 1.0;
    pEqn.ensure();
    zeroOutCoeffs(pEqn);
    if (!m.p_amg) {
        m.p_amg = std::make_shared<Amg>();
        m.p_amg->forPressure();
    }
    pEqn.amg = m.p_amg;
    pEqn.spd = true;
    for (int64_t i = 0; i <= c.non_ortho_correctors; ++i) {
        PhaseTimer pt("pressure corrector " + std::to_string(i), m.stream);
        // the correctors re-assemble the same matrix (D and the mesh are fixed; only the
        // explicit non-orthogonal part of b changes)
        struct Unchanged {
            Transport& e;
            Unchanged(Transport& t, bool on) : e(t) { e.matrix_unchanged = on; }
            ~Unchanged() { e.matrix_unchanged = false; }
        } unchanged(pEqn, i > 0);
        auto r = solve(pEqn, inner(so, c.pressure_max_iter, c.pressure_residual, c.p_ref_cell, c.p_ref_value, true));
        rep.push_back({pp->name + "_corr_" + std::to_string(i), r.iterations, r.initial_residual, r.final_residual,
                       r.converged != 0});
    }
    pp->has_fv = false;  // clearFaceValues
    return {pp, D};
}

// correctFields, SIMPLE.cpp:218-241
void correctFields(Vector& U, Vector& mdot, Scalar& p, const Tensor& D, Scalar& pp, double urf) {
    Mesh& m = *U.m;
    ensureGradient(pp);
    updatePrevTimeSteps(p);  // p->update(...) keeps the old values in p's history (scalar.cpp:311-320)
    launchCorrectFields(m.view(), U.c[0]->view(), U.c[1]->view(), U.c[2]->view(), D.view(), pp.view(), mdot.fd.p,
                        mdot.ff.p, p.v.p, urf, m.stream);
    for (auto& c : U.c) ++c->event;
    p.event += 2;
    p.has_fv = false;
}

// solveExplicitMomentum, PRIME.cpp:39-56
void solveExplicitMomentum(std::vector<Transport*>& mom) {
    for (auto* eq : mom) {
        updateCoeffs(*eq);
        Mesh& m = *eq->phi->m;
        m.kw.ensure(m.n_pad, m.pat.sell_nnz, false);
        explicitUpdate(m.matrix(eq->A.p), eq->b.p, eq->phi->v.p, m.kw.tmp.p, m.stream);
        PB_CUDA(cudaMemcpyAsync(eq->phi->v.p, m.kw.tmp.p, m.nc * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
        eq->phi->event += 3;
    }
}

}  // namespace

bool needsPressureReference(const Scalar& p) {  // SIMPLE.cpp:110-122
    for (int q = 0; q < p.m->npatch; ++q) {
        if (p.m->h->patches[q].empty) continue;
        if (isDirichlet(p.bc[q].kind)) return false;
    }
    return true;
}

void simpleStep(const PrismSIMPLEControls& c, std::vector<Transport*>& mom, Vector& U, Vector& mdot, Scalar& p,
                const PrismSolveOpts& so, std::vector<Report>& rep) {
    if (mom.size() != 2 && mom.size() != 3) fail(PRISM_BAD_ARG, "SIMPLE expects 2 or 3 momentum predictors");
    PhaseTimer pt("SIMPLE step", p.m->stream);
    solveImplicitMomentum(c, mom, so, rep);
    auto r = solvePressureEquation(c, mom, U, mdot, p, so, rep);
    PhaseTimer pc("correct fields", p.m->stream);
    correctFields(U, mdot, p, *r.D, *r.pp, c.pressure_urf);
}

void primeStep(const PrismSIMPLEControls& pc, std::vector<Transport*>& mom, Vector& U, Vector& mdot, Scalar& p,
               const PrismSolveOpts& so, std::vector<Report>& rep) {
    if (mom.size() != 2 && mom.size() != 3) fail(PRISM_BAD_ARG, "PRIME expects 2 or 3 momentum predictors");
    solveExplicitMomentum(mom);
    PrismSIMPLEControls c;
    simpleDefaults(&c);
    c.non_ortho_correctors = pc.non_ortho_correctors;
    c.pressure_urf = pc.pressure_urf;
    c.pressure_max_iter = pc.pressure_max_iter;
    c.pressure_residual = pc.pressure_residual;
    c.p_ref_cell = pc.p_ref_cell;
    c.p_ref_value = pc.p_ref_value;
    auto r = solvePressureEquation(c, mom, U, mdot, p, so, rep);
    correctFields(U, mdot, p, *r.D, *r.pp, pc.pressure_urf);
}

void pisoStep(const PrismPISOControls& pc, std::vector<Transport*>& mom, Vector& U, Vector& mdot, Scalar& p,
              const PrismSolveOpts& so, std::vector<Report>& rep) {
    PrismSIMPLEControls sc;
    simpleDefaults(&sc);
    sc.momentum_urf = pc.momentum_urf;
    sc.momentum_max_iter = pc.momentum_max_iter;
    sc.momentum_residual = pc.momentum_residual;
    sc.momentum_residual_stop = pc.momentum_residual_stop;
    sc.non_ortho_correctors = pc.non_ortho_correctors;
    sc.pressure_urf = pc.pressure_urf;
    sc.pressure_max_iter = pc.pressure_max_iter;
    sc.pressure_residual = pc.pressure_residual;
    sc.p_ref_cell = pc.p_ref_cell;
    sc.p_ref_value = pc.p_ref_value;
    sc.batched_momentum = pc.batched_momentum;
    for (int64_t i = 0; i < pc.outer_iterations; ++i) {
        for (int64_t j = 0; j < pc.momentum_implicit_steps; ++j) simpleStep(sc, mom, U, mdot, p, so, rep);
        for (int64_t j = 1; j < pc.pressure_correction_steps; ++j) primeStep(sc, mom, U, mdot, p, so, rep);
    }
}

}  // namespace pb

namespace pb {

// ------------------------------------------------------------------ steady fixed point + adjoint
FixedPointOut steadySolve(Transport& eq, const PrismSolveOpts& o, int max_outer, double outer_tol) {
    Scalar& phi = *eq.phi;
    Mesh& m = *phi.m;
    FixedPointOut out;
    DevBuf<double> prev(m.n_pad), scratch(2 * NUM_SMS * 8 + 2);
    double h[2];
    for (int it = 0; it < max_outer; ++it) {
        PB_CUDA(cudaMemcpyAsync(prev.p, phi.v.p, m.nc * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
        PrismSolveResult r = solve(eq, o);
        out.krylov += r.krylov_iterations;
        ++out.outer;
        if (r.status != PRISM_OK && out.status == PRISM_OK) out.status = r.status;
        diffNorms(m.nc, phi.v.p, prev.p, scratch.p, nullptr, scratch.p + 2 * NUM_SMS * 8, h, m.stream);
        out.change = h[1] > 0 ? std::sqrt(h[0] / h[1]) : std::sqrt(h[0]);
        if (!std::isfinite(out.change)) {
            out.status = PRISM_NONFINITE;
            break;
        }
        if (out.change <= outer_tol) {
            out.converged = true;
            break;
        }
    }
    return out;
}

namespace {
void checkAdjointSupported(const Transport& eq) {
    const Scalar& phi = *eq.phi;
    if (!eq.has_diff || eq.has_conv || eq.has_temporal || !eq.ks || eq.kt || eq.symmetry)
        fail(PRISM_BAD_ARG, "adjoint: only a diffusion equation with a scalar kappa field is supported");
    if (phi.coord >= 0) fail(PRISM_BAD_ARG, "adjoint: the field must be a scalar field");
    if (eq.corrected && phi.grad->type != PRISM_GRAD_LEAST_SQUARES)
        fail(PRISM_BAD_ARG, "adjoint: Corrected diffusion needs the least-squares gradient");
    for (const auto& src : eq.sources)
        if (src.kind != PRISM_SRC_CONSTANT) fail(PRISM_BAD_ARG, "adjoint: only ConstantScalar sources are supported");
}
}  // namespace

FixedPointOut adjointBackward(Transport& eq, const double* dJ, double* gk, double* gv, const PrismSolveOpts& o,
                              int max_outer, double outer_tol) {
    checkAdjointSupported(eq);
    Scalar& phi = *eq.phi;
    Mesh& m = *phi.m;
    cudaStream_t s = m.stream;
    FixedPointOut out;
    m.ensureLeastSquares();
    if (!m.cf_twin) {
        m.cf_twin.alloc(std::max<size_t>(m.h->cf_face.size(), 1));
        buildTwin(m.view(), m.cf_twin.p, s);
    }
    if (!m.tpos) {
        m.tpos.alloc(std::max<int64_t>(m.pat.sell_nnz, 1));
        buildTransposePositions(m.nc, m.pat.nslices, m.pat.rowptr.p, m.pat.sl_off.p, m.pat.sl_col.p, m.tpos.p, s);
    }
    // A at the current phi (a clean assembly), then A^T in the same pattern
    zeroOutCoeffs(eq);
    updateCoeffs(eq);
    if (eq.corrected) ensureGradient(phi);
    if (!eq.AT) eq.AT.alloc(std::max<int64_t>(m.pat.sell_nnz, 1));
    transposeValues(m.pat.sell_nnz, m.tpos.p, eq.A.p, eq.AT.p, s);
    SellMatrix AT = m.matrix(eq.AT.p);

    AdjointParams P{};
    P.m = m.view();
    P.phi = phi.view();
    P.ks = eq.ks->view();
    P.pinv = m.ls_pinv.p;
    P.w = m.ls_w.p;
    P.nk = (int64_t)m.h->cf_face.size();
    P.twin = m.cf_twin.p;
    P.corrected = eq.corrected;
    P.corrector = eq.corrector;

    const int64_t np = m.n_pad;
    DevBuf<double> d_dJ(np), lam(np), lam_prev(np), rhs(np), u(3 * np), d(np), d_gk(np), d_gv(std::max(m.nb, 1)),
        scratch(2 * NUM_SMS * 8 + 2);
    for (auto* b : {&d_dJ, &lam, &lam_prev, &rhs, &u, &d, &d_gk}) b->zero(s);
    d_dJ.upload(dJ, m.nc, s);

    Amg* amg = nullptr;
    if (choosePreconditioner(o.preconditioner, m.nc) == PRISM_PC_AMG) {
        if (!eq.amg_adj) eq.amg_adj = std::make_shared<Amg>();
        amg = eq.amg_adj.get();
    }
    const double ktol = o.krylov_tol > 0 ? o.krylov_tol : 1e-12;
    const long long kmax = o.krylov_max_iter > 0 ? o.krylov_max_iter : 2LL * m.nc;
    double h[2];
    for (int it = 0; it < max_outer; ++it) {
        adjointCorrection(P, lam.p, u.p, d.p, np, s);
        adjointRhs(P, d_dJ.p, lam.p, u.p, d.p, np, rhs.p, s);
        PB_CUDA(cudaMemcpyAsync(lam_prev.p, lam.p, m.nc * sizeof(double), cudaMemcpyDeviceToDevice, s));
        KrylovOut k = bicgstab(AT, rhs.p, lam.p, ktol, kmax, PRISM_PREC_FP64, 0.1, m.kw, s, amg, m.pat.rowptr.p,
                               m.pat.col.p);
        out.krylov += k.iterations;
        ++out.outer;
        if (k.status != PRISM_OK && out.status == PRISM_OK) out.status = k.status;
        diffNorms(m.nc, lam.p, lam_prev.p, scratch.p, nullptr, scratch.p + 2 * NUM_SMS * 8, h, s);
        out.change = h[1] > 0 ? std::sqrt(h[0] / h[1]) : std::sqrt(h[0]);
        if (!std::isfinite(out.change)) {
            out.status = PRISM_NONFINITE;
            break;
        }
        if (out.change <= outer_tol || !eq.corrected) {
            out.converged = true;
            break;
        }
    }
    adjointCorrection(P, lam.p, u.p, d.p, np, s);
    adjointGradients(P, lam.p, u.p, np, d_gk.p, d_gv.p, s);
    d_gk.download(gk, m.nc, s);
    if (gv) d_gv.download(gv, m.nb, s);
    PB_CUDA(cudaStreamSynchronize(s));
    zeroOutCoeffs(eq);
    return out;
}

}  // namespace pb

namespace pb {

// ------------------------------------------------------------------ batched solves
BatchHandle::~BatchHandle() {
    if (stream) {
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
    }
}

std::vector<PrismSolveResult> solveBatch(BatchHandle& h, std::vector<Transport*>& eqs, const PrismSolveOpts& o) {
    if (eqs.empty()) return {};
    if (o.method != PRISM_SOLVER_BICGSTAB) fail(PRISM_BAD_ARG, "batched solve: BiCGSTAB only");
    if (o.ref_cell >= 0) fail(PRISM_BAD_ARG, "batched solve: no reference cell");
    if (!h.stream) PB_CUDA(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
    std::vector<PrismSolveResult> res(eqs.size());
    std::vector<BatchSystem> sys(eqs.size());
    int64_t maxn = 0;
    const auto t0 = std::chrono::steady_clock::now();
    for (size_t i = 0; i < eqs.size(); ++i) {
        Transport& eq = *eqs[i];
        Mesh& m = *eq.phi->m;
        updateCoeffs(eq);
        relax(eq);
        ++eq.phi->event;
        SellMatrix A = m.matrix(eq.A.p);
        res[i].initial_residual = scaledResidual(A, eq.b.p, eq.phi->v.p, m.kw, m.stream);
        PB_CUDA(cudaStreamSynchronize(m.stream));
        BatchSystem& q = sys[i];
        q.n = m.nc;
        q.nslices = m.pat.nslices;
        q.nnz_padded = m.pat.sell_nnz;
        q.sl_off = m.pat.sl_off.p;
        q.sl_col = m.pat.sl_col.p;
        q.diag_pos = m.pat.diag_pos.p;
        q.vals = eq.A.p;
        q.b = eq.b.p;
        q.x = eq.phi->v.p;
        maxn = std::max<int64_t>(maxn, m.nc);
    }
    const bool mixed = o.precision == PRISM_PREC_MIXED;
    const double tol = o.krylov_tol > 0 ? o.krylov_tol : 1e-12;
    const double itol = o.inner_tol > 0 ? o.inner_tol : (mixed ? 1e-4 : std::max(0.5 * tol, 1e-15));
    const long long maxit = o.krylov_max_iter > 0 ? o.krylov_max_iter : 2 * maxn;
    const int max_inner = (int)std::min<long long>(maxit, 1 << 30);
    const auto t1 = std::chrono::steady_clock::now();
    std::vector<BatchOut> out = pb::solveBatch(sys, h.plan, mixed, tol, itol, max_inner, 64, maxit, h.stream);
    const auto t2 = std::chrono::steady_clock::now();
    for (size_t i = 0; i < eqs.size(); ++i) {
        Transport& eq = *eqs[i];
        Mesh& m = *eq.phi->m;
        eq.phi->event += 3;
        SellMatrix A = m.matrix(eq.A.p);
        const double fin = scaledResidual(A, eq.b.p, eq.phi->v.p, m.kw, m.stream);
        PrismSolveResult& r = res[i];
        r.iterations = 1;
        r.final_residual = fin;
        r.converged = fin < o.eps ? 1 : 0;
        r.status = std::isnan(fin) ? PRISM_NONFINITE : out[i].status;
        r.krylov_iterations = out[i].iterations;
        r.krylov_rel_residual = out[i].rel_residual;
        if (o.clear_coeffs) zeroOutCoeffs(eq);
    }
    if (verbose()) {
        for (auto* eq : eqs) PB_CUDA(cudaStreamSynchronize(eq->phi->m->stream));
        auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
        std::fprintf(stderr, "[prism] batched solve: assembly %.1f ms, solve %.1f ms, residuals %.1f ms\n", ms(t0, t1),
                     ms(t1, t2), ms(t2, std::chrono::steady_clock::now()));
    }
    return res;
}

// ------------------------------------------------------------------ diagnostics
// ops::div (operations.h:84-100)
void opsDiv(Vector& U, double* out) {
    checkVectorFlux(U, "ops::div()");
    Mesh& m = *U.m;
    launchDiv(m.view(), U.view(), out, m.stream);
}

// monitor::courantNumber (courant.cpp:7-24)
void courantNumber(Vector& mdot, double dt, double* out) {
    checkVectorFlux(mdot, "monitor::courantNumber()");
    Mesh& m = *mdot.m;
    launchCourant(m.view(), mdot.view(), dt, out, m.stream);
}

// ensureCache (export.cpp:44-71): vertex -> cells in cell order, built once per mesh
void ensurePointMap(Mesh& m) {
    if (m.points_ready) return;
    const HostMesh& h = *m.h;
    const int64_t nv = h.nv, nc = h.nc;
    std::vector<int64_t> off(nv + 1, 0);
    for (int64_t q = 0; q < h.cv_off[nc]; ++q) off[h.cv_node[q] + 1]++;
    for (int64_t v = 0; v < nv; ++v) {
        if (off[v + 1] == 0)
            fail(PRISM_INVALID_MESH,
                 "Vertex " + std::to_string(v) + " has no adjacent cells; point data cannot be computed.");
        off[v + 1] += off[v];
    }
    std::vector<int> cell(off[nv]);
    std::vector<int64_t> fill(off.begin(), off.end() - 1);
    for (int64_t c = 0; c < nc; ++c)
        for (int64_t q = h.cv_off[c]; q < h.cv_off[c + 1]; ++q) cell[fill[h.cv_node[q]]++] = (int)c;
    std::vector<double> xyz(3 * nv);
    for (int k = 0; k < 3; ++k) std::copy(h.vx[k].begin(), h.vx[k].end(), xyz.begin() + k * nv);
    m.vtx.upload(xyz, m.stream);
    m.v2c_off.upload(off, m.stream);
    m.v2c_cell.upload(cell, m.stream);
    PB_CUDA(cudaStreamSynchronize(m.stream));
    m.points_ready = true;
}

// cellToPoint (export.cpp:73-111)
void cellToPoint(Mesh& m, const double* const* comp, int ncomp, int64_t stride, double* out) {
    if (ncomp < 1 || ncomp > MAX_POINT_COMPONENTS) fail(PRISM_BAD_ARG, "n_components must be 1..9");
    ensurePointMap(m);
    PointMapView pm;
    pm.nv = m.h->nv;
    pm.vx = m.vtx.p;
    pm.vy = m.vtx.p + pm.nv;
    pm.vz = m.vtx.p + 2 * pm.nv;
    pm.off = m.v2c_off.p;
    pm.cell = m.v2c_cell.p;
    PointComponents pc;
    for (int k = 0; k < ncomp; ++k) pc.p[k] = comp[k];
    pc.stride = stride;
    pc.ncomp = ncomp;
    launchCellToPoint(m.view(), pm, pc, out, m.stream);
}

// ------------------------------------------------------------------ solves and steps as one graph
namespace {

// solve() with its loops as device-side conditional nodes (ISolver::solve's
// outer steps around bicgstab()'s passes, restarts and batches): the same
// kernels in the same order as the ordinary path, decided on the device.
PrismSolveResult solveCaptured(Transport& eq, const PrismSolveOpts& o) {
    Scalar& phi = *eq.phi;
    Mesh& m = *phi.m;
    if (g_capture->m != &m) fail(PRISM_BAD_ARG, "a graph step spans more than one mesh");
    if ((o.method != PRISM_SOLVER_BICGSTAB && o.method != PRISM_SOLVER_FCG) || o.precision != PRISM_PREC_FP64)
        fail(PRISM_BAD_ARG, "graph mode runs FP64 BiCGSTAB or flexible CG only");
    if (g_capture->used >= GRAPH_SLOTS) fail(PRISM_BAD_ARG, "too many solves in one graph step");
    const int slot = g_capture->used++;
    SolveCtl* ctl = m.graph_ctl.p + slot;
    cudaStream_t s = m.stream;
    updateCoeffs(eq);
    relax(eq);
    if (o.ref_cell >= 0 && o.ref_cell < m.nc)
        launchPinDev(eq.A.p, eq.b.p, m.pat.diag_pos.p, (int)o.ref_cell, o.ref_value, s);
    SellMatrix A = m.matrix(eq.A.p);
    const double ktol = o.krylov_tol > 0 ? o.krylov_tol : 1e-12;
    const long long kmax = o.krylov_max_iter > 0 ? o.krylov_max_iter : 2LL * m.nc;
    Amg* amg = nullptr;
    if (o.method == PRISM_SOLVER_FCG || pcFor(eq, o, A) == PRISM_PC_AMG) {
        if (!eq.amg) eq.amg = std::make_shared<Amg>();
        amg = eq.amg.get();
    }
    const long long n_iter = std::max<long long>(o.n_iter, 0);
    cudaGraphConditionalHandle outer = createConditional(s, 0);
    emitSolveBegin(ctl, n_iter, o.eps, kmax, ktol, outer, s);
    if (n_iter > 0) {
        ++phi.event;
        emitResidual(A, eq.b.p, phi.v.p, m.kw, s);
        emitInitResidual(ctl, m.kw, s);
        cudaStream_t body = m.cs.at(0);
        beginConditional(s, cudaGraphCondTypeWhile, outer, body);
        phi.event += 2;
        const HoldAmgValues hold(amg, eq.matrix_unchanged);
        emitBicgstab(A, eq.b.p, phi.v.p, ktol, kmax, m.kw, body, amg, m.pat.rowptr.p, m.pat.col.p, ctl, m.cs, 1,
                     flexibleFor(eq, o, amg));
        ++phi.event;
        emitResidual(A, eq.b.p, phi.v.p, m.kw, body);
        emitOuterStep(ctl, m.kw, outer, body);
        endConditional(body);
    }
    if (o.clear_coeffs) zeroOutCoeffs(eq);
    PrismSolveResult r{};
    r.iterations = -(slot + 1);  // the device record of this solve, read after the launch
    return r;
}

PrismSolveResult fromCtl(const SolveCtl& c) {
    PrismSolveResult r{};
    r.iterations = c.outer;
    r.initial_residual = c.init_res;
    r.final_residual = c.cur_res;
    r.converged = c.converged;
    r.status = c.status;
    r.krylov_iterations = c.krylov_iterations;
    r.krylov_rel_residual = c.krylov_rel;
    return r;
}

// Captures f (host code issuing the work of solves and steps on m's stream)
// into one graph, launches it (updating the previous call's executable graph
// in place when only parameters changed) and reads the solves' records back.
int runAsGraph(Mesh& m, const std::function<void()>& f) {
    // least-squares operators are built on the host at first use: build them now, outside the capture
    m.ensureLeastSquares();
    if (!m.graph_ctl) m.graph_ctl.alloc(GRAPH_SLOTS);
    if (!m.graph_host) PB_CUDA(cudaMallocHost(&m.graph_host, GRAPH_SLOTS * sizeof(SolveCtl)));
    for (int d = 0; d < 3; ++d) m.cs.at(d);
    GraphCapture ctx;
    ctx.m = &m;
    PB_CUDA(cudaStreamBeginCapture(m.stream, cudaStreamCaptureModeRelaxed));
    g_capture = &ctx;
    cudaGraph_t graph = nullptr;
    try {
        f();
    } catch (...) {
        g_capture = nullptr;
        cudaStreamEndCapture(m.stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        throw;
    }
    g_capture = nullptr;
    PB_CUDA(cudaStreamEndCapture(m.stream, &graph));
    bool updated = false;
    if (m.graph_exec) {
        cudaGraphExecUpdateResultInfo info;
        updated = cudaGraphExecUpdate(m.graph_exec, graph, &info) == cudaSuccess;
        if (!updated) {
            cudaGetLastError();
            cudaGraphExecDestroy(m.graph_exec);
            m.graph_exec = nullptr;
        }
    }
    if (!updated) {
        cudaError_t e = cudaGraphInstantiate(&m.graph_exec, graph, 0);
        if (e != cudaSuccess) m.graph_exec = nullptr;
        cudaGraphDestroy(graph);
        PB_CUDA(e);
    } else {
        cudaGraphDestroy(graph);
    }
    PB_CUDA(cudaGraphLaunch(m.graph_exec, m.stream));
    graphLaunchCounter().fetch_add(1, std::memory_order_relaxed);
    if (ctx.used)
        PB_CUDA(cudaMemcpyAsync(m.graph_host, m.graph_ctl.p, ctx.used * sizeof(SolveCtl), cudaMemcpyDeviceToHost,
                                m.stream));
    PB_CUDA(cudaStreamSynchronize(m.stream));
    return ctx.used;
}

}  // namespace

bool graphReady(const Transport& eq, const PrismSolveOpts& o) {
    const Mesh& m = *eq.phi->m;
    if ((o.method != PRISM_SOLVER_BICGSTAB && o.method != PRISM_SOLVER_FCG) || o.precision != PRISM_PREC_FP64)
        return false;
    if (!eq.A || !eq.b || m.kw.n != m.n_pad) return false;
    int pc = o.method == PRISM_SOLVER_FCG ? PRISM_PC_AMG : choosePreconditioner(o.preconditioner, m.nc);
    if (o.method != PRISM_SOLVER_FCG && o.preconditioner == PRISM_PC_AUTO && pc == PRISM_PC_AMG && !eq.spd &&
        autoJacobiRatio() > 0.0) {
        if (eq.auto_pc == 0) return false;  // chosen on an ordinary solve first
        pc = eq.auto_pc;
    }
    if (pc == PRISM_PC_AMG) {
        if (!eq.amg || !eq.amg->built || !m.kw.y) return false;
        for (auto& L : eq.amg->levels)
            if (!L->b || !L->dinv) return false;
        if (eq.amg->k_levels > 0 && !eq.amg->kscal) return false;
        if (flexibleFor(eq, o, eq.amg.get()) && fcgPre32(eq.amg.get())) {
            if (!m.kw.y32 || (!eq.amg->coarse_inv32 && eq.amg->coarse_inv)) return false;
            for (auto& L : eq.amg->levels)
                if (!L->b32 || !L->vals32) return false;
        }
    }
    return true;
}

bool stepGraphReady(const std::vector<Transport*>& mom, const Vector& U, const Scalar& p, const PrismSolveOpts& so,
                    bool momentum_solved) {
    const Mesh& m = *p.m;
    for (auto* eq : mom) {
        if (momentum_solved && !graphReady(*eq, so)) return false;
        if (!eq->A || !eq->b) return false;
    }
    if (!m.p_eq || !m.p_corr || !m.p_D || !m.p_eq->phi) return false;
    (void)U;
    return graphReady(*m.p_eq, so);
}

PrismSolveResult solveAsGraph(Transport& eq, const PrismSolveOpts& o) {
    Mesh& m = *eq.phi->m;
    PrismSolveResult out{};
    const int used = runAsGraph(m, [&] { out = solve(eq, o); });
    if (used != 1) fail(PRISM_INTERNAL, "graph solve recorded no solve");
    return fromCtl(m.graph_host[0]);
}

void stepAsGraph(Mesh& m, const std::function<void()>& step, std::vector<Report>& rep) {
    const size_t first = rep.size();
    const int used = runAsGraph(m, step);
    for (size_t i = first; i < rep.size(); ++i) {
        Report& r = rep[i];
        if (r.n >= 0) continue;
        const int slot = (int)(-r.n - 1);
        if (slot >= used) fail(PRISM_INTERNAL, "graph step report without a record");
        const SolveCtl& c = m.graph_host[slot];
        r.n = c.outer;
        r.init = c.init_res;
        r.fin = c.cur_res;
        r.conv = c.converged != 0;
    }
}

}  // namespace pb
