// prism_oracle.cpp -- CPU oracle for the Prism hot path. TEST INFRASTRUCTURE ONLY.
//
// This file checks the product and is not part of it: only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline / --impl reference leg load it. It restates, in
// plain single-threaded FP64 C++, the algorithms of eigemx/prism's hot path:
// the UNV -> PMesh conversion and face reordering, field face values and
// boundary handlers, Green-Gauss / least-squares gradients, convection /
// diffusion / source schemes, eqn::Transport, the BiCGSTAB(+ILUT) and Jacobi
// solvers and the SIMPLE / PRIME / PISO drivers. Every function cites the
// reference file:line it follows (paths relative to the reference's src/prism/).
//
// The reference itself cannot be built here: it needs Eigen3 (absent), the
// unvpp submodule (empty) and spdlog/fmt/nlohmann via vcpkg. So this is a
// restatement. Where Eigen supplies arithmetic (3-vectors, 3x3 inverse,
// setFromTriplets, BiCGSTAB, IncompleteLUT) the restatement uses Eigen's
// documented semantics: dot products summed in index order, setFromTriplets
// summing duplicates in insertion order, textbook BiCGSTAB (van der Vorst
// 1992) with Eigen's restart rule and default tolerance (machine epsilon,
// max 2n iterations), and Saad's ILUT (1994) with Eigen's defaults
// (droptol 1e-12, fill factor 10) in natural ordering (Eigen applies an AMD
// ordering first; ordering changes only the preconditioner, not the solution).
//
// It exports the same C-ABI as include/prism_b200.h with the prefix orc_.
// Result pins: tests/test_oracle_pins.py checks it against the reference's own
// known answers (tests/test_poisson.cpp, tests/test_advection_1d.cpp, ...).

#include "../include/prism_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace orc {

constexpr double EPSILON = std::numeric_limits<double>::epsilon(); // constants.h:12

struct Error {
    int status;
    std::string msg;
};
[[noreturn]] inline void fail(int status, const std::string& msg) { throw Error{status, msg}; }

thread_local std::string g_last_error;

// ---------------------------------------------------------------- 3-vectors
struct V3 {
    double x = 0, y = 0, z = 0;
    double& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
inline double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

struct M3 {
    double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
};
inline V3 mul(const M3& A, V3 v) {
    V3 r;
    for (int i = 0; i < 3; ++i) r[i] = (A.m[i][0] * v.x + A.m[i][1] * v.y) + A.m[i][2] * v.z;
    return r;
}
inline V3 mulT(const M3& A, V3 v) { // A^T v
    V3 r;
    for (int i = 0; i < 3; ++i) r[i] = (A.m[0][i] * v.x + A.m[1][i] * v.y) + A.m[2][i] * v.z;
    return r;
}
inline M3 matmul(const M3& A, const M3& B) {
    M3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            C.m[i][j] = (A.m[i][0] * B.m[0][j] + A.m[i][1] * B.m[1][j]) + A.m[i][2] * B.m[2][j];
    return C;
}
inline M3 transpose(const M3& A) {
    M3 T;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T.m[i][j] = A.m[j][i];
    return T;
}
// 3x3 inverse by the adjugate (cofactor) formula.
inline M3 inverse3(const M3& M) {
    const auto& a = M.m;
    double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    double c10 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    double c20 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    double det = (a[0][0] * c00 + a[0][1] * c10) + a[0][2] * c20;
    M3 r;
    r.m[0][0] = c00 / det;
    r.m[1][0] = c10 / det;
    r.m[2][0] = c20 / det;
    r.m[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    r.m[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    r.m[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    r.m[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    r.m[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    r.m[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    return r;
}

// ---------------------------------------------------------------- mesh
struct Face {
    std::vector<int64_t> verts;
    double area = 0.0;
    V3 normal, center;
    int64_t owner = -1, nbr = -1;
    int32_t patch = -1;
    V3 areaVector() const { return area * normal; } // face.h:20
};
struct Cell {
    std::vector<int64_t> faces;
    std::vector<int64_t> vids; // UNV element node order (cell.h:13, unv.cpp:206-207)
    double volume = 0.0;
    V3 center;
};
struct Patch {
    std::string name;
    bool empty = false;
    std::vector<int64_t> faces;
};

// Face::Face, mesh/face.cpp:5-41 (triangle fan about the vertex average).
inline void faceGeometry(Face& f, const std::vector<V3>& fv) {
    size_t n = fv.size();
    V3 gc{0, 0, 0};
    for (size_t i = 0; i < n; ++i) gc += fv[i];
    gc = gc / static_cast<double>(n);
    f.normal = {0, 0, 0};
    f.area = 0.0;
    f.center = {0, 0, 0};
    for (size_t i = 0; i < n; ++i) {
        const V3& v1 = fv[i];
        const V3& v2 = fv[(i + 1) % n];
        const V3& v3 = gc;
        V3 sub_center = ((v1 + v2) + v3) / 3.0;
        V3 sub_normal = cross(v2 - v1, v3 - v1);
        double sub_area = norm(sub_normal) / 2.0;
        f.normal += sub_normal;
        f.area += sub_area;
        f.center += sub_center * sub_area;
    }
    f.center = f.center / f.area;
    f.normal = f.normal / norm(f.normal);
}

// Cell::Cell, mesh/cell.cpp:7-41 (pyramids on the face-centre average).
inline void cellGeometry(Cell& c, const std::vector<Face>& faces) {
    V3 gc{0, 0, 0};
    for (auto fid : c.faces) gc += faces[fid].center;
    gc = gc / static_cast<double>(c.faces.size());
    c.volume = 0.0;
    c.center = {0, 0, 0};
    for (auto fid : c.faces) {
        const Face& f = faces[fid];
        double pv = std::abs(dot(f.normal, f.center - gc) * f.area) / 3;
        V3 pc = (f.center * 0.75) + (gc * 0.25);
        c.volume += pv;
        c.center += pv * pc;
    }
    c.center = c.center / c.volume;
}

struct Mesh {
    std::vector<V3> verts;
    std::vector<Face> faces;
    std::vector<Cell> cells;
    std::vector<Patch> patches;
    int64_t n_boundary = 0, n_nonempty = 0;
    std::vector<int64_t> rowptr, col; // CSR pattern (setFromTriplets of all inserts)
    std::vector<double> volumes;
    std::vector<int64_t> cell_orig;   // cell id before any reordering
    bool frozen = false;              // fields exist: the cells can no longer be renumbered

    int64_t nc() const { return (int64_t)cells.size(); }
    int64_t nf() const { return (int64_t)faces.size(); }
    bool interior(int64_t f) const { return faces[f].nbr >= 0; }
    int64_t other(int64_t c, int64_t f) const {
        return faces[f].owner == c ? faces[f].nbr : faces[f].owner;
    }
    // mesh/utilities.cpp:15-18
    V3 outward(int64_t f, int64_t c) const {
        V3 s = faces[f].areaVector();
        return faces[f].owner == c ? s : -s;
    }
    // mesh/utilities.cpp:28-40 (always called as (owner, neighbour) by the path)
    double gweight(int64_t f) const {
        const Face& fc = faces[f];
        const Cell& c = cells[fc.owner];
        const Cell& n = cells[fc.nbr];
        V3 d_Cf = fc.center - c.center;
        V3 d_fN = n.center - fc.center;
        V3 Sf = outward(f, fc.owner);
        V3 ef = Sf / norm(Sf);
        return dot(d_Cf, ef) / (dot(d_Cf, ef) + dot(d_fN, ef));
    }
    int64_t slot(int64_t i, int64_t j) const {
        auto b = col.begin() + rowptr[i], e = col.begin() + rowptr[i + 1];
        auto it = std::lower_bound(b, e, j);
        if (it == e || *it != j) fail(PRISM_INTERNAL, "slot not in pattern");
        return it - col.begin();
    }
};

// UnvToPMeshConverter (mesh/unv.cpp:61-372) followed by PMesh (mesh/pmesh.cpp:10-119).
static const int HEX_F[6][4] = {{1, 2, 6, 5}, {0, 4, 7, 3}, {2, 3, 7, 6},
                                {0, 1, 5, 4}, {4, 5, 6, 7}, {0, 3, 2, 1}}; // unv.cpp:19-31
static const int TET_F[4][3] = {{0, 2, 1}, {1, 2, 3}, {0, 1, 3}, {0, 3, 2}}; // unv.cpp:34-43
static const int WEDGE_T[2][3] = {{0, 2, 1}, {3, 4, 5}};                      // unv.cpp:46-58
static const int WEDGE_Q[3][4] = {{0, 1, 4, 3}, {0, 3, 5, 2}, {1, 2, 5, 4}};

struct VecHash {
    size_t operator()(const std::vector<int64_t>& v) const {
        size_t h = 1469598103934665603ull;
        for (auto x : v) h = (h ^ (size_t)x) * 1099511628211ull;
        return h;
    }
};

// cached volumes (pmesh.cpp:45-47) and the pattern produced by setFromTriplets of
// the assembly inserts (linear.cpp:21-28): each row holds its diagonal and its
// face neighbours, sorted by column.
void finishMesh(Mesh& m) {
    m.volumes.resize(m.cells.size());
    for (size_t c = 0; c < m.cells.size(); ++c) m.volumes[c] = m.cells[c].volume;
    if (m.cell_orig.size() != m.cells.size()) {
        m.cell_orig.resize(m.cells.size());
        for (size_t c = 0; c < m.cells.size(); ++c) m.cell_orig[c] = (int64_t)c;
    }
    int64_t nc = m.nc();
    std::vector<std::vector<int64_t>> rows(nc);
    for (int64_t c = 0; c < nc; ++c) rows[c].push_back(c);
    for (int64_t f = m.n_boundary; f < m.nf(); ++f) {
        rows[m.faces[f].owner].push_back(m.faces[f].nbr);
        rows[m.faces[f].nbr].push_back(m.faces[f].owner);
    }
    m.rowptr.assign(nc + 1, 0);
    for (int64_t c = 0; c < nc; ++c) {
        std::sort(rows[c].begin(), rows[c].end());
        rows[c].erase(std::unique(rows[c].begin(), rows[c].end()), rows[c].end());
        m.rowptr[c + 1] = m.rowptr[c] + (int64_t)rows[c].size();
    }
    m.col.clear();
    m.col.reserve(m.rowptr[nc]);
    for (auto& r : rows) m.col.insert(m.col.end(), r.begin(), r.end());
}

std::unique_ptr<Mesh> buildFromUnv(const PrismUnvMesh* d) {
    auto m = std::make_unique<Mesh>();
    if (d->n_nodes <= 0) fail(PRISM_INVALID_MESH, "UnvToPMeshConverter(): mesh has zero vertices");
    m->verts.resize(d->n_nodes);
    for (int64_t i = 0; i < d->n_nodes; ++i)
        m->verts[i] = {d->xyz[3 * i], d->xyz[3 * i + 1], d->xyz[3 * i + 2]};

    std::unordered_map<std::vector<int64_t>, int64_t, VecHash> lookup; // FacesLookupTrie
    std::map<int64_t, std::pair<int64_t, bool>> unv_to_bface;          // unv.h:36
    std::vector<int64_t> boundary_faces, interior_faces;
    std::vector<Face>& faces = m->faces;
    std::vector<Cell>& cells = m->cells;
    int64_t cell_counter = 0;

    auto makeFace = [&](const std::vector<int64_t>& vids) {
        Face f;
        f.verts = vids;
        std::vector<V3> fv;
        for (auto v : vids) {
            if (v < 0 || v >= d->n_nodes) fail(PRISM_INVALID_MESH, "element node index out of range");
            fv.push_back(m->verts[v]);
        }
        faceGeometry(f, fv);
        return f;
    };
    // processFace, unv.cpp:190-244
    auto processFace = [&](const std::vector<int64_t>& vids) -> int64_t {
        auto key = vids;
        std::sort(key.begin(), key.end());
        auto it = lookup.find(key);
        if (it != lookup.end()) {
            Face& f = faces[it->second];
            if (f.owner >= 0) {
                f.nbr = cell_counter;
            } else {
                f.owner = cell_counter;
                boundary_faces.push_back(it->second);
            }
            return it->second;
        }
        int64_t id = (int64_t)faces.size();
        Face f = makeFace(vids);
        f.owner = cell_counter;
        faces.push_back(std::move(f));
        lookup.emplace(std::move(key), id);
        interior_faces.push_back(id);
        return id;
    };

    // processCells, unv.cpp:124-160
    for (int64_t e = 0; e < d->n_elements; ++e) {
        int kind = d->elem_kind[e];
        std::vector<int64_t> en(d->elem_nodes + d->elem_offsets[e], d->elem_nodes + d->elem_offsets[e + 1]);
        switch (kind) {
            case PRISM_ELEM_LINE: break;
            case PRISM_ELEM_QUAD:
            case PRISM_ELEM_TRIANGLE: { // processBoundaryFace, unv.cpp:246-270
                auto key = en;
                std::sort(key.begin(), key.end());
                int64_t id = (int64_t)faces.size();
                faces.push_back(makeFace(en));
                lookup[key] = id;
                unv_to_bface[e] = {id, false};
                break;
            }
            case PRISM_ELEM_HEX:
            case PRISM_ELEM_TETRA:
            case PRISM_ELEM_WEDGE: { // processCell, unv.cpp:162-188
                Cell c;
                if (kind == PRISM_ELEM_HEX) {
                    if (en.size() != 8) fail(PRISM_INVALID_MESH, "hex element needs 8 nodes");
                    for (auto& fl : HEX_F) c.faces.push_back(processFace({en[fl[0]], en[fl[1]], en[fl[2]], en[fl[3]]}));
                } else if (kind == PRISM_ELEM_TETRA) {
                    if (en.size() != 4) fail(PRISM_INVALID_MESH, "tetra element needs 4 nodes");
                    for (auto& fl : TET_F) c.faces.push_back(processFace({en[fl[0]], en[fl[1]], en[fl[2]]}));
                } else {
                    if (en.size() != 6) fail(PRISM_INVALID_MESH, "wedge element needs 6 nodes");
                    for (auto& fl : WEDGE_T) c.faces.push_back(processFace({en[fl[0]], en[fl[1]], en[fl[2]]}));
                    for (auto& fl : WEDGE_Q) c.faces.push_back(processFace({en[fl[0]], en[fl[1]], en[fl[2]], en[fl[3]]}));
                }
                c.vids = en;
                cellGeometry(c, faces);
                cells.push_back(std::move(c));
                ++cell_counter;
                break;
            }
            default: fail(PRISM_INVALID_MESH, "unsupported element type");
        }
    }
    if (cells.empty()) fail(PRISM_INVALID_MESH, "mesh is empty or two dimensional");

    // processGroup, unv.cpp:298-355
    std::map<std::string, std::vector<int64_t>> name_to_faces;
    for (int32_t g = 0; g < d->n_groups; ++g) {
        if (d->group_is_vertex && d->group_is_vertex[g]) continue;
        std::vector<int64_t> gf;
        for (int64_t k = d->group_offsets[g]; k < d->group_offsets[g + 1]; ++k) {
            int64_t e = d->group_elements[k];
            auto& entry = unv_to_bface[e]; // default-inserts like std::map::operator[]
            if (e < 0 || e >= d->n_elements ||
                (d->elem_kind[e] != PRISM_ELEM_QUAD && d->elem_kind[e] != PRISM_ELEM_TRIANGLE))
                fail(PRISM_INVALID_MESH, "group contains non-face elements (cell zones)");
            gf.push_back(entry.first);
            entry.second = true;
        }
        name_to_faces.insert({d->group_names[g], std::move(gf)});
    }
    // checkBoundaryFaces, unv.cpp:357-371
    size_t undefined = 0;
    for (auto& [k, v] : unv_to_bface)
        if (!v.second) ++undefined;
    if (undefined > 0)
        fail(PRISM_INVALID_MESH, std::to_string(undefined) + " boundary faces are not part of any boundary patch");

    // patches in fields.json order, unv.cpp:84-97
    for (int32_t p = 0; p < d->n_patches; ++p) {
        Patch pa;
        pa.name = d->patch_names[p];
        pa.empty = d->patch_is_empty[p] != 0;
        pa.faces = name_to_faces[pa.name];
        for (auto fid : pa.faces) faces[fid].patch = p;
        m->patches.push_back(std::move(pa));
    }
    for (auto fid : boundary_faces)
        if (faces[fid].patch < 0) fail(PRISM_INVALID_MESH, "boundary face without a patch");

    // PMesh::buildFacePermutation, pmesh.cpp:51-90
    int64_t n_faces = (int64_t)faces.size();
    int64_t n_boundary = (int64_t)boundary_faces.size();
    int64_t n_nonempty = 0;
    for (auto fid : boundary_faces)
        if (!m->patches[faces[fid].patch].empty) ++n_nonempty;
    std::vector<int64_t> old_to_new(n_faces, 0);
    int64_t ne = 0, em = n_nonempty, in = n_boundary;
    for (auto fid : boundary_faces) old_to_new[fid] = m->patches[faces[fid].patch].empty ? em++ : ne++;
    for (auto fid : interior_faces) old_to_new[fid] = in++;
    if (in != n_faces) fail(PRISM_INVALID_MESH, "dangling boundary faces (not owned by any cell)");
    // reorderFaces / remapFaceIds, pmesh.cpp:92-123
    std::vector<Face> nf(n_faces);
    for (int64_t o = 0; o < n_faces; ++o) nf[old_to_new[o]] = std::move(faces[o]);
    faces = std::move(nf);
    for (auto& c : cells)
        for (auto& f : c.faces) f = old_to_new[f];
    for (auto& p : m->patches)
        for (auto& f : p.faces) f = old_to_new[f];
    m->n_boundary = n_boundary;
    m->n_nonempty = n_nonempty;
    for (int64_t f = 0; f < n_boundary; ++f)
        if (faces[f].nbr >= 0) fail(PRISM_INVALID_MESH, "boundary face with two cells");
    finishMesh(*m);
    return m;
}

// CuthillMckee (mesh/reorder.cpp:8-130), restated with the reference's own data
// structures: nodes sorted by degree (std::sort), a deque of not-visited nodes
// searched linearly, the not-visited neighbours of the queue front sorted by
// degree (std::sort) and appended. O(n^2): small meshes only.
struct RcmNode {
    size_t id = 0, degree = 0;
    std::vector<size_t> nbrs;
};
std::vector<size_t> cuthillMckeePermute(const Mesh& m) {
    std::vector<RcmNode> nodes;
    nodes.reserve(m.cells.size());
    for (size_t c = 0; c < m.cells.size(); ++c) {
        RcmNode node{c, 0, {}};
        for (auto f : m.cells[c].faces) {
            const Face& fc = m.faces[f];
            if (fc.nbr < 0) continue;
            node.nbrs.push_back((size_t)(fc.owner == (int64_t)c ? fc.nbr : fc.owner));
            node.degree++;
        }
        nodes.push_back(std::move(node));
    }
    auto byDegree = [](const RcmNode& a, const RcmNode& b) { return a.degree < b.degree; };
    std::sort(nodes.begin(), nodes.end(), byDegree);
    std::vector<size_t> perm;
    std::deque<RcmNode> queue;
    std::deque<RcmNode> not_visited(nodes.begin(), nodes.end());
    while (!not_visited.empty()) {
        queue.push_back(not_visited.front());
        not_visited.pop_front();
        while (!queue.empty()) {
            std::vector<RcmNode> nv;
            for (auto nid : queue.front().nbrs) {
                auto it = std::find_if(not_visited.begin(), not_visited.end(),
                                       [nid](const RcmNode& n) { return n.id == nid; });
                if (it != not_visited.end()) {
                    nv.push_back(*it);
                    not_visited.erase(it);
                }
            }
            std::sort(nv.begin(), nv.end(), byDegree);
            queue.insert(queue.end(), nv.begin(), nv.end());
            perm.push_back(queue.front().id);
            queue.pop_front();
        }
    }
    return perm;
}

// CuthillMckee::reorder, reorder.cpp:89-129: cells move to their new ids, faces keep
// theirs with owner/neighbour renamed. The reference leaves PMesh's cached volume
// vector (pmesh.cpp:45-47) in the old order; here it follows the cells, and the
// matrix pattern is rebuilt for the new numbering.
void reorderCells(Mesh& m, bool reverse) {
    auto perm = cuthillMckeePermute(m);
    if (reverse) std::reverse(perm.begin(), perm.end());
    std::vector<int64_t> old_to_new(perm.size());
    for (size_t i = 0; i < perm.size(); ++i) old_to_new[perm[i]] = (int64_t)i;
    std::vector<Cell> nc(m.cells.size());
    std::vector<int64_t> orig(m.cells.size());
    for (size_t i = 0; i < perm.size(); ++i) {
        nc[i] = m.cells[perm[i]];
        orig[i] = m.cell_orig[perm[i]];
    }
    m.cells.swap(nc);
    m.cell_orig.swap(orig);
    for (auto& f : m.faces) {
        f.owner = old_to_new[f.owner];
        if (f.nbr >= 0) f.nbr = old_to_new[f.nbr];
    }
    finishMesh(m);
}

// ---------------------------------------------------------------- fields
struct Grad {
    int type = PRISM_GRAD_LEAST_SQUARES;
    std::vector<V3> g;
    uint64_t computed = std::numeric_limits<uint64_t>::max();
    // least squares (least_squares.cpp:12-61)
    struct Entry {
        bool interior;
        int64_t other;
        V3 w;
    };
    std::vector<M3> pinv;
    std::vector<std::vector<Entry>> cache;
};

struct Scalar {
    Mesh* m = nullptr;
    std::string name;
    int coord = -1; // component of a vector field
    std::vector<double> v;
    std::vector<double> fv; // face values, empty when unset
    std::vector<PrismBC> bc;
    std::shared_ptr<Grad> grad;
    uint64_t event = 0;
    double& at(int64_t c) { ++event; return v[c]; } // operator[] non-const, scalar.cpp:355-360
    // HistoryManager (field/history.cpp:1-63): hist[0] = previous time step
    size_t hist_max = 0;
    std::vector<std::vector<double>> hist;
};

// HistoryManager::update, history.cpp:28-46 (Scalar::updatePrevTimeSteps, scalar.cpp:322-324)
void updatePrevTimeSteps(Scalar& s) {
    if (s.hist_max == 0) return;
    if (s.hist.size() == s.hist_max) s.hist.pop_back();
    s.hist.insert(s.hist.begin(), s.v);
}
// HistoryManager::resize, history.cpp:48-60
void setHistorySize(Scalar& s, size_t n) {
    if (n == s.hist_max) return;
    if (n < s.hist.size()) s.hist.resize(n);
    s.hist_max = n;
}

struct Vector {
    Mesh* m = nullptr;
    std::string name;
    std::shared_ptr<Scalar> c[3];
    std::vector<V3> fd;
    std::vector<double> ff;
    bool has_fd = false, has_ff = false;
    std::vector<PrismBC> bc;
    V3 cellValue(int64_t i) const { return {c[0]->v[i], c[1]->v[i], c[2]->v[i]}; }
};

struct Tensor {
    Mesh* m = nullptr;
    std::vector<M3> d;
    // Tensor::valueAtFace, tensor.cpp:58-77
    M3 valueAtFace(int64_t f) const {
        const Face& fc = m->faces[f];
        if (fc.nbr < 0) return d[fc.owner];
        double gc = m->gweight(f);
        M3 r;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) r.m[i][j] = (gc * d[fc.owner].m[i][j]) + ((1 - gc) * d[fc.nbr].m[i][j]);
        return r;
    }
};

std::shared_ptr<Grad> makeGrad(Mesh* m, int type) {
    auto g = std::make_shared<Grad>();
    g->type = type;
    g->g.assign(m->nc(), V3{0, 0, 0});
    if (type == PRISM_GRAD_LEAST_SQUARES) { // LeastSquares::setPseudoInvMatrices
        g->pinv.resize(m->nc());
        g->cache.resize(m->nc());
        for (int64_t c = 0; c < m->nc(); ++c) {
            M3 D;
            for (auto fid : m->cells[c].faces) {
                V3 r;
                bool inter = m->interior(fid);
                if (inter) r = m->cells[m->other(c, fid)].center - m->cells[c].center;
                else r = m->faces[fid].center - m->cells[c].center;
                double wk = 1 / (norm(r) + EPSILON);
                V3 w = r * wk;
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) D.m[i][j] += w[i] * r[j];
                if (inter) g->cache[c].push_back({true, m->other(c, fid), w});
                else if (!m->patches[m->faces[fid].patch].empty) g->cache[c].push_back({false, fid, w});
            }
            M3 Dt = transpose(D);
            g->pinv[c] = matmul(inverse3(matmul(Dt, D)), Dt);
        }
    }
    return g;
}

inline bool scalarHasHandler(int kind) {
    return kind == PRISM_BC_FIXED || kind == PRISM_BC_NOSLIP || kind == PRISM_BC_SYMMETRY ||
           kind == PRISM_BC_OUTLET || kind == PRISM_BC_ZERO_GRADIENT;
}
inline bool scalarIsDirichlet(int kind) { return kind == PRISM_BC_FIXED || kind == PRISM_BC_NOSLIP; }

// BoundaryPatch::getScalarBoundaryCondition (mesh/boundary.cpp:447-501)
double scalarBCValue(const Scalar& s, int32_t p) {
    const PrismBC& bc = s.bc[p];
    if (s.coord >= 0) {
        if (bc.value_kind != PRISM_BCV_VECTOR)
            fail(PRISM_BAD_ARG, "patch '" + s.m->patches[p].name + "' field is not a vector");
        return bc.vector[s.coord];
    }
    if (bc.value_kind != PRISM_BCV_SCALAR)
        fail(PRISM_BAD_ARG, "patch '" + s.m->patches[p].name + "' field '" + s.name + "' is not a scalar");
    return bc.value;
}
V3 vectorBCValue(const std::vector<PrismBC>& bcs, const Mesh* m, int32_t p) {
    if (bcs[p].value_kind != PRISM_BCV_VECTOR)
        fail(PRISM_BAD_ARG, "patch '" + m->patches[p].name + "' field is not a vector");
    return {bcs[p].vector[0], bcs[p].vector[1], bcs[p].vector[2]};
}

[[noreturn]] void noHandler(const Mesh* m, int32_t p, const std::string& who) {
    fail(PRISM_NO_BC_HANDLER, who + ": no boundary handler for patch '" + m->patches[p].name + "'");
}

// Scalar::valueAtFace, scalar.cpp:189-237 + field/scalar_boundary.h:53-77
double valueAtFace(const Scalar& s, int64_t f) {
    if (!s.fv.empty()) return s.fv[f];
    const Face& fc = s.m->faces[f];
    if (fc.nbr >= 0) {
        double gc = s.m->gweight(f);
        double val = gc * s.v[fc.owner];
        val += (1 - gc) * s.v[fc.nbr];
        return val;
    }
    int k = s.bc[fc.patch].kind;
    if (k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP) return scalarBCValue(s, fc.patch);
    if (k == PRISM_BC_SYMMETRY || k == PRISM_BC_OUTLET || k == PRISM_BC_ZERO_GRADIENT) return s.v[fc.owner];
    noHandler(s.m, fc.patch, "Scalar::valueAtBoundaryFace() for field " + s.name);
}

// GeneralVector::valueAtFace, vector.h:188-226 + field/vector_boundary.h:75-115
V3 valueAtFace(const Vector& U, int64_t f) {
    if (U.has_fd) return U.fd[f];
    const Face& fc = U.m->faces[f];
    if (fc.nbr < 0) {
        int k = U.bc[fc.patch].kind;
        if (k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP) return vectorBCValue(U.bc, U.m, fc.patch);
        V3 Uc = U.cellValue(fc.owner);
        if (k == PRISM_BC_SYMMETRY) return Uc - dot(Uc, fc.normal) * fc.normal;
        if (k == PRISM_BC_OUTLET || k == PRISM_BC_ZERO_GRADIENT) return Uc;
        noHandler(U.m, fc.patch, "GeneralVector::valueAtBoundaryFace() for field " + U.name);
    }
    return {valueAtFace(*U.c[0], f), valueAtFace(*U.c[1], f), valueAtFace(*U.c[2], f)};
}

// GeneralVector::fluxAtFace, vector.h:238-290 + vector_boundary.h:60-62,90-110
double fluxAtFace(const Vector& U, int64_t f) {
    if (U.has_ff) return U.ff[f];
    const Face& fc = U.m->faces[f];
    if (fc.nbr >= 0) return dot(valueAtFace(U, f), fc.areaVector());
    int k = U.bc[fc.patch].kind;
    if (k == PRISM_BC_NOSLIP || k == PRISM_BC_SYMMETRY) return 0.0;
    if (k == PRISM_BC_FIXED || k == PRISM_BC_OUTLET || k == PRISM_BC_ZERO_GRADIENT)
        return dot(valueAtFace(U, f), fc.areaVector());
    noHandler(U.m, fc.patch, "GeneralVector::fluxAtBoundaryFace() for field " + U.name);
}

// ---------------------------------------------------------------- gradients
void computeAllCellGradients(Scalar& s);

// GreenGauss::gradAtCell / LeastSquares::gradAtCell (lazy cache by event number)
V3 gradAtCell(Scalar& s, int64_t c) {
    if (s.event != s.grad->computed) computeAllCellGradients(s);
    return s.grad->g[c];
}

// GreenGauss::computeGradAtCell, green_gauss.cpp:47-88 (in place, cell order)
static void ggCell(Scalar& s, int64_t c) {
    Mesh* m = s.m;
    auto& g = s.grad->g;
    const Cell& cell = m->cells[c];
    V3 grad{0, 0, 0};
    for (auto fid : cell.faces) {
        const Face& fc = m->faces[fid];
        if (fc.nbr < 0) {
            if (m->patches[fc.patch].empty) continue;
            double phi = valueAtFace(s, fid);
            grad += phi * fc.areaVector();
            continue;
        }
        V3 Sf = m->outward(fid, c);
        int64_t n = m->other(c, fid);
        double face_phi = 0.5 * (s.v[c] + s.v[n]);
        V3 grad_sum = g[c] + g[n];
        V3 vec = fc.center - (0.5 * (cell.center + m->cells[n].center));
        face_phi += 0.5 * dot(grad_sum, vec);
        grad += Sf * face_phi;
    }
    grad = grad / cell.volume;
    g[c] = grad;
}

// LeastSquares::computeGradAtCell, least_squares.cpp:78-100
static void lsCell(Scalar& s, int64_t c) {
    V3 b{0, 0, 0};
    double phi_c = s.v[c];
    for (const auto& e : s.grad->cache[c]) {
        double other = e.interior ? s.v[e.other] : valueAtFace(s, e.other);
        b += e.w * (other - phi_c);
    }
    s.grad->g[c] = mul(s.grad->pinv[c], b);
}

void computeAllCellGradients(Scalar& s) {
    for (int64_t c = 0; c < s.m->nc(); ++c) {
        if (s.grad->type == PRISM_GRAD_GREEN_GAUSS) ggCell(s, c);
        else lsCell(s, c);
    }
    s.grad->computed = s.event;
}

// IGradient::gradAtFace, gradient.cpp:15-51 + gradient/boundary.cpp:6-34
V3 gradAtFace(Scalar& s, int64_t f) {
    Mesh* m = s.m;
    const Face& fc = m->faces[f];
    if (fc.nbr >= 0) {
        V3 go = gradAtCell(s, fc.owner);
        V3 gn = gradAtCell(s, fc.nbr);
        double gc = m->gweight(f);
        return (gc * go) + ((1. - gc) * gn);
    }
    int k = s.bc[fc.patch].kind;
    if (k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP) {
        V3 grad_c = gradAtCell(s, fc.owner);
        V3 d_Cf = fc.center - m->cells[fc.owner].center;
        V3 e = d_Cf / norm(d_Cf);
        double phi_b = valueAtFace(s, f);
        double phi_C = s.v[fc.owner];
        return (grad_c - dot(grad_c, e) * e) + ((phi_b - phi_C) / norm(d_Cf)) * e;
    }
    if (k == PRISM_BC_SYMMETRY || k == PRISM_BC_OUTLET || k == PRISM_BC_ZERO_GRADIENT)
        return gradAtCell(s, fc.owner);
    noHandler(m, fc.patch, "IGradient::gradAtBoundaryFace()");
}

// ---------------------------------------------------------------- schemes
struct LinSys {
    std::vector<double> A, b;
    void init(const Mesh* m) {
        A.assign(m->col.size(), 0.0);
        b.assign(m->nc(), 0.0);
    }
};

enum SchemeKind { SK_CONV, SK_DIFF, SK_TEMPORAL };
struct Scheme {
    SchemeKind kind;
    int temporal = 0;  // PRISM_TEMPORAL_*
    double dt = 1e-5;  // ITemporal default, temporal.h:22
    int conv = 0;
    bool corrected = false;
    int corrector = PRISM_CORR_OVER_RELAXED;
    Vector* U = nullptr;
    Scalar* kappa_s = nullptr;
    Tensor* kappa_t = nullptr;
    LinSys ls;
};
struct Source {
    int kind, sign, coord;
    Scalar* s = nullptr;
    Vector* U = nullptr;
    std::vector<double> b;
};

struct Transport {
    Scalar* phi;
    std::vector<Scheme> schemes;
    std::vector<Source> sources;
    LinSys ls;
    double urf = 1.0;
    bool symmetry = false;
    int conv_idx = -1, diff_idx = -1;
};

struct W {
    double l, k;
};
// weightsNVF, convection.cpp:69-128 (SMART keeps the integer divisions 1/6, 5/6, 3/8 == 0)
W weightsNVF(int scheme, double t) {
    switch (scheme) {
        case PRISM_CONV_UPWIND: return {1.0, 0.0};
        case PRISM_CONV_CENTRAL: return {0.5, 0.5};
        case PRISM_CONV_LINEAR_UPWIND: return {1.5, 0.0};
        case PRISM_CONV_QUICK: return {0.75, 3.0 / 8.0};
        case PRISM_CONV_FROMM: return {1.0, 0.25};
        case PRISM_CONV_MINMOD:
            if (t > 0.0 && t < 0.5) return {1.5, 0.0};
            if (t >= 0.5 && t < 1.0) return {0.5, 0.5};
            return {1.0, 0};
        case PRISM_CONV_MUSCL:
            if (t > 0.0 && t < 0.25) return {2, 0.0};
            if (t >= 0.25 && t < 0.75) return {1, 0.25};
            if (t >= 0.75 && t < 1.0) return {0, 1.0};
            return {1.0, 0};
        case PRISM_CONV_SMART: {
            const int sixth = 1 / 6, five_sixth = 5 / 6;
            if (t > 0.0 && t < sixth) return {4, 0.0};
            if (t >= sixth && t < five_sixth) return {0.75, 3 / 8};
            if (t >= five_sixth && t < 1.0) return {0, 1.0};
            return {1.0, 0};
        }
    }
    return {1.0, 0.0};
}

inline double stdmax(double a, double b) { return (a < b) ? b : a; } // std::max semantics

// Upwind::interpolate, convection.cpp:46-67 (+ convection_hr.cpp:6-23)
struct Coeffs {
    double aC, aN, b;
};
Coeffs interpolate(Scalar& phi, int scheme, double m_dot, int64_t c, int64_t n) {
    Mesh* m = phi.m;
    auto phiU = [&](int64_t cc, int64_t dn) {
        V3 d_CD = m->cells[dn].center - m->cells[cc].center;
        return phi.v[dn] - (2 * dot(gradAtCell(phi, cc), d_CD));
    };
    auto tilde = [&](int64_t cc, int64_t dn) {
        double pu = phiU(cc, dn);
        return (phi.v[cc] - pu) / (phi.v[dn] - pu);
    };
    double t = tilde(c, n);
    double pu = phiU(c, n);
    W wp = weightsNVF(scheme, t);
    double aC = stdmax(m_dot, 0.0) * wp.l;
    double aN = stdmax(m_dot, 0.0) * wp.k;
    double b = -stdmax(m_dot, 0.0) * (1 - wp.l - wp.k) * pu;
    t = tilde(n, c);
    pu = phiU(n, c);
    W wm = weightsNVF(scheme, t);
    aC += -stdmax(-m_dot, 0.0) * wm.k;
    aN += -stdmax(-m_dot, 0.0) * wm.l;
    b += stdmax(-m_dot, 0.0) * (1 - wm.l - wm.k) * pu;
    return {aC, aN, b};
}

inline void insert(LinSys& ls, const Mesh* m, int64_t i, int64_t j, double v) { ls.A[m->slot(i, j)] += v; }

// IConvection::applyInterior/applyBoundary (convection.cpp:18-44, convection_boundary.cpp:4-61)
void applyConvection(Scheme& s, Scalar& phi) {
    Mesh* m = phi.m;
    std::fill(s.ls.A.begin(), s.ls.A.end(), 0.0); // setFromTriplets replaces the matrix
    for (int32_t p = 0; p < (int32_t)m->patches.size(); ++p) {
        const Patch& pa = m->patches[p];
        if (pa.empty) continue;
        int k = phi.bc[p].kind;
        if (k == PRISM_BC_FIXED) {
            for (auto fid : pa.faces) {
                int64_t o = m->faces[fid].owner;
                double phi_wall = scalarBCValue(phi, p);
                double mdot = fluxAtFace(*s.U, fid);
                insert(s.ls, m, o, o, stdmax(mdot, 0.0));
                s.ls.b[o] += stdmax(-mdot, 0.0) * phi_wall;
            }
        } else if (k == PRISM_BC_NOSLIP || k == PRISM_BC_SYMMETRY) {
        } else if (k == PRISM_BC_OUTLET || k == PRISM_BC_ZERO_GRADIENT) {
            for (auto fid : pa.faces) {
                int64_t o = m->faces[fid].owner;
                V3 Uf = valueAtFace(*s.U, fid);
                double mdot = dot(Uf, m->faces[fid].areaVector());
                insert(s.ls, m, o, o, mdot);
            }
        } else {
            noHandler(m, p, "applyBoundary() applied by IConvection");
        }
    }
    for (int64_t f = m->n_boundary; f < m->nf(); ++f) {
        int64_t o = m->faces[f].owner, n = m->faces[f].nbr;
        double mdot = fluxAtFace(*s.U, f);
        Coeffs a = interpolate(phi, s.conv, mdot, o, n);
        Coeffs x = interpolate(phi, s.conv, -mdot, n, o);
        insert(s.ls, m, o, o, a.aC);
        insert(s.ls, m, o, n, a.aN);
        insert(s.ls, m, n, n, x.aC);
        insert(s.ls, m, n, o, x.aN);
        s.ls.b[o] += a.b;
        s.ls.b[n] += x.b;
    }
}

// IDiffusionCoeff::multiply, diffusion_coeff.cpp:8-30
V3 kappaFace(const Scheme& s, V3 v, int64_t f) {
    if (s.kappa_s) return valueAtFace(*s.kappa_s, f) * v;
    return mulT(s.kappa_t->valueAtFace(f), v);
}
V3 kappaCell(const Scheme& s, V3 v, int64_t c) {
    if (s.kappa_s) return s.kappa_s->v[c] * v;
    return mulT(s.kappa_t->d[c], v);
}
// nonortho.cpp:7-21
void decompose(int corr, V3 S, V3 e, V3& E, V3& T) {
    if (corr == PRISM_CORR_OVER_RELAXED) E = (dot(S, S) / (dot(e, S) + EPSILON)) * e;
    else if (corr == PRISM_CORR_MINIMUM) E = dot(e, S) * e;
    else E = norm(S) * e;
    T = S - E;
}

// NonCorrected / Corrected (diffusion.h:116-205, diffusion_boundary.h:113-234)
void applyDiffusion(Scheme& s, Scalar& phi) {
    Mesh* m = phi.m;
    std::fill(s.ls.A.begin(), s.ls.A.end(), 0.0);
    for (int32_t p = 0; p < (int32_t)m->patches.size(); ++p) {
        const Patch& pa = m->patches[p];
        if (pa.empty) continue;
        int k = phi.bc[p].kind;
        if (k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP) {
            for (auto fid : pa.faces) {
                const Face& fc = m->faces[fid];
                int64_t o = fc.owner;
                double phi_wall = valueAtFace(phi, fid);
                V3 d_Cf = fc.center - m->cells[o].center;
                double dn = norm(d_Cf);
                if (!s.corrected) {
                    V3 Sp = kappaCell(s, fc.areaVector(), o);
                    double g = dot(Sp, d_Cf) / (dn * dn + EPSILON);
                    insert(s.ls, m, o, o, g);
                    s.ls.b[o] += g * phi_wall;
                } else {
                    V3 e = d_Cf / dn;
                    V3 Sp = kappaCell(s, fc.areaVector(), o);
                    V3 E, T;
                    decompose(s.corrector, Sp, e, E, T);
                    double g = dot(E, d_Cf) / (dn * dn + EPSILON);
                    insert(s.ls, m, o, o, g);
                    s.ls.b[o] += (g * phi_wall) + dot(T, gradAtFace(phi, fid));
                }
            }
        } else if (k == PRISM_BC_SYMMETRY || k == PRISM_BC_OUTLET || k == PRISM_BC_ZERO_GRADIENT) {
        } else if (k == PRISM_BC_FIXED_GRADIENT) {
            for (auto fid : pa.faces) {
                const Face& fc = m->faces[fid];
                if (phi.coord >= 0)
                    fail(PRISM_BAD_ARG, "patch '" + pa.name + "' does not have a field named '" + phi.name + "'");
                V3 wall_grad = vectorBCValue(phi.bc, m, p);
                V3 Sp = kappaCell(s, fc.areaVector(), fc.owner);
                s.ls.b[fc.owner] += -dot(wall_grad, Sp);
            }
        } else {
            noHandler(m, p, "applyBoundary() applied by a diffusion scheme");
        }
    }
    for (int64_t f = m->n_boundary; f < m->nf(); ++f) {
        const Face& fc = m->faces[f];
        int64_t o = fc.owner, n = fc.nbr;
        V3 d_CF = m->cells[n].center - m->cells[o].center;
        double dn = norm(d_CF);
        double g;
        V3 T;
        if (!s.corrected) {
            V3 Sp = kappaFace(s, fc.areaVector(), f);
            g = dot(Sp, d_CF) / (dn * dn + EPSILON);
        } else {
            V3 e = d_CF / dn;
            V3 Sf = m->outward(f, o);
            V3 Sp = kappaFace(s, Sf, f);
            V3 E;
            decompose(s.corrector, Sp, e, E, T);
            g = dot(E, d_CF) / (dn * dn + EPSILON);
        }
        insert(s.ls, m, o, o, g);
        insert(s.ls, m, n, n, g);
        insert(s.ls, m, o, n, -g);
        insert(s.ls, m, n, o, -g);
        if (s.corrected) {
            V3 gf = gradAtFace(phi, f);
            s.ls.b[o] += dot(T, gf);
            s.ls.b[n] += -dot(T, gf);
        }
    }
}

// ops::div (operations.h:84-100,144-169)
double fluxSumAtCell(const Vector& U, int64_t c) {
    const Mesh* m = U.m;
    double sum = 0.0;
    for (auto fid : m->cells[c].faces) {
        const Face& fc = m->faces[fid];
        if (fc.nbr < 0 && m->patches[fc.patch].empty) continue;
        double flux = fluxAtFace(U, fid);
        if (fc.owner != c) flux = -flux;
        sum += flux;
    }
    return sum;
}

// ConstantScalar / Divergence / Gradient ::apply (scheme/source/*.h)
void applySource(Source& s, Mesh* m) {
    int64_t nc = m->nc();
    s.b.assign(nc, 0.0);
    if (s.kind == PRISM_SRC_CONSTANT) {
        ++s.s->event; // values() non-const
        for (int64_t c = 0; c < nc; ++c) s.b[c] = s.s->v[c] * m->volumes[c];
    } else if (s.kind == PRISM_SRC_DIVERGENCE) {
        for (int64_t c = 0; c < nc; ++c) {
            double d = fluxSumAtCell(*s.U, c) / m->cells[c].volume;
            s.b[c] = d * m->volumes[c];
        }
    } else {
        for (int64_t c = 0; c < nc; ++c) s.b[c] = gradAtCell(*s.s, c)[s.coord] * m->volumes[c];
    }
    if (s.sign == PRISM_SIGN_NEGATIVE)
        for (auto& x : s.b) x = -x;
}

// eqn::boundary::Symmetry<Transport>::apply, equation/symmetry.cpp:54-90
void applySymmetry(Transport& eq, int32_t p) {
    Mesh* m = eq.phi->m;
    if (eq.conv_idx < 0 || eq.diff_idx < 0)
        fail(PRISM_BAD_ARG, "symmetry handler needs a convection and a diffusion scheme");
    if (eq.phi->coord < 0) fail(PRISM_BAD_ARG, "symmetry handler needs a vector component field");
    Vector* U = eq.schemes[eq.conv_idx].U;
    const Scheme& diff = eq.schemes[eq.diff_idx];
    LinSys sys;
    sys.init(m);
    for (auto fid : m->patches[p].faces) {
        const Face& fc = m->faces[fid];
        int64_t o = fc.owner;
        V3 n = fc.normal;
        V3 d_Cb = fc.center - m->cells[o].center;
        double d_normal = dot(d_Cb, n);
        V3 Uc = U->cellValue(o);
        V3 Sf = fc.areaVector();
        double g = 2 * norm(kappaCell(diff, Sf, o)) / d_normal;
        double ac, b;
        if (eq.phi->coord == 0) { ac = n.x * n.x; b = ((Uc.y * n.y) + (Uc.z * n.z)) * n.x; }
        else if (eq.phi->coord == 1) { ac = n.y * n.y; b = ((Uc.x * n.x) + (Uc.z * n.z)) * n.y; }
        else { ac = n.z * n.z; b = ((Uc.x * n.x) + (Uc.y * n.y)) * n.z; }
        insert(sys, m, o, o, g * ac);
        sys.b[o] += -g * b;
    }
    for (size_t k = 0; k < sys.A.size(); ++k) eq.ls.A[k] += sys.A[k];
    for (int64_t c = 0; c < m->nc(); ++c) eq.ls.b[c] += sys.b[c];
}

// BackwardEuler::applyIncompressible (backward_euler.cpp:62-83) and
// AdamMoulton::applyIncompressible (adam_moulton.cpp:62-99): the scheme's matrix is
// the diagonal alone and its rhs is assigned (no accumulation across applies).
void applyTemporal(Scheme& s, Scalar& phi) {
    Mesh* m = phi.m;
    const std::string who = s.temporal == PRISM_TEMPORAL_BACKWARD_EULER ? "BackwardEuler" : "AdamMoulton";
    if (phi.hist.empty())
        fail(PRISM_BAD_ARG, "prism::scheme::temporal::" + who + "::apply() was called for field `" + phi.name +
                                "`, but the field does not have any previous time step values stored.");
    std::fill(s.ls.A.begin(), s.ls.A.end(), 0.0);
    const std::vector<double>& vol = m->volumes;
    const std::vector<double>& p1 = phi.hist[0];
    if (s.temporal == PRISM_TEMPORAL_ADAM_MOULTON && phi.hist.size() >= 2) {
        const std::vector<double>& p2 = phi.hist[1];
        for (int64_t c = 0; c < m->nc(); ++c) {
            s.ls.A[m->slot(c, c)] = ((3.0 / 2.0) * vol[c]) / s.dt;
            s.ls.b[c] = (2.0 * (vol[c] * p1[c])) / s.dt;
        }
        for (int64_t c = 0; c < m->nc(); ++c) s.ls.b[c] += (-0.5 * (vol[c] * p2[c])) / s.dt;
    } else {  // BackwardEuler, or AdamMoulton's first step
        for (int64_t c = 0; c < m->nc(); ++c) {
            s.ls.A[m->slot(c, c)] = vol[c] / s.dt;
            s.ls.b[c] = (vol[c] * p1[c]) / s.dt;
        }
    }
}

// Transport::updateCoeffs, transport.cpp:4-21
void updateCoeffs(Transport& eq) {
    Mesh* m = eq.phi->m;
    for (auto& s : eq.schemes) {
        if (s.kind == SK_CONV) applyConvection(s, *eq.phi);
        else if (s.kind == SK_DIFF) applyDiffusion(s, *eq.phi);
        else applyTemporal(s, *eq.phi);
        for (size_t k = 0; k < s.ls.A.size(); ++k) eq.ls.A[k] += s.ls.A[k];
        for (int64_t c = 0; c < m->nc(); ++c) eq.ls.b[c] += s.ls.b[c];
    }
    for (auto& src : eq.sources) {
        applySource(src, m);
        for (int64_t c = 0; c < m->nc(); ++c) eq.ls.b[c] += src.b[c];
    }
    if (eq.symmetry) // applyBoundaryIfExists, boundary.h:127-159
        for (int32_t p = 0; p < (int32_t)m->patches.size(); ++p)
            if (!m->patches[p].empty && eq.phi->bc[p].kind == PRISM_BC_SYMMETRY) applySymmetry(eq, p);
}

// Transport::zeroOutCoeffs, transport.cpp:23-36
void zeroOutCoeffs(Transport& eq) {
    for (auto& s : eq.schemes) {
        std::fill(s.ls.A.begin(), s.ls.A.end(), 0.0);
        std::fill(s.ls.b.begin(), s.ls.b.end(), 0.0);
    }
    for (auto& src : eq.sources) std::fill(src.b.begin(), src.b.end(), 0.0);
    std::fill(eq.ls.A.begin(), eq.ls.A.end(), 0.0);
    std::fill(eq.ls.b.begin(), eq.ls.b.end(), 0.0);
}

// Transport::relax, transport.cpp:54-64
void relax(Transport& eq) {
    Mesh* m = eq.phi->m;
    ++eq.phi->event;
    double a = eq.urf;
    for (int64_t c = 0; c < m->nc(); ++c) {
        int64_t k = m->slot(c, c);
        eq.ls.b[c] += ((1.0 - a) / a) * (eq.ls.A[k] * eq.phi->v[c]);
    }
    for (int64_t c = 0; c < m->nc(); ++c) eq.ls.A[m->slot(c, c)] /= a;
}

// ---------------------------------------------------------------- linear algebra
struct CSR {
    int64_t n;
    const int64_t* rp;
    const int64_t* ci;
    const double* v;
};
void spmv(const CSR& A, const std::vector<double>& x, std::vector<double>& y) {
    y.assign(A.n, 0.0);
    for (int64_t i = 0; i < A.n; ++i) {
        double s = 0.0;
        for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) s += A.v[k] * x[A.ci[k]];
        y[i] = s;
    }
}
double diagOf(const CSR& A, int64_t i) {
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if (A.ci[k] == i) return A.v[k];
    return 0.0;
}

// residual(), numerics/solver.cpp:8-24. Each maxCoeff() is a reduction seeded with the first
// coefficient and folded with std::max, so a NaN in the first position propagates and a NaN
// further on is dropped (Eigen's scalar max keeps its first argument when either is NaN).
double scaledResidual(const CSR& A, const std::vector<double>& x, const std::vector<double>& b) {
    std::vector<double> Ax;
    spmv(A, x, Ax);
    if (A.n == 0) return 0.0;
    double denom = std::abs(diagOf(A, 0) * x[0]);
    for (int64_t i = 1; i < A.n; ++i) denom = std::max(denom, std::abs(diagOf(A, i) * x[i]));
    denom += EPSILON;
    double r = std::abs(Ax[0] - b[0]) / denom;
    for (int64_t i = 1; i < A.n; ++i) r = std::max(r, std::abs(Ax[i] - b[i]) / denom);
    return r;
}

// ILUT (Saad 1994) with Eigen's IncompleteLUT defaults: droptol 1e-12, fill factor 10.
struct ILUT {
    int64_t n = 0;
    std::vector<int64_t> lp, lc, up, uc; // L strictly lower (unit diagonal), U with diagonal first
    std::vector<double> lv, uv;
    void factor(const CSR& A, double droptol = 1e-12, int fillfactor = 10) {
        n = A.n;
        int64_t nnz = A.rp[n];
        int64_t fill_in = (fillfactor * nnz) / std::max<int64_t>(n, 1) + 1;
        lp.assign(1, 0); up.assign(1, 0);
        lc.clear(); lv.clear(); uc.clear(); uv.clear();
        std::vector<double> w(n, 0.0);
        std::vector<char> mark(n, 0);
        std::vector<int64_t> Lidx, Uidx;
        for (int64_t i = 0; i < n; ++i) {
            Lidx.clear(); Uidx.clear();
            double rownorm = 0.0;
            bool diag_seen = false;
            for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
                int64_t j = A.ci[k];
                w[j] = A.v[k];
                mark[j] = 1;
                rownorm += A.v[k] * A.v[k];
                if (j < i) Lidx.push_back(j);
                else if (j > i) Uidx.push_back(j);
                else diag_seen = true;
            }
            if (!diag_seen) { w[i] = 0.0; mark[i] = 1; }
            rownorm = std::sqrt(rownorm);
            // eliminate in increasing column order (new fill enters Lidx)
            std::vector<int64_t> done;
            while (true) {
                int64_t kmin = -1; size_t pos = 0;
                for (size_t q = 0; q < Lidx.size(); ++q)
                    if (kmin < 0 || Lidx[q] < kmin) { kmin = Lidx[q]; pos = q; }
                if (kmin < 0) break;
                Lidx.erase(Lidx.begin() + pos);
                int64_t k = kmin;
                double ukk = uv[up[k]]; // diagonal stored first
                double fact = w[k] / ukk;
                if (std::abs(fact) <= droptol * rownorm) { w[k] = 0.0; mark[k] = 0; continue; }
                w[k] = fact;
                done.push_back(k);
                for (int64_t q = up[k] + 1; q < up[k + 1]; ++q) {
                    int64_t j = uc[q];
                    if (!mark[j]) {
                        mark[j] = 1; w[j] = 0.0;
                        if (j < i) Lidx.push_back(j);
                        else if (j > i) Uidx.push_back(j);
                    }
                    w[j] -= fact * uv[q];
                }
            }
            // keep the fill_in largest entries of each part
            auto keep = [&](std::vector<int64_t>& idx) {
                std::vector<int64_t> kept;
                for (auto j : idx)
                    if (std::abs(w[j]) > droptol * rownorm) kept.push_back(j);
                if ((int64_t)kept.size() > fill_in) {
                    std::nth_element(kept.begin(), kept.begin() + fill_in, kept.end(),
                                     [&](int64_t a, int64_t b) { return std::abs(w[a]) > std::abs(w[b]); });
                    kept.resize(fill_in);
                }
                std::sort(kept.begin(), kept.end());
                return kept;
            };
            auto Lk = keep(done);
            auto Uk = keep(Uidx);
            for (auto j : Lk) { lc.push_back(j); lv.push_back(w[j]); }
            lp.push_back((int64_t)lc.size());
            double d = w[i];
            if (d == 0.0) d = (0.0001 + droptol) * rownorm;
            uc.push_back(i); uv.push_back(d);
            for (auto j : Uk) { uc.push_back(j); uv.push_back(w[j]); }
            up.push_back((int64_t)uc.size());
            for (auto j : done) { w[j] = 0.0; mark[j] = 0; }
            for (auto j : Uidx) { w[j] = 0.0; mark[j] = 0; }
            for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) { w[A.ci[k]] = 0.0; mark[A.ci[k]] = 0; }
            w[i] = 0.0; mark[i] = 0;
        }
    }
    void solve(const std::vector<double>& b, std::vector<double>& x) const {
        x = b;
        for (int64_t i = 0; i < n; ++i) {
            double s = x[i];
            for (int64_t q = lp[i]; q < lp[i + 1]; ++q) s -= lv[q] * x[lc[q]];
            x[i] = s;
        }
        for (int64_t i = n - 1; i >= 0; --i) {
            double s = x[i];
            for (int64_t q = up[i] + 1; q < up[i + 1]; ++q) s -= uv[q] * x[uc[q]];
            x[i] = s / uv[up[i]];
        }
    }
};

inline double vdot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

// Eigen::BiCGSTAB<SparseMatrix, IncompleteLUT>::compute(A).solveWithGuess(b, x)
// (numerics/bicgstab.cpp:7-9): textbook right-preconditioned BiCGSTAB with a
// restart when r0.r vanishes, tolerance = machine epsilon, max 2n iterations.
int64_t bicgstabStep(const CSR& A, const std::vector<double>& b, std::vector<double>& x) {
    int64_t n = A.n;
    ILUT P;
    P.factor(A);
    const double tol = EPSILON;
    int64_t maxIters = 2 * n;
    std::vector<double> r(n), r0, Ax;
    spmv(A, x, Ax);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
    r0 = r;
    double r0_sqnorm = vdot(r0, r0);
    double rhs_sqnorm = vdot(b, b);
    if (rhs_sqnorm == 0) { std::fill(x.begin(), x.end(), 0.0); return 0; }
    double rho = 1, alpha = 1, w = 1;
    std::vector<double> v(n, 0.0), p(n, 0.0), y(n), z(n), s(n), t(n);
    double tol2 = tol * tol * rhs_sqnorm;
    double eps2 = EPSILON * EPSILON;
    int64_t i = 0, restarts = 0;
    while (vdot(r, r) > tol2 && i < maxIters) {
        double rho_old = rho;
        rho = vdot(r0, r);
        if (std::abs(rho) < eps2 * r0_sqnorm) {
            spmv(A, x, Ax);
            for (int64_t k = 0; k < n; ++k) r[k] = b[k] - Ax[k];
            r0 = r;
            rho = r0_sqnorm = vdot(r, r);
            if (restarts++ == 0) i = 0;
        }
        double beta = (rho / rho_old) * (alpha / w);
        for (int64_t k = 0; k < n; ++k) p[k] = r[k] + beta * (p[k] - w * v[k]);
        P.solve(p, y);
        spmv(A, y, v);
        alpha = rho / vdot(r0, v);
        for (int64_t k = 0; k < n; ++k) s[k] = r[k] - alpha * v[k];
        P.solve(s, z);
        spmv(A, z, t);
        double tmp = vdot(t, t);
        if (tmp > 0.0) w = vdot(t, s) / tmp;
        else w = 0.0;
        for (int64_t k = 0; k < n; ++k) x[k] += alpha * y[k] + w * z[k];
        for (int64_t k = 0; k < n; ++k) r[k] = s[k] - w * t[k];
        ++i;
    }
    return i;
}

// Jacobi::step, numerics/jacobi.cpp:5-9
void jacobiStep(const CSR& A, const std::vector<double>& b, std::vector<double>& x) {
    std::vector<double> Ax;
    spmv(A, x, Ax);
    for (int64_t i = 0; i < A.n; ++i) {
        double dinv = 1.0 / diagOf(A, i);
        double r = b[i] - Ax[i];
        x[i] = x[i] + dinv * r;
    }
}

// ISolver::solve, numerics/solver.cpp:27-82
PrismSolveResult solve(Transport& eq, const PrismSolveOpts& o) {
    Mesh* m = eq.phi->m;
    updateCoeffs(eq);
    relax(eq);
    if (o.ref_cell >= 0 && o.ref_cell < m->nc()) {
        int64_t k = m->slot(o.ref_cell, o.ref_cell);
        double diag = eq.ls.A[k];
        eq.ls.A[k] += diag;
        eq.ls.b[o.ref_cell] += diag * o.ref_value;
    }
    CSR A{m->nc(), m->rowptr.data(), m->col.data(), eq.ls.A.data()};
    PrismSolveResult res{};
    double init_res = 0.0, cur = 0.0;
    bool conv = false;
    int64_t iter = 0, kry = 0;
    Scalar& phi = *eq.phi;
    for (; iter < o.n_iter; ++iter) {
        if (iter == 0) { ++phi.event; init_res = scaledResidual(A, phi.v, eq.ls.b); }
        phi.event += 2;
        if (o.method == PRISM_SOLVER_JACOBI) jacobiStep(A, eq.ls.b, phi.v);
        else kry += bicgstabStep(A, eq.ls.b, phi.v);
        ++phi.event;
        cur = scaledResidual(A, phi.v, eq.ls.b);
        if (cur < o.eps) { conv = true; ++iter; break; }
    }
    if (o.clear_coeffs) zeroOutCoeffs(eq);
    res.iterations = iter;
    res.initial_residual = init_res;
    res.final_residual = cur;
    res.converged = conv ? 1 : 0;
    res.krylov_iterations = kry;
    res.status = PRISM_OK;
    return res;
}

// ---------------------------------------------------------------- SIMPLE / PRIME / PISO
// Defaults of SIMPLEControls (SIMPLE.h:14-43) and PISOControls (PISO.h:11-49).
inline void simpleDefaults(PrismSIMPLEControls* c) {
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
inline void pisoDefaults(PrismPISOControls* c) {
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

struct Report {
    std::string name;
    int64_t n;
    double init, fin;
    bool conv;
};

PrismSolveOpts solverOpts(int64_t n_iter, double eps, int64_t ref, double refv, bool clear) {
    PrismSolveOpts o{};
    o.method = PRISM_SOLVER_BICGSTAB;
    o.n_iter = n_iter;
    o.eps = eps;
    o.ref_cell = ref;
    o.ref_value = refv;
    o.clear_coeffs = clear ? 1 : 0;
    return o;
}

// Transport::setUnderRelaxFactor, transport.cpp:38-52 (out of range: value kept)
void setURF(Transport& eq, double f) {
    if (f < 0.0 || f > 1.0) return;
    eq.urf = f;
}

// solveImplicitMomentum, SIMPLE.cpp:19-41
void solveImplicitMomentum(const PrismSIMPLEControls& c, std::vector<Transport*>& mom, std::vector<Report>& rep) {
    for (auto* eq : mom) {
        setURF(*eq, c.momentum_urf);
        auto r = solve(*eq, solverOpts(c.momentum_max_iter, c.momentum_residual, -1, 0.0, false));
        rep.push_back({eq->phi->name, r.iterations, r.initial_residual, r.final_residual, r.converged != 0});
    }
}

// pressureEquationCoeffsTensor, SIMPLE.cpp:77-108
std::unique_ptr<Tensor> pressureCoeffs(std::vector<Transport*>& mom, Mesh* m) {
    auto D = std::make_unique<Tensor>();
    D->m = m;
    D->d.assign(m->nc(), M3{});
    for (int64_t c = 0; c < m->nc(); ++c) {
        int64_t k = m->slot(c, c);
        D->d[c].m[0][0] = m->volumes[c] / (mom[0]->ls.A[k] + EPSILON);
        D->d[c].m[1][1] = m->volumes[c] / (mom[1]->ls.A[k] + EPSILON);
        D->d[c].m[2][2] = mom.size() == 3 ? m->volumes[c] / (mom[2]->ls.A[k] + EPSILON) : 1.0;
    }
    for (auto* eq : mom) zeroOutCoeffs(*eq);
    return D;
}

// needsPressureReference, SIMPLE.cpp:110-122
bool needsPressureReference(const Scalar& p) {
    for (size_t q = 0; q < p.m->patches.size(); ++q) {
        if (p.m->patches[q].empty) continue;
        if (scalarIsDirichlet(p.bc[q].kind)) return false;
    }
    return true;
}

// GeneralVector::initFaceData + mapFaceValues + mapInteriorFaceValues (vector.h:338-397)
void initFaceData(Vector& U) {
    Mesh* m = U.m;
    std::vector<V3> fd(m->nf(), V3{0, 0, 0});
    std::vector<double> ff(m->nf(), 0.0);
    for (auto& pa : m->patches) {
        if (pa.empty) continue;
        for (auto fid : pa.faces) {
            fd[fid] = valueAtFace(U, fid);
            ff[fid] = fluxAtFace(U, fid);
        }
    }
    U.fd = std::move(fd);
    U.ff = std::move(ff);
    U.has_fd = U.has_ff = true;
}

// rhieChowCorrectFace + pressureGradCalculated (operations/rhie_chow.h:47-63, rhie_chow.cpp:5-25)
V3 rhieChow(int64_t f, Vector& U, const Tensor& D, Scalar& P) {
    Mesh* m = U.m;
    const Face& fc = m->faces[f];
    V3 Uf = valueAtFace(U, f);
    M3 Df = D.valueAtFace(f);
    V3 gavg = gradAtFace(P, f);
    V3 d_CF = m->cells[fc.nbr].center - m->cells[fc.owner].center;
    double dn = norm(d_CF);
    V3 e = d_CF / dn;
    double gortho = (P.v[fc.nbr] - P.v[fc.owner]) / dn;
    V3 gcalc = gavg + ((gortho - dot(gavg, e)) * e);
    return Uf - mul(Df, gcalc - gavg);
}

struct PressureResult {
    std::unique_ptr<Scalar> pprime;
    std::unique_ptr<Tensor> D;
};

// solvePressureEquation, SIMPLE.cpp:124-196
// mdot.mapFaceValues(U.valueAtFace); mdot.mapInteriorFaceValues(rhieChowCorrectFace)
// (SIMPLE.cpp:136-138)
void rhieChowFaces(Vector& mdot, Vector& U, const Tensor& D, Scalar& p) {
    Mesh* m = p.m;
    initFaceData(mdot);
    for (int64_t f = m->n_boundary; f < m->nf(); ++f) {
        V3 u = valueAtFace(U, f);
        mdot.fd[f] = u;
        mdot.ff[f] = dot(u, m->faces[f].areaVector());
    }
    for (auto& pa : m->patches) {
        if (pa.empty) continue;
        for (auto fid : pa.faces) {
            V3 u = valueAtFace(U, fid);
            mdot.fd[fid] = u;
            mdot.ff[fid] = dot(u, m->faces[fid].areaVector());
        }
    }
    for (int64_t f = m->n_boundary; f < m->nf(); ++f) {
        V3 u = rhieChow(f, U, D, p);
        mdot.fd[f] = u;
        mdot.ff[f] = dot(u, m->faces[f].areaVector());
    }
}

PressureResult solvePressureEquation(PrismSIMPLEControls c, std::vector<Transport*>& mom, Vector& U, Vector& mdot,
                                     Scalar& p, std::vector<Report>& rep) {
    Mesh* m = p.m;
    auto D = pressureCoeffs(mom, m);
    rhieChowFaces(mdot, U, *D, p);
    // p' field named like p, zero valued, fresh gradient scheme (scalar.cpp:260-304)
    auto pp = std::make_unique<Scalar>();
    pp->m = m;
    pp->name = p.name;
    pp->v.assign(m->nc(), 0.0);
    pp->bc = p.bc;
    pp->grad = makeGrad(m, p.grad->type);
    // constrainPPrime, SIMPLE.cpp:43-75
    std::vector<double> fv(m->nf(), 0.0);
    for (size_t q = 0; q < m->patches.size(); ++q) {
        const Patch& pa = m->patches[q];
        if (pa.empty) continue;
        int k = pp->bc[q].kind;
        if (!scalarHasHandler(k)) noHandler(m, (int32_t)q, "prism::algo::constrainPPrime()");
        if (scalarIsDirichlet(k) || k == PRISM_BC_SYMMETRY) {
            for (auto fid : pa.faces) fv[fid] = 0.0;
            continue;
        }
        for (auto fid : pa.faces) fv[fid] = valueAtFace(*pp, fid);
    }
    pp->fv = std::move(fv);
    if (c.p_ref_cell < 0 && needsPressureReference(*pp)) c.p_ref_cell = 0;
    Transport pEqn;
    pEqn.phi = pp.get();
    pEqn.ls.init(m);
    Scheme lap;
    lap.kind = SK_DIFF;
    lap.corrected = true;
    lap.kappa_t = D.get();
    lap.ls.init(m);
    pEqn.schemes.push_back(std::move(lap));
    pEqn.diff_idx = 0;
    Source div;
    div.kind = PRISM_SRC_DIVERGENCE;
    div.sign = PRISM_SIGN_NEGATIVE;
    div.coord = 0;
    div.U = &mdot;
    pEqn.sources.push_back(div);
    for (int64_t i = 0; i <= c.non_ortho_correctors; ++i) {
        auto r = solve(pEqn, solverOpts(c.pressure_max_iter, c.pressure_residual, c.p_ref_cell, c.p_ref_value, true));
        rep.push_back({pp->name + "_corr_" + std::to_string(i), r.iterations, r.initial_residual, r.final_residual,
                       r.converged != 0});
    }
    pp->fv.clear(); // clearFaceValues
    return {std::move(pp), std::move(D)};
}

// correctFields, SIMPLE.cpp:218-241
void correctFields(Vector& U, Vector& mdot, Scalar& p, const Tensor& D, Scalar& pp, double urf) {
    Mesh* m = U.m;
    for (int64_t c = 0; c < m->nc(); ++c) {
        V3 upd = U.cellValue(c) - mul(D.d[c], gradAtCell(pp, c));
        U.c[0]->at(c) = upd.x;
        U.c[1]->at(c) = upd.y;
        U.c[2]->at(c) = upd.z;
    }
    for (int64_t f = m->n_boundary; f < m->nf(); ++f) {
        V3 u = valueAtFace(mdot, f) - mul(D.valueAtFace(f), gradAtFace(pp, f));
        mdot.fd[f] = u;
        mdot.ff[f] = dot(u, m->faces[f].areaVector());
    }
    ++p.event;
    updatePrevTimeSteps(p);  // Scalar::update, scalar.cpp:311-320
    for (int64_t c = 0; c < m->nc(); ++c) p.v[c] = p.v[c] + (urf * pp.v[c]);
    ++p.event;
    p.fv.clear();
}

void simpleStep(const PrismSIMPLEControls& c, std::vector<Transport*>& mom, Vector& U, Vector& mdot, Scalar& p,
                std::vector<Report>& rep) {
    if (mom.size() != 2 && mom.size() != 3) fail(PRISM_BAD_ARG, "SIMPLE expects 2 or 3 momentum predictors");
    solveImplicitMomentum(c, mom, rep);
    auto r = solvePressureEquation(c, mom, U, mdot, p, rep);
    correctFields(U, mdot, p, *r.D, *r.pprime, c.pressure_urf);
}

// solveExplicitMomentum, PRIME.cpp:39-56
void solveExplicitMomentum(std::vector<Transport*>& mom) {
    for (auto* eq : mom) {
        updateCoeffs(*eq);
        Mesh* m = eq->phi->m;
        CSR A{m->nc(), m->rowptr.data(), m->col.data(), eq->ls.A.data()};
        std::vector<double> Ax;
        eq->phi->event += 2;
        spmv(A, eq->phi->v, Ax);
        std::vector<double> nv(m->nc());
        for (int64_t i = 0; i < m->nc(); ++i) {
            double ac = eq->ls.A[m->slot(i, i)];
            double H = Ax[i] - ac * eq->phi->v[i];
            nv[i] = (-H + eq->ls.b[i]) / ac;
        }
        ++eq->phi->event;
        eq->phi->v = nv;
    }
}

void primeStep(const PrismSIMPLEControls& pc, std::vector<Transport*>& mom, Vector& U, Vector& mdot, Scalar& p,
               std::vector<Report>& rep) {
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
    auto r = solvePressureEquation(c, mom, U, mdot, p, rep);
    correctFields(U, mdot, p, *r.D, *r.pprime, pc.pressure_urf);
}

// PISO::step, PISO.cpp:10-55
void pisoStep(const PrismPISOControls& pc, std::vector<Transport*>& mom, Vector& U, Vector& mdot, Scalar& p,
              std::vector<Report>& rep) {
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
    for (int64_t i = 0; i < pc.outer_iterations; ++i) {
        for (int64_t j = 0; j < pc.momentum_implicit_steps; ++j) simpleStep(sc, mom, U, mdot, p, rep);
        for (int64_t j = 1; j < pc.pressure_correction_steps; ++j) primeStep(sc, mom, U, mdot, p, rep);
    }
}

} // namespace orc

// ============================================================== C-ABI (orc_)
using namespace orc;

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

#define ORC_API extern "C" __attribute__((visibility("default")))
#define GUARD(...)                                                                       \
    try {                                                                                \
        __VA_ARGS__;                                                                     \
        return PRISM_OK;                                                                 \
    } catch (const Error& e) {                                                           \
        g_last_error = e.msg;                                                            \
        return e.status;                                                                 \
    } catch (const std::exception& e) {                                                  \
        g_last_error = e.what();                                                         \
        return PRISM_INTERNAL;                                                           \
    }
#define CHECK_ARG(cond, msg) \
    if (!(cond)) fail(PRISM_BAD_ARG, msg)

ORC_API const char* orc_last_error(void) { return g_last_error.c_str(); }
ORC_API const char* orc_status_string(int s) {
    static const char* names[] = {"OK", "NOT_CONVERGED", "BREAKDOWN", "NONFINITE", "BAD_ARG", "CUDA_ERROR",
                                  "INVALID_MESH", "NO_BC_HANDLER", "SPIN_TIMEOUT", "INTERNAL", "OUT_OF_MEMORY"};
    return (s >= 0 && s <= 10) ? names[s] : "UNKNOWN";
}

ORC_API int orc_mesh_from_unv(const PrismUnvMesh* d, PrismMesh** out) {
    GUARD({
        CHECK_ARG(d && out, "null argument");
        auto pm = new PrismMesh();
        pm->m = buildFromUnv(d);
        *out = pm;
    })
}
ORC_API int orc_mesh_info(const PrismMesh* pm, PrismMeshInfo* info) {
    GUARD({
        CHECK_ARG(pm && info, "null argument");
        const Mesh& m = *pm->m;
        info->n_cells = m.nc();
        info->n_faces = m.nf();
        info->n_boundary_faces = m.n_boundary;
        info->n_nonempty_boundary_faces = m.n_nonempty;
        info->nnz = (int64_t)m.col.size();
        info->n_patches = (int32_t)m.patches.size();
        info->n_vertices = (int64_t)m.verts.size();
        int64_t ncv = 0;
        for (auto& c : m.cells) ncv += (int64_t)c.vids.size();
        info->n_cell_vertices = ncv;
        // levels of the in-place Green-Gauss sweep dependency (lower-id neighbours)
        std::vector<int32_t> lev(m.nc(), 0);
        int32_t nl = 0;
        for (int64_t c = 0; c < m.nc(); ++c) {
            int32_t l = 0;
            for (auto f : m.cells[c].faces)
                if (m.faces[f].nbr >= 0) {
                    int64_t o = m.other(c, f);
                    if (o < c) l = std::max(l, lev[o] + 1);
                }
            lev[c] = l;
            nl = std::max(nl, l + 1);
        }
        info->n_gs_levels = nl;
    })
}
ORC_API int orc_mesh_export(const PrismMesh* pm, PrismMeshExport* o) {
    GUARD({
        CHECK_ARG(pm && o, "null argument");
        const Mesh& m = *pm->m;
        int64_t nf = m.nf(), nc = m.nc();
        for (int64_t f = 0; f < nf; ++f) {
            const Face& fc = m.faces[f];
            if (o->owner) o->owner[f] = fc.owner;
            if (o->neighbor) o->neighbor[f] = fc.nbr;
            if (o->face_patch) o->face_patch[f] = fc.nbr >= 0 ? -1 : fc.patch;
            if (o->face_area) o->face_area[f] = fc.area;
            for (int k = 0; k < 3; ++k) {
                if (o->face_normal) o->face_normal[k * nf + f] = fc.normal[k];
                if (o->face_center) o->face_center[k * nf + f] = fc.center[k];
            }
        }
        int64_t pos = 0;
        for (int64_t c = 0; c < nc; ++c) {
            if (o->cell_volume) o->cell_volume[c] = m.cells[c].volume;
            for (int k = 0; k < 3; ++k)
                if (o->cell_center) o->cell_center[k * nc + c] = m.cells[c].center[k];
            if (o->cell_face_offsets) o->cell_face_offsets[c] = pos;
            for (auto f : m.cells[c].faces) {
                if (o->cell_faces) o->cell_faces[pos] = f;
                ++pos;
            }
        }
        if (o->cell_face_offsets) o->cell_face_offsets[nc] = pos;
        for (int64_t i = 0; i <= nc; ++i)
            if (o->csr_rowptr) o->csr_rowptr[i] = m.rowptr[i];
        for (size_t k = 0; k < m.col.size(); ++k)
            if (o->csr_col) o->csr_col[k] = m.col[k];
        pos = 0;
        for (size_t p = 0; p < m.patches.size(); ++p) {
            if (o->patch_face_offsets) o->patch_face_offsets[p] = pos;
            for (auto f : m.patches[p].faces) {
                if (o->patch_faces) o->patch_faces[pos] = f;
                ++pos;
            }
        }
        if (o->patch_face_offsets) o->patch_face_offsets[m.patches.size()] = pos;
        const int64_t nv = (int64_t)m.verts.size();
        for (int64_t v = 0; v < nv; ++v)
            for (int k = 0; k < 3; ++k)
                if (o->vertex_coords) o->vertex_coords[k * nv + v] = m.verts[v][k];
        pos = 0;
        for (int64_t c = 0; c < nc; ++c) {
            if (o->cell_vertex_offsets) o->cell_vertex_offsets[c] = pos;
            for (auto v : m.cells[c].vids) {
                if (o->cell_vertices) o->cell_vertices[pos] = v;
                ++pos;
            }
        }
        if (o->cell_vertex_offsets) o->cell_vertex_offsets[nc] = pos;
        if (o->cell_original) std::copy(m.cell_orig.begin(), m.cell_orig.end(), o->cell_original);
    })
}
ORC_API int orc_mesh_destroy(PrismMesh* pm) { GUARD({ delete pm; }) }
ORC_API int orc_mesh_reorder(PrismMesh* pm, int32_t reverse) {
    GUARD({
        CHECK_ARG(pm, "null argument");
        CHECK_ARG(!pm->m->frozen, "reorder the mesh before creating fields on it");
        reorderCells(*pm->m, reverse != 0);
    })
}

ORC_API int orc_scalar_create(PrismMesh* pm, const char* name, const double* values, int32_t grad_scheme,
                              const PrismBC* bcs, PrismScalar** out) {
    GUARD({
        CHECK_ARG(pm && name && bcs && out, "null argument");
        pm->m->frozen = true;
        CHECK_ARG(grad_scheme == PRISM_GRAD_LEAST_SQUARES || grad_scheme == PRISM_GRAD_GREEN_GAUSS, "bad gradient scheme");
        auto s = std::make_shared<Scalar>();
        s->m = pm->m.get();
        s->name = name;
        s->v.assign(s->m->nc(), 0.0);
        if (values) std::copy(values, values + s->m->nc(), s->v.begin());
        s->bc.assign(bcs, bcs + s->m->patches.size());
        s->grad = makeGrad(s->m, grad_scheme);
        auto* ps = new PrismScalar();
        ps->s = s;
        *out = ps;
    })
}
ORC_API int orc_scalar_destroy(PrismScalar* s) { GUARD({ delete s; }) }
ORC_API int orc_scalar_set_values(PrismScalar* ps, const double* v) {
    GUARD({
        CHECK_ARG(ps && v, "null argument");
        ++ps->s->event;
        std::copy(v, v + ps->s->m->nc(), ps->s->v.begin());
    })
}
ORC_API int orc_scalar_get_values(const PrismScalar* ps, double* v) {
    GUARD({
        CHECK_ARG(ps && v, "null argument");
        std::copy(ps->s->v.begin(), ps->s->v.end(), v);
    })
}
ORC_API int orc_scalar_set_face_values(PrismScalar* ps, const double* fv) {
    GUARD({
        CHECK_ARG(ps, "null argument");
        if (fv) ps->s->fv.assign(fv, fv + ps->s->m->nf());
        else ps->s->fv.clear();
    })
}
ORC_API int orc_scalar_face_values(PrismScalar* ps, double* out) {
    GUARD({
        CHECK_ARG(ps && out, "null argument");
        Mesh* m = ps->s->m;
        for (int64_t f = 0; f < m->nf(); ++f) {
            const Face& fc = m->faces[f];
            out[f] = (fc.nbr < 0 && m->patches[fc.patch].empty) ? 0.0 : valueAtFace(*ps->s, f);
        }
    })
}
ORC_API int orc_scalar_grad(PrismScalar* ps, double* out) {
    GUARD({
        CHECK_ARG(ps && out, "null argument");
        int64_t n = ps->s->m->nc();
        for (int64_t c = 0; c < n; ++c) {
            V3 g = gradAtCell(*ps->s, c);
            out[c] = g.x;
            out[n + c] = g.y;
            out[2 * n + c] = g.z;
        }
    })
}
ORC_API int orc_scalar_set_history_size(PrismScalar* ps, int32_t n) {
    GUARD({
        CHECK_ARG(ps && n >= 0, "bad argument");
        setHistorySize(*ps->s, (size_t)n);
    })
}
ORC_API int orc_scalar_update_prev_time_steps(PrismScalar* ps) {
    GUARD({
        CHECK_ARG(ps, "null argument");
        updatePrevTimeSteps(*ps->s);
    })
}
ORC_API int orc_scalar_update(PrismScalar* ps, const double* v) {
    GUARD({
        CHECK_ARG(ps && v, "null argument");
        updatePrevTimeSteps(*ps->s);
        std::copy(v, v + ps->s->m->nc(), ps->s->v.begin());
        ++ps->s->event;
        ps->s->fv.clear();
    })
}
ORC_API int orc_scalar_history(const PrismScalar* ps, int32_t index, double* out, int32_t* available) {
    GUARD({
        CHECK_ARG(ps && out && available && index >= 0, "bad argument");
        const Scalar& s = *ps->s;
        *available = (size_t)index < s.hist.size() ? 1 : 0;
        if (*available) std::copy(s.hist[index].begin(), s.hist[index].end(), out);
    })
}
ORC_API int orc_scalar_compute_gradients(PrismScalar* ps) {
    GUARD({
        CHECK_ARG(ps, "null argument");
        computeAllCellGradients(*ps->s);
    })
}
// Scalar::setGradScheme (scalar.cpp:252-258): a fresh scheme object of the kind
ORC_API int orc_scalar_set_grad_scheme(PrismScalar* ps, int32_t grad_scheme) {
    GUARD({
        CHECK_ARG(ps, "null argument");
        CHECK_ARG(grad_scheme == PRISM_GRAD_LEAST_SQUARES || grad_scheme == PRISM_GRAD_GREEN_GAUSS, "bad gradient scheme");
        ps->s->grad = makeGrad(ps->s->m, grad_scheme);
    })
}

ORC_API int orc_vector_create(PrismMesh* pm, const char* name, const double* values, int32_t grad_scheme,
                              const PrismBC* bcs, PrismVector** out) {
    GUARD({
        CHECK_ARG(pm && name && bcs && out, "null argument");
        pm->m->frozen = true;
        CHECK_ARG(grad_scheme == PRISM_GRAD_LEAST_SQUARES || grad_scheme == PRISM_GRAD_GREEN_GAUSS, "bad gradient scheme");
        auto* pv = new PrismVector();
        pv->v = std::make_unique<Vector>();
        Vector& U = *pv->v;
        U.m = pm->m.get();
        U.name = name;
        U.bc.assign(bcs, bcs + U.m->patches.size());
        int64_t n = U.m->nc();
        const char* suf[3] = {"_x", "_y", "_z"};
        for (int k = 0; k < 3; ++k) {
            auto s = std::make_shared<Scalar>();
            s->m = U.m;
            s->name = std::string(name) + suf[k];
            s->coord = k;
            s->v.assign(n, 0.0);
            if (values) std::copy(values + k * n, values + (k + 1) * n, s->v.begin());
            s->bc = U.bc;
            s->grad = makeGrad(U.m, grad_scheme);
            U.c[k] = s;
            pv->comp[k].s = s;
        }
        *out = pv;
    })
}
ORC_API int orc_vector_clone(const PrismVector* src, PrismVector** out) {
    GUARD({
        CHECK_ARG(src && out, "null argument");
        auto* pv = new PrismVector();
        pv->v = std::make_unique<Vector>(*src->v);
        for (int k = 0; k < 3; ++k) {
            auto s = std::make_shared<Scalar>(*src->v->c[k]); // copies share the gradient scheme
            pv->v->c[k] = s;
            pv->comp[k].s = s;
        }
        *out = pv;
    })
}
ORC_API int orc_vector_destroy(PrismVector* v) { GUARD({ delete v; }) }
ORC_API int orc_vector_component(PrismVector* pv, int32_t coord, PrismScalar** out) {
    GUARD({
        CHECK_ARG(pv && out && coord >= 0 && coord < 3, "bad argument");
        *out = &pv->comp[coord];
    })
}
ORC_API int orc_vector_set_values(PrismVector* pv, const double* v) {
    GUARD({
        CHECK_ARG(pv && v, "null argument");
        int64_t n = pv->v->m->nc();
        for (int k = 0; k < 3; ++k) {
            ++pv->v->c[k]->event;
            std::copy(v + k * n, v + (k + 1) * n, pv->v->c[k]->v.begin());
        }
    })
}
ORC_API int orc_vector_get_values(const PrismVector* pv, double* v) {
    GUARD({
        CHECK_ARG(pv && v, "null argument");
        int64_t n = pv->v->m->nc();
        for (int k = 0; k < 3; ++k) std::copy(pv->v->c[k]->v.begin(), pv->v->c[k]->v.end(), v + k * n);
    })
}
ORC_API int orc_vector_face_flux(PrismVector* pv, double* out) {
    GUARD({
        CHECK_ARG(pv && out, "null argument");
        Mesh* m = pv->v->m;
        for (int64_t f = 0; f < m->nf(); ++f) {
            const Face& fc = m->faces[f];
            out[f] = (fc.nbr < 0 && m->patches[fc.patch].empty) ? 0.0 : fluxAtFace(*pv->v, f);
        }
    })
}

// GeneralVector::setFaceFluxValues, vector.h:359-377
ORC_API int orc_vector_set_face_flux(PrismVector* pv, const double* flux) {
    GUARD({
        CHECK_ARG(pv && flux, "null argument");
        Vector& U = *pv->v;
        U.ff.assign(flux, flux + U.m->nf());
        U.has_ff = true;
    })
}

// ---------------------------------------------------------------- diagnostics
namespace {
std::shared_ptr<Scalar> resultScalar(Mesh* m, const std::string& name, std::vector<double> v) {
    // field::Scalar(name, mesh, data): no boundary handlers, least-squares gradient
    auto s = std::make_shared<Scalar>();
    s->m = m;
    s->name = name;
    s->v = std::move(v);
    PrismBC none{};
    none.kind = PRISM_BC_UNKNOWN;
    s->bc.assign(m->patches.size(), none);
    s->grad = makeGrad(m, PRISM_GRAD_LEAST_SQUARES);
    return s;
}

// ensureCache, export.cpp:44-71: vertex -> adjacent cells in cell order
std::vector<std::vector<int64_t>> vertexCells(const Mesh& m) {
    std::vector<std::vector<int64_t>> v2c(m.verts.size());
    for (int64_t c = 0; c < m.nc(); ++c)
        for (auto v : m.cells[c].vids) v2c[v].push_back(c);
    return v2c;
}

// cellToPoint, export.cpp:73-111
std::vector<double> cellToPoint(const Mesh& m, const double* cell_data, int64_t ncomp) {
    auto v2c = vertexCells(m);
    const int64_t nv = (int64_t)m.verts.size();
    std::vector<double> out(nv * ncomp, 0.0);
    for (int64_t v = 0; v < nv; ++v) {
        const auto& adj = v2c[v];
        if (adj.empty())
            fail(PRISM_INVALID_MESH,
                 "Vertex " + std::to_string(v) + " has no adjacent cells; point data cannot be computed.");
        std::vector<double> w(adj.size());
        double sw = 0.0;
        for (size_t i = 0; i < adj.size(); ++i) {
            double d = norm(m.verts[v] - m.cells[adj[i]].center);
            w[i] = 1.0 / std::max(d, EPSILON);
            sw += w[i];
        }
        for (size_t i = 0; i < adj.size(); ++i) {
            double wi = w[i] / sw;
            for (int64_t k = 0; k < ncomp; ++k) out[v * ncomp + k] += wi * cell_data[adj[i] * ncomp + k];
        }
    }
    return out;
}
}  // namespace

// ops::div, operations.h:84-100 (fluxSumAtCell, :144-169)
ORC_API int orc_ops_div(PrismVector* pv, PrismScalar** out) {
    GUARD({
        CHECK_ARG(pv && out, "null argument");
        const Vector& U = *pv->v;
        Mesh* m = U.m;
        std::vector<double> d(m->nc());
        for (int64_t c = 0; c < m->nc(); ++c) d[c] = fluxSumAtCell(U, c) / m->cells[c].volume;
        auto* ps = new PrismScalar();
        ps->s = resultScalar(m, "div(" + U.name + ")", std::move(d));
        *out = ps;
    })
}

// monitor::courantNumber, courant.cpp:7-24
ORC_API int orc_courant_number(PrismVector* pv, double dt, PrismScalar** out) {
    GUARD({
        CHECK_ARG(pv && out, "null argument");
        const Vector& U = *pv->v;
        Mesh* m = U.m;
        std::vector<double> co(m->nc(), 0.0);
        for (int64_t c = 0; c < m->nc(); ++c) {
            double flux_sum = 0.0;
            for (auto f : m->cells[c].faces) {
                const Face& fc = m->faces[f];
                if (fc.nbr < 0 && m->patches[fc.patch].empty) continue;
                flux_sum += std::abs(fluxAtFace(U, f));
            }
            co[c] = 0.5 * dt * flux_sum / m->cells[c].volume;
        }
        auto* ps = new PrismScalar();
        ps->s = resultScalar(m, "Co", std::move(co));
        *out = ps;
    })
}

ORC_API int orc_cell_to_point(PrismMesh* pm, const double* cell_data, int32_t ncomp, double* point_data) {
    GUARD({
        CHECK_ARG(pm && cell_data && point_data, "null argument");
        CHECK_ARG(ncomp >= 1 && ncomp <= 9, "n_components must be 1..9");
        auto r = cellToPoint(*pm->m, cell_data, ncomp);
        std::copy(r.begin(), r.end(), point_data);
    })
}
ORC_API int orc_scalar_to_points(PrismScalar* ps, double* point_data) {
    GUARD({
        CHECK_ARG(ps && point_data, "null argument");
        auto r = cellToPoint(*ps->s->m, ps->s->v.data(), 1);
        std::copy(r.begin(), r.end(), point_data);
    })
}
ORC_API int orc_vector_to_points(PrismVector* pv, double* point_data) {
    GUARD({
        CHECK_ARG(pv && point_data, "null argument");
        const Vector& U = *pv->v;
        const int64_t n = U.m->nc();
        std::vector<double> flat(3 * n);  // flattenVector, export.cpp:139-151
        for (int64_t c = 0; c < n; ++c)
            for (int k = 0; k < 3; ++k) flat[3 * c + k] = U.c[k]->v[c];
        auto r = cellToPoint(*U.m, flat.data(), 3);
        std::copy(r.begin(), r.end(), point_data);
    })
}

ORC_API int orc_tensor_create(PrismMesh* pm, const char* name, const double* values, PrismTensor** out) {
    GUARD({
        CHECK_ARG(pm && out, "null argument");
        pm->m->frozen = true;
        (void)name;
        auto* pt = new PrismTensor();
        pt->t = std::make_unique<Tensor>();
        pt->t->m = pm->m.get();
        int64_t n = pt->t->m->nc();
        pt->t->d.assign(n, M3{});
        for (int64_t c = 0; c < n; ++c)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    pt->t->d[c].m[i][j] = values ? values[(3 * i + j) * n + c] : (i == j ? 1.0 : 0.0);
        *out = pt;
    })
}
ORC_API int orc_tensor_destroy(PrismTensor* t) { GUARD({ delete t; }) }

ORC_API int orc_rhie_chow(PrismVector* pmdot, PrismVector* pU, PrismTensor* pD, PrismScalar* pp) {
    GUARD({
        CHECK_ARG(pmdot && pU && pD && pp, "null argument");
        rhieChowFaces(*pmdot->v, *pU->v, *pD->t, *pp->s);
    })
}

ORC_API int orc_transport_create(PrismScalar* phi, PrismTransport** out) {
    GUARD({
        CHECK_ARG(phi && out, "null argument");
        auto* pt = new PrismTransport();
        pt->eq.phi = phi->s.get();
        pt->eq.ls.init(phi->s->m);
        *out = pt;
    })
}
ORC_API int orc_transport_destroy(PrismTransport* eq) { GUARD({ delete eq; }) }
ORC_API int orc_transport_add_convection(PrismTransport* pt, int32_t scheme, PrismVector* U) {
    GUARD({
        CHECK_ARG(pt && U && scheme >= PRISM_CONV_UPWIND && scheme <= PRISM_CONV_SMART, "bad argument");
        Scheme s;
        s.kind = SK_CONV;
        s.conv = scheme;
        s.U = U->v.get();
        s.ls.init(pt->eq.phi->m);
        pt->eq.schemes.push_back(std::move(s));
        pt->eq.conv_idx = (int)pt->eq.schemes.size() - 1;
    })
}
ORC_API int orc_transport_add_diffusion(PrismTransport* pt, int32_t corrected, int32_t corrector, PrismScalar* ks,
                                        PrismTensor* kt) {
    GUARD({
        CHECK_ARG(pt && ((ks != nullptr) != (kt != nullptr)), "exactly one diffusion coefficient");
        CHECK_ARG(corrector >= 0 && corrector <= 2, "bad corrector");
        Scheme s;
        s.kind = SK_DIFF;
        s.corrected = corrected != 0;
        s.corrector = corrector;
        s.kappa_s = ks ? ks->s.get() : nullptr;
        s.kappa_t = kt ? kt->t.get() : nullptr;
        s.ls.init(pt->eq.phi->m);
        pt->eq.schemes.push_back(std::move(s));
        pt->eq.diff_idx = (int)pt->eq.schemes.size() - 1;
    })
}
ORC_API int orc_transport_add_temporal(PrismTransport* pt, int32_t kind, double dt) {
    GUARD({
        CHECK_ARG(pt, "null argument");
        CHECK_ARG(kind == PRISM_TEMPORAL_BACKWARD_EULER || kind == PRISM_TEMPORAL_ADAM_MOULTON, "bad temporal scheme");
        CHECK_ARG(dt > 0.0, "prism::scheme::temporal::ITemporal(phi, dt): dt must be positive");
        for (const auto& q : pt->eq.schemes)
            CHECK_ARG(q.kind != SK_TEMPORAL, "equation already has a temporal scheme");
        Scheme s;
        s.kind = SK_TEMPORAL;
        s.temporal = kind;
        s.dt = dt;
        s.ls.init(pt->eq.phi->m);
        pt->eq.schemes.push_back(std::move(s));
    })
}
ORC_API int orc_transport_set_time_step(PrismTransport* pt, double dt) {
    GUARD({
        CHECK_ARG(pt, "null argument");
        CHECK_ARG(dt > 0.0, "prism::scheme::temporal::ITemporal::setTimeStep(): dt must be positive");
        bool found = false;
        for (auto& q : pt->eq.schemes)
            if (q.kind == SK_TEMPORAL) {
                q.dt = dt;
                found = true;
            }
        CHECK_ARG(found, "equation has no temporal scheme");
    })
}
ORC_API int orc_transport_add_source(PrismTransport* pt, int32_t kind, int32_t sign, PrismScalar* ss,
                                     PrismVector* sv, int32_t coord) {
    GUARD({
        CHECK_ARG(pt, "null argument");
        Source s;
        s.kind = kind;
        s.sign = sign;
        s.coord = coord;
        if (kind == PRISM_SRC_DIVERGENCE) { CHECK_ARG(sv, "divergence needs a vector"); s.U = sv->v.get(); }
        else { CHECK_ARG(ss, "source needs a scalar"); s.s = ss->s.get(); }
        CHECK_ARG(kind != PRISM_SRC_GRADIENT || (coord >= 0 && coord < 3), "bad coord");
        pt->eq.sources.push_back(s);
    })
}
ORC_API int orc_transport_add_symmetry_handler(PrismTransport* pt) {
    GUARD({
        CHECK_ARG(pt, "null argument");
        pt->eq.symmetry = true;
    })
}
ORC_API int orc_transport_set_urf(PrismTransport* pt, double f) { GUARD({ CHECK_ARG(pt, "null"); setURF(pt->eq, f); }) }
ORC_API int orc_transport_update_coeffs(PrismTransport* pt) { GUARD({ CHECK_ARG(pt, "null"); updateCoeffs(pt->eq); }) }
ORC_API int orc_transport_relax(PrismTransport* pt) { GUARD({ CHECK_ARG(pt, "null"); relax(pt->eq); }) }
ORC_API int orc_transport_zero_coeffs(PrismTransport* pt) { GUARD({ CHECK_ARG(pt, "null"); zeroOutCoeffs(pt->eq); }) }
ORC_API int orc_transport_get_system(const PrismTransport* pt, double* vals, double* rhs) {
    GUARD({
        CHECK_ARG(pt, "null");
        if (vals) std::copy(pt->eq.ls.A.begin(), pt->eq.ls.A.end(), vals);
        if (rhs) std::copy(pt->eq.ls.b.begin(), pt->eq.ls.b.end(), rhs);
    })
}

ORC_API void orc_solve_opts_default(PrismSolveOpts* o) {
    std::memset(o, 0, sizeof(*o));
    o->method = PRISM_SOLVER_BICGSTAB;
    o->precision = PRISM_PREC_FP64;
    o->n_iter = 10;
    o->eps = 1e-7;
    o->ref_cell = -1;
    o->clear_coeffs = 1;
}
ORC_API int orc_solve(PrismTransport* pt, const PrismSolveOpts* o, PrismSolveResult* r) {
    GUARD({
        CHECK_ARG(pt && o && r, "null argument");
        *r = solve(pt->eq, *o);
    })
}
ORC_API int orc_solve_csr(int64_t n, const int64_t* rp, const int64_t* ci, const double* v, const double* b,
                          double* x, const PrismSolveOpts* o, PrismSolveResult* r) {
    GUARD({
        CHECK_ARG(rp && ci && v && b && x && o, "null argument");
        CSR A{n, rp, ci, v};
        std::vector<double> bb(b, b + n), xx(x, x + n);
        int64_t k = 0;
        if (o->method == PRISM_SOLVER_JACOBI) jacobiStep(A, bb, xx);
        else k = bicgstabStep(A, bb, xx);
        std::copy(xx.begin(), xx.end(), x);
        if (r) {
            std::memset(r, 0, sizeof(*r));
            r->iterations = 1;
            r->krylov_iterations = k;
            r->final_residual = scaledResidual(A, xx, bb);
        }
    })
}

ORC_API void orc_simple_controls_default(PrismSIMPLEControls* c) { simpleDefaults(c); }
ORC_API void orc_piso_controls_default(PrismPISOControls* c) { pisoDefaults(c); }

static std::vector<Transport*> momVec(PrismTransport* const* mom, int32_t n) {
    std::vector<Transport*> v;
    for (int32_t i = 0; i < n; ++i) v.push_back(&mom[i]->eq);
    return v;
}
static void writeReports(const std::vector<Report>& rep, PrismReport* out, int32_t max, int32_t* n) {
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
ORC_API int orc_simple_step(const PrismSIMPLEControls* c, PrismTransport* const* mom, int32_t n_mom, PrismVector* U,
                            PrismVector* mdot, PrismScalar* p, const PrismSolveOpts* so, PrismReport* rep, int32_t max,
                            int32_t* n) {
    GUARD({
        CHECK_ARG(c && mom && U && mdot && p, "null argument");
        (void)so;
        auto v = momVec(mom, n_mom);
        std::vector<Report> r;
        simpleStep(*c, v, *U->v, *mdot->v, *p->s, r);
        writeReports(r, rep, max, n);
    })
}
ORC_API int orc_prime_step(const PrismSIMPLEControls* c, PrismTransport* const* mom, int32_t n_mom, PrismVector* U,
                           PrismVector* mdot, PrismScalar* p, const PrismSolveOpts* so, PrismReport* rep, int32_t max,
                           int32_t* n) {
    GUARD({
        CHECK_ARG(c && mom && U && mdot && p, "null argument");
        (void)so;
        auto v = momVec(mom, n_mom);
        std::vector<Report> r;
        primeStep(*c, v, *U->v, *mdot->v, *p->s, r);
        writeReports(r, rep, max, n);
    })
}
ORC_API int orc_piso_step(const PrismPISOControls* c, PrismTransport* const* mom, int32_t n_mom, PrismVector* U,
                          PrismVector* mdot, PrismScalar* p, const PrismSolveOpts* so, PrismReport* rep, int32_t max,
                          int32_t* n) {
    GUARD({
        CHECK_ARG(c && mom && U && mdot && p, "null argument");
        (void)so;
        auto v = momVec(mom, n_mom);
        std::vector<Report> r;
        pisoStep(*c, v, *U->v, *mdot->v, *p->s, r);
        writeReports(r, rep, max, n);
    })
}
ORC_API int orc_needs_pressure_reference(PrismScalar* p, int32_t* out) {
    GUARD({
        CHECK_ARG(p && out, "null argument");
        *out = needsPressureReference(*p->s) ? 1 : 0;
    })
}

