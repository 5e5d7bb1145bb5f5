// mesh_build.cpp -- host conversion of a UNV-form mesh to the flattened PMesh.
//
// Reproduces the face numbering of UnvToPMeshConverter (mesh/unv.cpp:124-372)
// and the PMesh face permutation (mesh/pmesh.cpp:51-123):
//   * faces are created in order of first appearance: boundary elements as they
//     are read, cell faces in cell order and local face order (unv.cpp:19-58);
//   * the first cell touching a face owns it, the second is its neighbour;
//   * boundary faces are ordered by the moment their owner was assigned;
//   * PMesh orders faces [non-empty boundary | empty boundary | interior].
// Face and cell geometry follow mesh/face.cpp:5-41 and mesh/cell.cpp:7-41 with
// the same operation order (host code, no FMA contraction).
//
// Faces are matched by sorting 128-bit keys of their sorted vertex ids rather
// than by the reference's vertex trie: O(N log N), a few seconds for 10^7 cell
// faces, with identical results.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <thread>

#include "mesh_build.h"

namespace pb {

namespace {

struct V3 {
    double x, y, z;
};
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 divs(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

const int kHexFaces[6][4] = {{1, 2, 6, 5}, {0, 4, 7, 3}, {2, 3, 7, 6}, {0, 1, 5, 4}, {4, 5, 6, 7}, {0, 3, 2, 1}};
const int kTetFaces[4][3] = {{0, 2, 1}, {1, 2, 3}, {0, 1, 3}, {0, 3, 2}};
const int kWedgeFaces[5][4] = {{0, 2, 1, -1}, {3, 4, 5, -1}, {0, 1, 4, 3}, {0, 3, 5, 2}, {1, 2, 5, 4}};

int nLocalFaces(int kind) { return kind == PRISM_ELEM_HEX ? 6 : kind == PRISM_ELEM_TETRA ? 4 : 5; }

// vertex ids of local face l of element e (l < 0: the element itself)
int faceVerts(const PrismUnvMesh* d, int64_t e, int l, int64_t* out) {
    const int64_t* en = d->elem_nodes + d->elem_offsets[e];
    int kind = d->elem_kind[e];
    if (l < 0) {
        int n = (int)(d->elem_offsets[e + 1] - d->elem_offsets[e]);
        for (int i = 0; i < n; ++i) out[i] = en[i];
        return n;
    }
    if (kind == PRISM_ELEM_HEX) {
        for (int i = 0; i < 4; ++i) out[i] = en[kHexFaces[l][i]];
        return 4;
    }
    if (kind == PRISM_ELEM_TETRA) {
        for (int i = 0; i < 3; ++i) out[i] = en[kTetFaces[l][i]];
        return 3;
    }
    int n = kWedgeFaces[l][3] < 0 ? 3 : 4;
    for (int i = 0; i < n; ++i) out[i] = en[kWedgeFaces[l][i]];
    return n;
}

// f(begin, end) over [0, n) split across host threads; f must not throw
template <typename F>
void parallelFor(int64_t n, F&& f) {
    const unsigned hw = std::thread::hardware_concurrency();
    const unsigned nt = std::min<unsigned>(hw ? hw : 1, 32);
    if (n < 200000 || nt == 1) {
        f(int64_t(0), n);
        return;
    }
    const int64_t chunk = (n + nt - 1) / nt;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) {
        const int64_t b = t * chunk, e = std::min<int64_t>(n, b + chunk);
        if (b >= e) break;
        th.emplace_back([&f, b, e] { f(b, e); });
    }
    for (auto& x : th) x.join();
}

struct Key {
    uint64_t hi, lo;
    bool operator<(const Key& o) const { return hi != o.hi ? hi < o.hi : lo < o.lo; }
    bool operator==(const Key& o) const { return hi == o.hi && lo == o.lo; }
};
Key makeKey(const int64_t* v, int n) {
    uint64_t s[4] = {~0ull, ~0ull, ~0ull, ~0ull};
    for (int i = 0; i < n; ++i) s[i] = (uint64_t)v[i];
    std::sort(s, s + n);
    return {(s[0] << 32) | (s[1] & 0xffffffffull), (s[2] << 32) | (s[3] & 0xffffffffull)};
}

// Face::Face (mesh/face.cpp:5-41)
void faceGeometry(const V3* fv, int n, double& area, V3& normal, V3& center) {
    V3 gc{0, 0, 0};
    for (int i = 0; i < n; ++i) gc = add(gc, fv[i]);
    gc = divs(gc, (double)n);
    normal = {0, 0, 0};
    area = 0.0;
    center = {0, 0, 0};
    for (int i = 0; i < n; ++i) {
        V3 v1 = fv[i], v2 = fv[(i + 1) % n], v3 = gc;
        V3 sc = divs(add(add(v1, v2), v3), 3.0);
        V3 sn = cross(sub(v2, v1), sub(v3, v1));
        double sa = std::sqrt(dot(sn, sn)) / 2.0;
        normal = add(normal, sn);
        area += sa;
        center = add(center, scale(sc, sa));
    }
    center = divs(center, area);
    normal = divs(normal, std::sqrt(dot(normal, normal)));
}

}  // namespace

std::unique_ptr<HostMesh> buildHostMesh(const PrismUnvMesh* d) {
    if (!d) fail(PRISM_BAD_ARG, "null mesh description");
    if (d->n_nodes <= 0) fail(PRISM_INVALID_MESH, "UnvToPMeshConverter(): mesh has zero vertices");
    if (d->n_nodes >= (int64_t(1) << 31)) fail(PRISM_INVALID_MESH, "too many nodes");
    const int64_t ne = d->n_elements;
    std::vector<V3> X(d->n_nodes);
    for (int64_t i = 0; i < d->n_nodes; ++i) X[i] = {d->xyz[3 * i], d->xyz[3 * i + 1], d->xyz[3 * i + 2]};

    // ---- occurrences of faces in reading order
    struct Occ {
        Key key;
        int64_t elem;
        int32_t local;  // -1: boundary element
        int32_t cell;   // -1: boundary element
    };
    // validation and counts (serial), then the keys of every occurrence (threads)
    std::vector<int64_t> cell_elem;
    std::vector<int64_t> occ_off(ne + 1, 0);
    std::vector<int32_t> cell_of_elem(ne, -1);
    int64_t tmp[8];
    for (int64_t e = 0; e < ne; ++e) {
        int k = d->elem_kind[e];
        int64_t nn = d->elem_offsets[e + 1] - d->elem_offsets[e];
        const int64_t* en = d->elem_nodes + d->elem_offsets[e];
        for (int64_t i = 0; i < nn; ++i)
            if (en[i] < 0 || en[i] >= d->n_nodes) fail(PRISM_INVALID_MESH, "element node index out of range");
        int cnt = 0;
        if (k == PRISM_ELEM_LINE) {
        } else if (k == PRISM_ELEM_TRIANGLE || k == PRISM_ELEM_QUAD) {
            int n = faceVerts(d, e, -1, tmp);
            if (n != (k == PRISM_ELEM_QUAD ? 4 : 3)) fail(PRISM_INVALID_MESH, "bad boundary element");
            cnt = 1;
        } else if (k == PRISM_ELEM_HEX || k == PRISM_ELEM_TETRA || k == PRISM_ELEM_WEDGE) {
            int need = k == PRISM_ELEM_HEX ? 8 : k == PRISM_ELEM_TETRA ? 4 : 6;
            if (nn != need) fail(PRISM_INVALID_MESH, "cell element with a wrong node count");
            cell_of_elem[e] = (int32_t)cell_elem.size();
            cell_elem.push_back(e);
            cnt = nLocalFaces(k);
        } else {
            fail(PRISM_INVALID_MESH, "unsupported element type");
        }
        occ_off[e + 1] = occ_off[e] + cnt;
    }
    std::vector<Occ> occ(occ_off[ne]);
    parallelFor(ne, [&](int64_t e0, int64_t e1) {
        int64_t t[8];
        for (int64_t e = e0; e < e1; ++e) {
            const int64_t o0 = occ_off[e], cnt = occ_off[e + 1] - o0;
            if (cnt == 0) continue;
            if (cell_of_elem[e] < 0) {
                int n = faceVerts(d, e, -1, t);
                occ[o0] = {makeKey(t, n), e, -1, -1};
            } else {
                for (int l = 0; l < (int)cnt; ++l) {
                    int n = faceVerts(d, e, l, t);
                    occ[o0 + l] = {makeKey(t, n), e, l, cell_of_elem[e]};
                }
            }
        }
    });
    if (cell_elem.empty()) fail(PRISM_INVALID_MESH, "mesh is empty or two dimensional");
    if (cell_elem.size() >= (size_t(1) << 31)) fail(PRISM_INVALID_MESH, "too many cells");

    // ---- match occurrences: order by (key, reading order). A stable counting sort
    // on the smallest node id groups the occurrences into small buckets (the faces
    // around one node), each then sorted by the full key: O(n) instead of a global sort.
    std::vector<int64_t> ord(occ.size());
    {
        std::vector<int64_t> start((size_t)d->n_nodes + 1, 0);
        for (const Occ& o : occ) start[(o.key.hi >> 32) + 1]++;
        for (int64_t v = 0; v < d->n_nodes; ++v) start[v + 1] += start[v];
        std::vector<int64_t> fill(start.begin(), start.end() - 1);
        for (size_t o = 0; o < occ.size(); ++o) ord[fill[occ[o].key.hi >> 32]++] = (int64_t)o;
        parallelFor(d->n_nodes, [&](int64_t v0, int64_t v1) {
            for (int64_t v = v0; v < v1; ++v) {
                auto b = ord.begin() + start[v], e = ord.begin() + start[v + 1];
                if (e - b > 1)
                    std::sort(b, e, [&](int64_t a, int64_t c) {
                        if (occ[a].key == occ[c].key) return a < c;
                        return occ[a].key < occ[c].key;
                    });
            }
        });
    }
    struct Run {
        int64_t first;   // occurrence index of creation
        int64_t owner_occ;
        int32_t owner, nbr;
        bool bface;
    };
    std::vector<Run> runs;
    std::vector<int64_t> run_of_occ(occ.size());
    for (size_t i = 0; i < ord.size();) {
        size_t j = i;
        while (j < ord.size() && occ[ord[j]].key == occ[ord[i]].key) ++j;
        Run r{ord[i], -1, -1, -1, occ[ord[i]].cell < 0};
        size_t q = i;
        if (r.bface) ++q;
        for (; q < j; ++q) {
            const Occ& o = occ[ord[q]];
            if (o.cell < 0) fail(PRISM_INVALID_MESH, "duplicated boundary face element");
            if (r.owner < 0) { r.owner = o.cell; r.owner_occ = ord[q]; }
            else if (r.nbr < 0) r.nbr = o.cell;
            else fail(PRISM_INVALID_MESH, "a face shared by more than two cells");
        }
        if (r.bface && r.nbr >= 0) fail(PRISM_INVALID_MESH, "boundary face element between two cells");
        if (r.bface && r.owner < 0) fail(PRISM_INVALID_MESH, "dangling boundary face (not owned by any cell)");
        if (!r.bface && r.nbr < 0) fail(PRISM_INVALID_MESH, "cell face on no boundary patch and no neighbour");
        for (size_t q2 = i; q2 < j; ++q2) run_of_occ[ord[q2]] = (int64_t)runs.size();
        runs.push_back(r);
        i = j;
    }
    const int64_t nf = (int64_t)runs.size();

    // ---- groups -> patches (unv.cpp:298-371, 84-97)
    std::vector<char> in_group(ne, 0);
    std::map<std::string, std::vector<int64_t>> name_to_runs;
    for (int32_t g = 0; g < d->n_groups; ++g) {
        if (d->group_is_vertex && d->group_is_vertex[g]) continue;
        std::vector<int64_t> rs;
        for (int64_t q = d->group_offsets[g]; q < d->group_offsets[g + 1]; ++q) {
            int64_t e = d->group_elements[q];
            if (e < 0 || e >= ne || (d->elem_kind[e] != PRISM_ELEM_QUAD && d->elem_kind[e] != PRISM_ELEM_TRIANGLE))
                fail(PRISM_INVALID_MESH, "group contains non-face elements (cell zones)");
            in_group[e] = 1;
            rs.push_back(e);
        }
        name_to_runs.insert({d->group_names[g], std::move(rs)});
    }
    // element -> run for boundary elements
    std::vector<int64_t> run_of_elem(ne, -1);
    for (size_t o = 0; o < occ.size(); ++o)
        if (occ[o].cell < 0) run_of_elem[occ[o].elem] = run_of_occ[o];
    int64_t undefined = 0;
    for (int64_t e = 0; e < ne; ++e)
        if ((d->elem_kind[e] == PRISM_ELEM_QUAD || d->elem_kind[e] == PRISM_ELEM_TRIANGLE) && !in_group[e]) ++undefined;
    if (undefined)
        fail(PRISM_INVALID_MESH, std::to_string(undefined) + " boundary faces are not part of any boundary patch");

    auto hm = std::make_unique<HostMesh>();
    std::vector<int32_t> run_patch(runs.size(), -1);
    std::vector<std::vector<int64_t>> patch_runs(d->n_patches);
    for (int32_t p = 0; p < d->n_patches; ++p) {
        HostMesh::Patch pa;
        pa.name = d->patch_names[p];
        pa.empty = d->patch_is_empty[p] != 0;
        auto it = name_to_runs.find(pa.name);
        if (it != name_to_runs.end())
            for (auto e : it->second) {
                run_patch[run_of_elem[e]] = p;
                patch_runs[p].push_back(run_of_elem[e]);
            }
        hm->patches.push_back(std::move(pa));
    }

    // ---- PMesh permutation (pmesh.cpp:51-90)
    std::vector<int64_t> bruns, iruns;
    for (size_t r = 0; r < runs.size(); ++r) (runs[r].bface ? bruns : iruns).push_back((int64_t)r);
    for (auto r : bruns)
        if (run_patch[r] < 0) fail(PRISM_INVALID_MESH, "boundary face without a patch");
    // boundary faces in the order their owners were assigned, interior faces in creation
    // order; both orders are by distinct occurrence indices, so a placement by index sorts them
    {
        std::vector<int64_t> at(occ.size(), -1);
        for (auto r : bruns) at[runs[r].owner_occ] = r;
        bruns.clear();
        for (auto r : at)
            if (r >= 0) bruns.push_back(r);
        std::fill(at.begin(), at.end(), -1);
        for (auto r : iruns) at[runs[r].first] = r;
        iruns.clear();
        for (auto r : at)
            if (r >= 0) iruns.push_back(r);
    }
    int64_t nb = (int64_t)bruns.size(), nne = 0;
    for (auto r : bruns)
        if (!hm->patches[run_patch[r]].empty) ++nne;
    std::vector<int64_t> new_id(runs.size());
    int64_t pos_ne = 0, pos_e = nne, pos_i = nb;
    for (auto r : bruns) new_id[r] = hm->patches[run_patch[r]].empty ? pos_e++ : pos_ne++;
    for (auto r : iruns) new_id[r] = pos_i++;

    // ---- flatten
    const int64_t nc = (int64_t)cell_elem.size();
    hm->nc = nc;
    hm->nf = nf;
    hm->nb = nb;
    hm->nne = nne;
    hm->owner.assign(nf, -1);
    hm->nbr.assign(nf, -1);
    hm->patch.assign(nf, -1);
    hm->area.assign(nf, 0.0);
    for (int k = 0; k < 3; ++k) {
        hm->normal[k].assign(nf, 0.0);
        hm->fc[k].assign(nf, 0.0);
        hm->cc[k].assign(nc, 0.0);
    }
    hm->vol.assign(nc, 0.0);
    parallelFor((int64_t)runs.size(), [&](int64_t r0, int64_t r1) {
        V3 fv[8];
        int64_t t[8];
        for (int64_t r = r0; r < r1; ++r) {
            int64_t f = new_id[r];
            const Occ& o = occ[runs[r].first];
            int n = faceVerts(d, o.elem, o.local, t);
            for (int i = 0; i < n; ++i) fv[i] = X[t[i]];
            double a;
            V3 nrm, ctr;
            faceGeometry(fv, n, a, nrm, ctr);
            hm->area[f] = a;
            hm->normal[0][f] = nrm.x; hm->normal[1][f] = nrm.y; hm->normal[2][f] = nrm.z;
            hm->fc[0][f] = ctr.x; hm->fc[1][f] = ctr.y; hm->fc[2][f] = ctr.z;
            hm->owner[f] = runs[r].owner;
            hm->nbr[f] = runs[r].nbr;
            hm->patch[f] = run_patch[r];
        }
    });
    for (int32_t p = 0; p < d->n_patches; ++p)
        for (auto r : patch_runs[p]) hm->patches[p].faces.push_back((int32_t)new_id[r]);

    // cell faces in local order (occurrences of a cell are contiguous in reading order)
    hm->cf_off.assign(nc + 1, 0);
    for (size_t o = 0; o < occ.size(); ++o)
        if (occ[o].cell >= 0) hm->cf_off[occ[o].cell + 1]++;
    for (int64_t c = 0; c < nc; ++c) hm->cf_off[c + 1] += hm->cf_off[c];
    hm->cf_face.assign(hm->cf_off[nc], -1);
    {
        std::vector<int64_t> fill(hm->cf_off.begin(), hm->cf_off.end() - 1);
        for (size_t o = 0; o < occ.size(); ++o)
            if (occ[o].cell >= 0) hm->cf_face[fill[occ[o].cell]++] = (int32_t)new_id[run_of_occ[o]];
    }
    // Cell::Cell (mesh/cell.cpp:7-41)
    for (int64_t c = 0; c < nc; ++c) {
        V3 gc{0, 0, 0};
        int64_t b = hm->cf_off[c], e = hm->cf_off[c + 1];
        for (int64_t q = b; q < e; ++q) {
            int32_t f = hm->cf_face[q];
            gc = add(gc, V3{hm->fc[0][f], hm->fc[1][f], hm->fc[2][f]});
        }
        gc = divs(gc, (double)(e - b));
        double vol = 0.0;
        V3 ctr{0, 0, 0};
        for (int64_t q = b; q < e; ++q) {
            int32_t f = hm->cf_face[q];
            V3 fcv{hm->fc[0][f], hm->fc[1][f], hm->fc[2][f]};
            V3 nrm{hm->normal[0][f], hm->normal[1][f], hm->normal[2][f]};
            double pv = std::abs(dot(nrm, sub(fcv, gc)) * hm->area[f]) / 3;
            V3 pc = add(scale(fcv, 0.75), scale(gc, 0.25));
            vol += pv;
            ctr = add(ctr, scale(pc, pv));
        }
        ctr = divs(ctr, vol);
        hm->vol[c] = vol;
        hm->cc[0][c] = ctr.x; hm->cc[1][c] = ctr.y; hm->cc[2][c] = ctr.z;
    }
    // geometric weight per interior face (mesh/utilities.cpp:28-40, owner orientation)
    hm->gc.assign(nf - nb, 0.0);
    for (int64_t f = nb; f < nf; ++f) {
        int32_t o = hm->owner[f], n = hm->nbr[f];
        V3 fcv{hm->fc[0][f], hm->fc[1][f], hm->fc[2][f]};
        V3 co{hm->cc[0][o], hm->cc[1][o], hm->cc[2][o]};
        V3 cn{hm->cc[0][n], hm->cc[1][n], hm->cc[2][n]};
        V3 nrm{hm->normal[0][f], hm->normal[1][f], hm->normal[2][f]};
        V3 Sf = scale(nrm, hm->area[f]);
        Sf = V3{hm->area[f] * nrm.x, hm->area[f] * nrm.y, hm->area[f] * nrm.z};
        V3 ef = divs(Sf, std::sqrt(dot(Sf, Sf)));
        V3 dCf = sub(fcv, co), dfN = sub(cn, fcv);
        hm->gc[f - nb] = dot(dCf, ef) / (dot(dCf, ef) + dot(dfN, ef));
    }
    // vertices and cell vertex lists (kept for point data and export)
    hm->nv = d->n_nodes;
    for (int k = 0; k < 3; ++k) {
        hm->vx[k].resize(d->n_nodes);
        for (int64_t i = 0; i < d->n_nodes; ++i) hm->vx[k][i] = d->xyz[3 * i + k];
    }
    hm->cv_off.assign(nc + 1, 0);
    for (int64_t c = 0; c < nc; ++c) {
        int64_t e = cell_elem[c];
        hm->cv_off[c + 1] = hm->cv_off[c] + (d->elem_offsets[e + 1] - d->elem_offsets[e]);
    }
    hm->cv_node.resize(hm->cv_off[nc]);
    for (int64_t c = 0; c < nc; ++c) {
        int64_t e = cell_elem[c];
        const int64_t* en = d->elem_nodes + d->elem_offsets[e];
        for (int64_t q = hm->cv_off[c]; q < hm->cv_off[c + 1]; ++q) hm->cv_node[q] = (int32_t)en[q - hm->cv_off[c]];
    }
    hm->cell_orig.resize(nc);
    std::iota(hm->cell_orig.begin(), hm->cell_orig.end(), 0);
    return hm;
}

// The reference keeps a deque of not-visited nodes and searches it linearly
// (O(n^2)); a node leaves that deque exactly when it is enqueued, so an
// "enqueued" flag per cell and a cursor over the degree-sorted list give the
// same sequence in O(n log n). Both std::sort calls see the same sequences
// with the same comparator as the reference's, so ties resolve alike.
std::vector<int64_t> cuthillMckee(const HostMesh& h) {
    struct Node {
        int64_t id, degree;
    };
    const int64_t nc = h.nc;
    std::vector<Node> nodes(nc);
    for (int64_t c = 0; c < nc; ++c) {
        int64_t d = 0;
        for (int64_t q = h.cf_off[c]; q < h.cf_off[c + 1]; ++q)
            if (h.nbr[h.cf_face[q]] >= 0) ++d;
        nodes[c] = {c, d};
    }
    auto byDegree = [](const Node& a, const Node& b) { return a.degree < b.degree; };
    std::vector<Node> sorted = nodes;
    std::sort(sorted.begin(), sorted.end(), byDegree);
    std::vector<char> enqueued(nc, 0);
    std::vector<Node> queue(nc), nv;
    std::vector<int64_t> perm;
    perm.reserve(nc);
    int64_t head = 0, tail = 0;
    size_t cursor = 0;
    while ((int64_t)perm.size() < nc) {
        while (enqueued[sorted[cursor].id]) ++cursor;
        enqueued[sorted[cursor].id] = 1;
        queue[tail++] = sorted[cursor];
        while (head < tail) {
            const int64_t c = queue[head].id;
            nv.clear();
            for (int64_t q = h.cf_off[c]; q < h.cf_off[c + 1]; ++q) {
                const int32_t f = h.cf_face[q];
                if (h.nbr[f] < 0) continue;
                const int64_t n = h.owner[f] == c ? h.nbr[f] : h.owner[f];
                if (enqueued[n]) continue;
                enqueued[n] = 1;
                nv.push_back(nodes[n]);
            }
            std::sort(nv.begin(), nv.end(), byDegree);
            for (const Node& x : nv) queue[tail++] = x;
            perm.push_back(c);
            ++head;
        }
    }
    return perm;
}

void permuteCells(HostMesh& h, const std::vector<int64_t>& perm) {
    const int64_t nc = h.nc;
    if ((int64_t)perm.size() != nc) fail(PRISM_INTERNAL, "permutation size");
    std::vector<int32_t> o2n(nc);
    for (int64_t i = 0; i < nc; ++i) o2n[perm[i]] = (int32_t)i;
    auto gather = [&](auto& v) {
        auto old = v;
        for (int64_t i = 0; i < nc; ++i) v[i] = old[perm[i]];
    };
    for (int k = 0; k < 3; ++k) gather(h.cc[k]);
    gather(h.vol);
    gather(h.cell_orig);
    auto lists = [&](std::vector<int64_t>& off, auto& items) {
        std::vector<int64_t> noff(nc + 1, 0);
        auto nitems = items;
        for (int64_t i = 0; i < nc; ++i) {
            const int64_t b = off[perm[i]], e = off[perm[i] + 1];
            noff[i + 1] = noff[i] + (e - b);
            std::copy(items.begin() + b, items.begin() + e, nitems.begin() + noff[i]);
        }
        off.swap(noff);
        items.swap(nitems);
    };
    lists(h.cf_off, h.cf_face);
    lists(h.cv_off, h.cv_node);
    for (int64_t f = 0; f < h.nf; ++f) {
        h.owner[f] = o2n[h.owner[f]];
        if (h.nbr[f] >= 0) h.nbr[f] = o2n[h.nbr[f]];
    }
}

}  // namespace pb
