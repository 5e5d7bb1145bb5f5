// mesh_build_check.cpp -- the host mesh builder (prism_b200/csrc/mesh_build.cpp) behind
// a small C interface, so that tests can compile it with AddressSanitizer and
// UndefinedBehaviorSanitizer and drive it on the CPU: UNV descriptor -> HostMesh
// (face matching, ordering, geometry), Cuthill-McKee renumbering, and the arrays the
// device upload reads. Built by tests/test_host_sanitizers.py; not part of the library.
#include <algorithm>
#include <cstring>
#include <exception>
#include <string>

#include "../../prism_b200/csrc/mesh_build.h"

namespace {
std::string g_error;
}

extern "C" {

const char* mb_last_error(void) { return g_error.c_str(); }

// Same contract as prism_mesh_from_unv for the host part: 0 and *out = the mesh, or
// non-zero with the message in mb_last_error().
int mb_mesh_from_unv(const PrismUnvMesh* d, void** out) {
    try {
        *out = pb::buildHostMesh(d).release();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

int mb_mesh_info(void* hm, PrismMeshInfo* info) {
    const pb::HostMesh& h = *static_cast<pb::HostMesh*>(hm);
    std::memset(info, 0, sizeof(*info));
    info->n_cells = h.nc;
    info->n_faces = h.nf;
    info->n_boundary_faces = h.nb;
    info->n_nonempty_boundary_faces = h.nne;
    info->n_patches = (int32_t)h.patches.size();
    info->n_vertices = h.nv;
    info->n_cell_vertices = (int64_t)h.cv_node.size();
    return 0;
}

// CuthillMckee::permute + reorder on the host arrays (reverse: the reversed order)
int mb_reorder(void* hm, int reverse) {
    try {
        pb::HostMesh& h = *static_cast<pb::HostMesh*>(hm);
        std::vector<int64_t> perm = pb::cuthillMckee(h);
        if (reverse) std::reverse(perm.begin(), perm.end());
        pb::permuteCells(h, perm);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// owner, neighbour (-1 on boundary faces) and area per face; volume and centre per cell;
// cell -> face lists (offsets nc + 1, faces; cf_face null: offsets only)
void mb_export(void* hm, int32_t* owner, int32_t* nbr, double* area, double* vol, double* cc, int64_t* cf_off,
               int32_t* cf_face) {
    const pb::HostMesh& h = *static_cast<pb::HostMesh*>(hm);
    std::copy(h.owner.begin(), h.owner.end(), owner);
    std::copy(h.nbr.begin(), h.nbr.end(), nbr);
    std::copy(h.area.begin(), h.area.end(), area);
    std::copy(h.vol.begin(), h.vol.end(), vol);
    for (int k = 0; k < 3; ++k) std::copy(h.cc[k].begin(), h.cc[k].end(), cc + k * h.nc);
    std::copy(h.cf_off.begin(), h.cf_off.end(), cf_off);
    if (cf_face) std::copy(h.cf_face.begin(), h.cf_face.end(), cf_face);
}

void mb_destroy(void* hm) { delete static_cast<pb::HostMesh*>(hm); }

}  // extern "C"
