// mesh_build.h -- flattened PMesh on the host (input of the device upload).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "common.h"

namespace pb {

struct HostMesh {
    int64_t nc = 0, nf = 0, nb = 0, nne = 0;
    std::vector<int32_t> owner, nbr, patch;  // per face; nbr -1 / patch -1 where absent
    std::vector<double> area, normal[3], fc[3];
    std::vector<double> cc[3], vol;
    std::vector<double> gc;                  // per interior face (index f - nb)
    std::vector<int64_t> cf_off;             // cell -> faces (reference local order)
    std::vector<int32_t> cf_face;
    // PMesh::vertices() (every UNV node) and Cell::verticesIds() (element node order)
    int64_t nv = 0;
    std::vector<double> vx[3];
    std::vector<int64_t> cv_off;
    std::vector<int32_t> cv_node;
    std::vector<int64_t> cell_orig;  // id of each cell before any reordering
    struct Patch {
        std::string name;
        bool empty = false;
        std::vector<int32_t> faces;
    };
    std::vector<Patch> patches;
};

std::unique_ptr<HostMesh> buildHostMesh(const PrismUnvMesh* d);

// CuthillMckee::permute (mesh/reorder.cpp:40-87): new -> old cell ids
std::vector<int64_t> cuthillMckee(const HostMesh& h);
// CuthillMckee::reorder (reorder.cpp:89-129) on the host arrays: cells (centres,
// volumes, face and vertex lists) move to their new ids, faces keep theirs with
// owner and neighbour renamed
void permuteCells(HostMesh& h, const std::vector<int64_t>& new_to_old);

}  // namespace pb
