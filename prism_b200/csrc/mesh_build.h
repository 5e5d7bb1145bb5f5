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
    struct Patch {
        std::string name;
        bool empty = false;
        std::vector<int32_t> faces;
    };
    std::vector<Patch> patches;
};

std::unique_ptr<HostMesh> buildHostMesh(const PrismUnvMesh* d);

}  // namespace pb
