// Drop-in use of the C++ mirror API (include/prism_b200.hpp), written the way the
// reference's own Poisson test is (tests/test_poisson.cpp:24-50): Corrected(c = I, P)
// + ConstantScalar(S) on an n x n x 1 hex box, 5 non-orthogonal correctors of
// solve(15 steps). Prints the solution, one value per line.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "prism_b200.hpp"

using namespace prism_b200;

int main(int argc, char** argv) {
    const int n = argc > 1 ? std::atoi(argv[1]) : 16;
    // UNV-form box: nodes, boundary quads grouped by patch, then hexes (x fastest)
    mesh::UnvMesh unv;
    auto nid = [&](int i, int j, int k) { return (int64_t)((k * (n + 1) + j) * (n + 1) + i); };
    for (int k = 0; k <= 1; ++k)
        for (int j = 0; j <= n; ++j)
            for (int i = 0; i <= n; ++i) {
                unv.xyz.push_back((double)i / n);
                unv.xyz.push_back(-0.5 + (double)j / n);
                unv.xyz.push_back(0.1 * k);
            }
    auto hexNodes = [&](int i, int j) {
        return std::vector<int64_t>{nid(i, j, 0), nid(i + 1, j, 0), nid(i + 1, j + 1, 0), nid(i, j + 1, 0),
                                    nid(i, j, 1), nid(i + 1, j, 1), nid(i + 1, j + 1, 1), nid(i, j + 1, 1)};
    };
    auto addFace = [&](const std::vector<int64_t>& c, std::initializer_list<int> loc, mesh::UnvMesh::Group& g) {
        g.elements.push_back((int64_t)unv.elem_kind.size());
        unv.elem_kind.push_back(PRISM_ELEM_QUAD);
        for (int l : loc) unv.elem_nodes.push_back(c[l]);
        unv.elem_offsets.push_back((int64_t)unv.elem_nodes.size());
    };
    mesh::UnvMesh::Group left{"left"}, right{"right"}, bottom{"bottom"}, top{"top"}, back{"back"}, front{"front"};
    for (int j = 0; j < n; ++j) addFace(hexNodes(0, j), {0, 4, 7, 3}, left);
    for (int j = 0; j < n; ++j) addFace(hexNodes(n - 1, j), {1, 2, 6, 5}, right);
    for (int i = 0; i < n; ++i) addFace(hexNodes(i, 0), {0, 1, 5, 4}, bottom);
    for (int i = 0; i < n; ++i) addFace(hexNodes(i, n - 1), {2, 3, 7, 6}, top);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) addFace(hexNodes(i, j), {0, 3, 2, 1}, back);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) addFace(hexNodes(i, j), {4, 5, 6, 7}, front);
    unv.groups = {left, right, bottom, top, back, front};
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            unv.elem_kind.push_back(PRISM_ELEM_HEX);
            for (auto v : hexNodes(i, j)) unv.elem_nodes.push_back(v);
            unv.elem_offsets.push_back((int64_t)unv.elem_nodes.size());
        }
    // patches sorted by name as MeshBoundary builds them; front/back empty
    std::vector<mesh::PatchInfo> patches{{"back", true}, {"bottom"}, {"front", true}, {"left"}, {"right"}, {"top"}};
    auto pm = std::make_shared<mesh::PMesh>(unv, patches);

    std::vector<field::BC> pbc(patches.size());
    for (size_t p = 0; p < patches.size(); ++p)
        pbc[p] = patches[p].empty ? field::BC{PRISM_BC_EMPTY, PRISM_BCV_NIL, 0.0, {0, 0, 0}}
                                  : field::BC{PRISM_BC_FIXED, PRISM_BCV_SCALAR, 0.0, {0, 0, 0}};
    std::vector<field::BC> none(patches.size(), field::BC{PRISM_BC_UNKNOWN, PRISM_BCV_NIL, 0.0, {0, 0, 0}});
    // source at the cell centres (uniform box: centres are the cell midpoints)
    std::vector<double> src(pm->cellCount());
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            double x = (i + 0.5) / n, y = -0.5 + (j + 0.5) / n;
            src[j * n + i] = 2 * M_PI * M_PI * std::sin(M_PI * x) * std::cos(M_PI * y);
        }
    auto P = std::make_shared<field::Scalar>("P", pm, 0.0, pbc, PRISM_GRAD_GREEN_GAUSS);
    auto S = std::make_shared<field::Scalar>("S", pm, src, none);
    auto c = std::make_shared<field::Tensor>("c", pm);
    eqn::Transport eq(scheme::diffusion::Corrected(c, P), scheme::source::ConstantScalar<>(S));
    solver::BiCGSTAB solver;
    for (int i = 0; i < 5; ++i) solver.solve(eq, 15, 1e-20);
    for (double v : P->values()) std::printf("%.17g\n", v);
    // diagnostics of a uniform flow (1, 0, 0) through the same mesh, on stderr:
    // Courant number 0.5 * dt * 2u/h = u dt n everywhere, zero divergence, and the
    // solution interpolated to the vertices
    std::vector<field::BC> ubc(patches.size());
    for (size_t p = 0; p < patches.size(); ++p)
        ubc[p] = patches[p].empty ? field::BC{PRISM_BC_EMPTY, PRISM_BCV_NIL, 0.0, {0, 0, 0}}
                                  : field::BC{PRISM_BC_FIXED, PRISM_BCV_VECTOR, 0.0, {1, 0, 0}};
    const double u0[3] = {1.0, 0.0, 0.0};
    field::Vector U("U", pm, u0, ubc);
    auto co = monitor::courantNumber(U, 0.01).values();
    auto dv = ops::div(U).values();
    auto pts = P->toPoints();
    std::fprintf(stderr, "Co[0] %.6g div[0] %.3g points %zu\n", co[0], dv[0], pts.size());
    return 0;
}
