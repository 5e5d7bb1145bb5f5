// unvpp-API shim (test infrastructure): the I-DEAS UNV reader the reference's
// converter calls (src/prism/mesh/unv.cpp:3-5, 63, 127-147, 305-353). The
// reference pins its `external/unvpp` submodule, which is empty in this
// checkout, so this header restates the reader's observable result from the
// call sites: vertices in file order (dataset 2411), every element of dataset
// 2412 in file order with 0-based vertex indices, and the groups of datasets
// 2467/2477/2452/2435 with 0-based element (or vertex) indices. It reads the
// same text the Python reader prism_b200/io.py reads, and also a binary dump
// of that result (extension .unvbin, written by oracle/ref_lib.py), so that
// large synthetic meshes need not go through text.
#pragma once

#include <array>
#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <map>
#include <optional>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace unvpp {

enum class ElementType { Line, Triangle, Quad, Tetra, Wedge, Hex };
enum class GroupType { Vertex, Element, Mixed };

class Element {
  public:
    Element(ElementType t, std::vector<size_t> v) : type_(t), v_(std::move(v)) {}
    auto type() const -> ElementType { return type_; }
    auto vertices_ids() const -> const std::vector<size_t>& { return v_; }

  private:
    ElementType type_;
    std::vector<size_t> v_;
};

class Group {
  public:
    Group(std::string name, GroupType t, std::vector<size_t> ids, std::set<ElementType> types)
        : name_(std::move(name)), type_(t), ids_(std::move(ids)), types_(std::move(types)) {}
    auto name() const -> const std::string& { return name_; }
    auto type() const -> GroupType { return type_; }
    auto elements_ids() const -> const std::vector<size_t>& { return ids_; }
    auto vertices_ids() const -> const std::vector<size_t>& { return ids_; }
    auto unique_element_types() const -> const std::set<ElementType>& { return types_; }

  private:
    std::string name_;
    GroupType type_;
    std::vector<size_t> ids_;
    std::set<ElementType> types_;
};

class Mesh {
  public:
    Mesh(std::vector<std::array<double, 3>> v,
         std::optional<std::vector<Element>> e,
         std::optional<std::vector<Group>> g)
        : v_(std::move(v)), e_(std::move(e)), g_(std::move(g)) {}
    auto vertices() const -> const std::vector<std::array<double, 3>>& { return v_; }
    auto elements() const -> const std::optional<std::vector<Element>>& { return e_; }
    auto groups() const -> const std::optional<std::vector<Group>>& { return g_; }

  private:
    std::vector<std::array<double, 3>> v_;
    std::optional<std::vector<Element>> e_;
    std::optional<std::vector<Group>> g_;
};

namespace detail {
inline auto nodesUsed(ElementType t) -> size_t {
    switch (t) {
        case ElementType::Line: return 2;
        case ElementType::Triangle: return 3;
        case ElementType::Quad: return 4;
        case ElementType::Tetra: return 4;
        case ElementType::Wedge: return 6;
        case ElementType::Hex: return 8;
    }
    return 0;
}

// FE descriptor ids of dataset 2412
inline auto kindOf(int fe) -> std::optional<ElementType> {
    switch (fe) {
        case 11: case 21: case 22: case 23: case 24: return ElementType::Line;
        case 41: case 51: case 61: case 74: case 81: case 91: return ElementType::Triangle;
        case 44: case 54: case 64: case 71: case 84: case 94: return ElementType::Quad;
        case 111: return ElementType::Tetra;
        case 112: return ElementType::Wedge;
        case 115: return ElementType::Hex;
        default: return std::nullopt;
    }
}

inline auto toDouble(std::string t) -> double {
    for (auto& ch : t)
        if (ch == 'D' || ch == 'd') ch = 'E';
    return std::stod(t);
}

inline auto trim(const std::string& s) -> std::string {
    auto b = s.find_first_not_of(" \t\r");
    if (b == std::string::npos) return "";
    auto e = s.find_last_not_of(" \t\r");
    return s.substr(b, e - b + 1);
}

inline auto finishGroups(const std::vector<std::pair<std::string, std::vector<std::pair<long, long>>>>& raw,
                         const std::map<long, size_t>& node_idx,
                         const std::map<long, size_t>& elem_idx,
                         const std::vector<Element>& elems) -> std::vector<Group> {
    std::vector<Group> groups;
    for (const auto& [name, ents] : raw) {
        bool all_nodes = !ents.empty();
        for (const auto& [t, _] : ents) all_nodes = all_nodes && (t == 7);
        std::vector<size_t> ids;
        std::set<ElementType> types;
        if (all_nodes) {
            for (const auto& [_, tag] : ents) ids.push_back(node_idx.at(tag));
            groups.emplace_back(name, GroupType::Vertex, std::move(ids), std::move(types));
        } else {
            for (const auto& [t, tag] : ents)
                if (t == 8) {
                    auto k = elem_idx.at(tag);
                    ids.push_back(k);
                    types.insert(elems[k].type());
                }
            groups.emplace_back(name, GroupType::Element, std::move(ids), std::move(types));
        }
    }
    return groups;
}

inline auto readText(const std::filesystem::path& path) -> Mesh {
    std::ifstream fh(path);
    if (!fh) throw std::runtime_error("unvpp::read(): cannot open " + path.string());
    std::vector<std::string> lines;
    for (std::string l; std::getline(fh, l);) lines.push_back(l);
    const size_t n = lines.size();
    std::vector<std::array<double, 3>> coords;
    std::map<long, size_t> node_idx, elem_idx;
    std::vector<Element> elems;
    std::vector<std::pair<std::string, std::vector<std::pair<long, long>>>> raw;
    size_t i = 0;
    while (i < n) {
        if (trim(lines[i]) != "-1" || i + 1 >= n) {
            ++i;
            continue;
        }
        const std::string ds = trim(lines[i + 1]);
        size_t j = i + 2;
        if (ds == "2411") {
            while (j < n && trim(lines[j]) != "-1") {
                std::istringstream a(lines[j]), b(lines[j + 1]);
                long label;
                a >> label;
                std::string x, y, z;
                b >> x >> y >> z;
                node_idx[label] = coords.size();
                coords.push_back({toDouble(x), toDouble(y), toDouble(z)});
                j += 2;
            }
        } else if (ds == "2412") {
            while (j < n && trim(lines[j]) != "-1") {
                std::istringstream rec(lines[j]);
                long label, fe, pp, mp, color, nn;
                rec >> label >> fe >> pp >> mp >> color >> nn;
                ++j;
                if (fe == 11 || fe == 21 || fe == 22 || fe == 23 || fe == 24) ++j;
                std::vector<long> nodes;
                while (static_cast<long>(nodes.size()) < nn) {
                    std::istringstream t(lines[j]);
                    for (long v; t >> v;) nodes.push_back(v);
                    ++j;
                }
                auto kind = kindOf(static_cast<int>(fe));
                if (!kind) throw std::runtime_error("unvpp::read(): unsupported element descriptor");
                std::vector<size_t> ids;
                for (size_t q = 0; q < nodesUsed(*kind); ++q) ids.push_back(node_idx.at(nodes[q]));
                elem_idx[label] = elems.size();
                elems.emplace_back(*kind, std::move(ids));
            }
        } else if (ds == "2467" || ds == "2477" || ds == "2452" || ds == "2435") {
            while (j < n && trim(lines[j]) != "-1") {
                std::istringstream hdr(lines[j]);
                std::vector<long> h;
                for (long v; hdr >> v;) h.push_back(v);
                long count = h.back();
                std::string name = trim(lines[j + 1]);
                j += 2;
                std::vector<std::pair<long, long>> ents;
                while (static_cast<long>(ents.size()) < count) {
                    std::istringstream t(lines[j]);
                    std::vector<long> v;
                    for (long q; t >> q;) v.push_back(q);
                    for (size_t q = 0; q + 1 < v.size(); q += 4) ents.emplace_back(v[q], v[q + 1]);
                    ++j;
                }
                raw.emplace_back(name, std::move(ents));
            }
        }
        while (j < n && trim(lines[j]) != "-1") ++j;
        i = j + 1;
    }
    auto groups = finishGroups(raw, node_idx, elem_idx, elems);
    return Mesh(std::move(coords), std::move(elems), std::move(groups));
}

// Binary dump: magic "UNVB", int64 counts, then the arrays (little endian):
//   n_nodes, xyz[3 n_nodes] f64; n_elem, kind[n_elem] i8 (ElementType order),
//   offsets[n_elem + 1] i64, nodes[offsets[n_elem]] i64; n_groups, then per group
//   name_len i64, name bytes, is_vertex i8, count i64, ids[count] i64.
inline auto readBinary(const std::filesystem::path& path) -> Mesh {
    std::ifstream fh(path, std::ios::binary);
    if (!fh) throw std::runtime_error("unvpp::read(): cannot open " + path.string());
    char magic[4];
    fh.read(magic, 4);
    if (std::string(magic, 4) != "UNVB") throw std::runtime_error("unvpp::read(): bad binary header");
    auto i64 = [&]() {
        int64_t v;
        fh.read(reinterpret_cast<char*>(&v), 8);
        return v;
    };
    int64_t nn = i64();
    std::vector<std::array<double, 3>> coords(static_cast<size_t>(nn));
    fh.read(reinterpret_cast<char*>(coords.data()), static_cast<std::streamsize>(24 * nn));
    int64_t ne = i64();
    std::vector<int8_t> kind(static_cast<size_t>(ne));
    fh.read(reinterpret_cast<char*>(kind.data()), static_cast<std::streamsize>(ne));
    std::vector<int64_t> off(static_cast<size_t>(ne + 1));
    fh.read(reinterpret_cast<char*>(off.data()), static_cast<std::streamsize>(8 * (ne + 1)));
    std::vector<int64_t> nodes(static_cast<size_t>(off[ne]));
    fh.read(reinterpret_cast<char*>(nodes.data()), static_cast<std::streamsize>(8 * off[ne]));
    std::vector<Element> elems;
    elems.reserve(static_cast<size_t>(ne));
    for (int64_t e = 0; e < ne; ++e)
        elems.emplace_back(static_cast<ElementType>(kind[e]),
                           std::vector<size_t>(nodes.begin() + off[e], nodes.begin() + off[e + 1]));
    int64_t ng = i64();
    std::vector<Group> groups;
    for (int64_t g = 0; g < ng; ++g) {
        int64_t len = i64();
        std::string name(static_cast<size_t>(len), '\0');
        fh.read(name.data(), len);
        int8_t is_vertex;
        fh.read(reinterpret_cast<char*>(&is_vertex), 1);
        int64_t cnt = i64();
        std::vector<int64_t> ids(static_cast<size_t>(cnt));
        fh.read(reinterpret_cast<char*>(ids.data()), static_cast<std::streamsize>(8 * cnt));
        std::vector<size_t> sids(ids.begin(), ids.end());
        std::set<ElementType> types;
        if (!is_vertex)
            for (auto k : sids) types.insert(elems[k].type());
        groups.emplace_back(name, is_vertex ? GroupType::Vertex : GroupType::Element, std::move(sids),
                            std::move(types));
    }
    if (!fh) throw std::runtime_error("unvpp::read(): truncated binary mesh " + path.string());
    return Mesh(std::move(coords), std::move(elems), std::move(groups));
}
} // namespace detail

inline auto read(const std::filesystem::path& path) -> Mesh {
    if (path.extension() == ".unvbin") return detail::readBinary(path);
    return detail::readText(path);
}

} // namespace unvpp
