"""Readers for Prism's on-disk case format: I-DEAS UNV meshes and fields.json.

`read_unv` returns the mesh in the form the converter consumes (nodes, the
element list in file order, element groups); `read_case` parses fields.json and
the per-field <name>.json boundary files the way mesh/boundary.cpp:291-319 does
(patches sorted by name, a patch is "empty" when the first field -- by name --
declares it "empty", component fields U_x resolve to U). Together they replace
the reference's UnvToPMeshConverter inputs (mesh/unv.cpp:61-110, using the
unvpp reader) and MeshBoundary (mesh/boundary.cpp:291-319).
"""
import json
import os

import numpy as np

from . import _abi as A

# UNV FE descriptor ids -> element kinds (dataset 2412)
_BEAMS = {11, 21, 22, 23, 24}
_FE_KIND = {}
for _k in _BEAMS:
    _FE_KIND[_k] = A.ELEM_LINE
for _k in (41, 51, 61, 74, 81, 91):
    _FE_KIND[_k] = A.ELEM_TRIANGLE
for _k in (44, 54, 64, 71, 84, 94):
    _FE_KIND[_k] = A.ELEM_QUAD
_FE_KIND[111] = A.ELEM_TETRA
_FE_KIND[112] = A.ELEM_WEDGE
_FE_KIND[115] = A.ELEM_HEX
_NODES_USED = {A.ELEM_LINE: 2, A.ELEM_TRIANGLE: 3, A.ELEM_QUAD: 4, A.ELEM_TETRA: 4,
               A.ELEM_WEDGE: 6, A.ELEM_HEX: 8}


class UnvData:
    """Nodes, element list and groups of a UNV file (0-based indices)."""

    def __init__(self, xyz, elem_kind, elem_offsets, elem_nodes, groups):
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        self.elem_kind = np.ascontiguousarray(elem_kind, dtype=np.int32)
        self.elem_offsets = np.ascontiguousarray(elem_offsets, dtype=np.int64)
        self.elem_nodes = np.ascontiguousarray(elem_nodes, dtype=np.int64)
        # list of (name, is_vertex_group, element_or_node_indices)
        self.groups = groups

    @property
    def n_nodes(self):
        return self.xyz.shape[0]

    @property
    def n_elements(self):
        return self.elem_kind.shape[0]


def _f(tok):
    return float(tok.replace("D", "E").replace("d", "e"))


def read_unv(path):
    """Parse datasets 2411 (nodes), 2412 (elements) and 2467/2477/2452/2435 (groups)."""
    with open(path) as fh:
        lines = fh.read().split("\n")
    n = len(lines)
    node_label_to_idx, coords = {}, []
    elem_label_to_idx, kinds, offsets, conn = {}, [], [0], []
    raw_groups = []
    i = 0
    while i < n:
        if lines[i].strip() != "-1" or i + 1 >= n:
            i += 1
            continue
        ds = lines[i + 1].strip()
        j = i + 2
        if ds == "2411":
            while lines[j].strip() != "-1":
                label = int(lines[j].split()[0])
                x = [_f(t) for t in lines[j + 1].split()[:3]]
                node_label_to_idx[label] = len(coords)
                coords.append(x)
                j += 2
        elif ds == "2412":
            while lines[j].strip() != "-1":
                rec = lines[j].split()
                label, fe, nn = int(rec[0]), int(rec[1]), int(rec[5])
                j += 1
                if fe in _BEAMS:
                    j += 1
                nodes = []
                while len(nodes) < nn:
                    nodes.extend(int(t) for t in lines[j].split())
                    j += 1
                kind = _FE_KIND.get(fe)
                if kind is None:
                    raise A.PrismError(A.INVALID_MESH, f"unsupported UNV element descriptor {fe}")
                elem_label_to_idx[label] = len(kinds)
                kinds.append(kind)
                conn.append(nodes[: _NODES_USED[kind]])
                offsets.append(offsets[-1] + _NODES_USED[kind])
        elif ds in ("2467", "2477", "2452", "2435"):
            while lines[j].strip() != "-1":
                count = int(lines[j].split()[-1])
                name = lines[j + 1].strip()
                j += 2
                ents = []
                while len(ents) < count:
                    t = [int(v) for v in lines[j].split()]
                    for q in range(0, len(t), 4):
                        ents.append((t[q], t[q + 1]))
                    j += 1
                raw_groups.append((name, ents))
        while j < n and lines[j].strip() != "-1":
            j += 1
        i = j + 1
    xyz = np.array(coords, dtype=np.float64).reshape(-1, 3)
    flat = [node_label_to_idx[v] for c in conn for v in c]
    groups = []
    for name, ents in raw_groups:
        types = {t for t, _ in ents}
        if types == {7}:
            groups.append((name, True, np.array([node_label_to_idx[g] for _, g in ents], np.int64)))
        else:
            groups.append((name, False, np.array([elem_label_to_idx[g] for t, g in ents if t == 8],
                                                 np.int64)))
    return UnvData(xyz, kinds, offsets, flat, groups)


class FieldBC:
    """Boundary condition of one field on one patch."""

    def __init__(self, kind_str, value=None):
        self.kind_str = kind_str
        self.kind = A.BC_KIND_BY_NAME.get(kind_str, A.BC_UNKNOWN)
        if value is None:
            self.value_kind, self.value, self.vector = A.BCV_NIL, 0.0, (0.0, 0.0, 0.0)
        elif isinstance(value, (list, tuple)):
            if len(value) != 3:
                raise ValueError("expected array of size 3")
            self.value_kind, self.value, self.vector = A.BCV_VECTOR, 0.0, tuple(float(v) for v in value)
        else:
            self.value_kind, self.value, self.vector = A.BCV_SCALAR, float(value), (0.0, 0.0, 0.0)

    def to_c(self):
        b = A.BC()
        b.kind, b.value_kind, b.value = self.kind, self.value_kind, self.value
        b.vector[:] = self.vector
        return b


class Case:
    """Patches (sorted by name) and per-field boundary conditions of a case."""

    def __init__(self, patch_names, fields, field_info):
        self.patch_names = list(patch_names)
        self.fields = fields          # name -> [FieldBC per patch]
        self.field_info = field_info  # name -> {"type":..., "gradScheme":...}
        first = sorted(fields)[0] if fields else None
        self.patch_is_empty = [bool(first) and fields[first][p].kind_str == "empty"
                               for p in range(len(self.patch_names))]

    def bcs(self, field_name):
        """PrismBC array (one per patch) for a field; component names fall back to the vector."""
        name = field_name
        if name not in self.fields and len(name) > 2 and name[-2] == "_" and name[-1] in "xyz":
            name = name[:-2]
        if name not in self.fields:
            raise KeyError(f"no boundary conditions for field '{field_name}'")
        arr = (A.BC * len(self.patch_names))()
        for p, bc in enumerate(self.fields[name]):
            arr[p] = bc.to_c()
        return arr

    def grad_scheme(self, field_name):
        """fields.json gradScheme lookup (scalar.cpp:260-304): Green-Gauss or least squares."""
        name = field_name
        info = self.field_info.get(name)
        gs = (info or {}).get("gradScheme")
        if gs in ("green-gauss", "greenGauss"):
            return A.GRAD_GREEN_GAUSS
        return A.GRAD_LEAST_SQUARES

    @staticmethod
    def from_dict(patches, fields, field_info=None):
        """patches: iterable of names; fields: name -> {patch: (kind, value)}."""
        names = sorted(patches)
        fmap = {}
        for fname, per in fields.items():
            fmap[fname] = [FieldBC(*per[p]) if isinstance(per[p], tuple) else FieldBC(per[p])
                           for p in names]
        return Case(names, fmap, field_info or {f: {} for f in fields})


def read_case(fields_json_path):
    """MeshBoundary (mesh/boundary.cpp:291-319) for a fields.json file."""
    with open(fields_json_path) as fh:
        doc = json.load(fh)
    base = os.path.dirname(fields_json_path)
    docs = {}
    for f in doc.get("fields", []) if isinstance(doc.get("fields"), list) else []:
        if isinstance(f, dict) and "name" in f:
            path = os.path.join(base, f["name"] + ".json")
            if os.path.exists(path):
                with open(path) as fh:
                    docs[f["name"]] = json.load(fh)
    return case_from_docs(doc, docs)


def case_from_docs(doc, field_docs):
    """MeshBoundary from an already parsed fields.json document and the parsed
    <name>.json documents (name -> document)."""
    if "fields" not in doc or not isinstance(doc["fields"], list):
        raise ValueError("Couldn't find definition for fields in boundary conditions file")
    info = {}
    order = []
    for f in doc["fields"]:
        if "name" not in f or "type" not in f:
            raise ValueError("Field must contain name and type")
        info[f["name"]] = f
        order.append(f["name"])
    per_field = {}
    for name in order:
        if name not in field_docs:
            raise ValueError("Some field defined in `fields.json` file are not present in a "
                             "dedicated boundary conditions file")
        d = field_docs[name]
        if "patches" not in d or not isinstance(d["patches"], list):
            raise ValueError(f"file `{name}` doesn't contain a `patches` array")
        m = {}
        for p in d["patches"]:
            if "name" not in p or "type" not in p:
                raise ValueError(f"file `{name}` either doesn't contain `name` or `type` field")
            m.setdefault(p["name"], FieldBC(p["type"], p.get("value")))
        per_field[name] = m
    if not per_field:
        return Case([], {}, info)
    first_map = per_field[order[0]]
    for m in per_field.values():
        if len(m) != len(first_map):
            raise ValueError("boundary conditions files are not consistent")
    names = sorted(first_map)
    fields = {f: [per_field[f][p] for p in names] for f in per_field}
    return Case(names, fields, info)
