"""Synthetic meshes in the form a UNV file hands to the converter.

Each generator returns an `io.UnvData`: nodes, then the element list in the
order a Salome export writes it (boundary faces patch by patch, then the
volume cells), plus one element group per patch. Feeding this to
`prism_mesh_from_unv` goes through exactly the conversion a UNV file goes
through (mesh/unv.cpp:124-372), so face ordering, owners and neighbours are
those the reference would build from the same file.

Patches of a box: left (x=x0), right (x=x1), bottom (y=y0), top (y=y1),
back (z=z0), front (z=z1).
"""
import numpy as np

from . import _abi as A
from .io import UnvData

PATCHES = ("left", "right", "bottom", "top", "back", "front")


def _assemble(xyz, faces_by_patch, cells, cell_kind):
    kinds, counts, conn, groups = [], [], [], []
    start = 0
    for name in PATCHES:
        fl = faces_by_patch[name]
        nverts = fl.shape[1]
        kinds.append(np.full(fl.shape[0], A.ELEM_QUAD if nverts == 4 else A.ELEM_TRIANGLE, dtype=np.int32))
        counts.append(np.full(fl.shape[0], nverts, dtype=np.int64))
        conn.append(fl.reshape(-1))
        groups.append((name, False, np.arange(start, start + fl.shape[0], dtype=np.int64)))
        start += fl.shape[0]
    kinds.append(np.full(cells.shape[0], cell_kind, dtype=np.int32))
    counts.append(np.full(cells.shape[0], cells.shape[1], dtype=np.int64))
    conn.append(cells.reshape(-1))
    counts = np.concatenate(counts)
    offs = np.zeros(len(counts) + 1, dtype=np.int64)
    np.cumsum(counts, out=offs[1:])
    return UnvData(xyz, np.concatenate(kinds), offs, np.concatenate(conn).astype(np.int64), groups)


def _grid_nodes(nx, ny, nz, lengths, origin, jitter, seed):
    lx, ly, lz = lengths
    x0, y0, z0 = origin
    xs = x0 + lx * np.arange(nx + 1) / nx
    ys = y0 + ly * np.arange(ny + 1) / ny
    zs = z0 + lz * np.arange(nz + 1) / nz
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    xyz = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    if jitter:
        rng = np.random.default_rng(seed)
        h = np.array([lx / nx, ly / ny, lz / nz])
        d = rng.uniform(-jitter, jitter, size=xyz.shape) * h
        k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
        interior = ((i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)).ravel()
        xyz[interior] += d[interior]
    return xyz


def box_hex(nx, ny, nz, lengths=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0), jitter=0.0, seed=0):
    """Structured nx*ny*nz hex box; cells in x-fastest order. `jitter` moves each
    interior node by U(-jitter*h, jitter*h) per coordinate (seeded)."""
    xyz = _grid_nodes(nx, ny, nz, lengths, origin, jitter, seed)

    def nid(i, j, k):
        return (k * (ny + 1) + j) * (nx + 1) + i

    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    c = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                  nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1),
                  nid(i, j + 1, k + 1)], axis=1).astype(np.int64)
    # boundary quads with the owner cell's local face vertex order (outward normals)
    def sel(mask, cols):
        return c[mask][:, cols]

    faces = {
        "left": sel(i == 0, [0, 4, 7, 3]),
        "right": sel(i == nx - 1, [1, 2, 6, 5]),
        "bottom": sel(j == 0, [0, 1, 5, 4]),
        "top": sel(j == ny - 1, [2, 3, 7, 6]),
        "back": sel(k == 0, [0, 3, 2, 1]),
        "front": sel(k == nz - 1, [4, 5, 6, 7]),
    }
    return _assemble(xyz, faces, c, A.ELEM_HEX)


# Kuhn (Freudenthal) split of the unit cube into 6 tets along the 0-6 diagonal,
# corners numbered as the hex above.
_KUHN = [(0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)]


def box_tet(nx, ny, nz, lengths=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0), jitter=0.0, seed=0):
    """nx*ny*nz cubes, each split into 6 positively oriented tets (Kuhn split)."""
    h = box_hex(nx, ny, nz, lengths, origin, jitter, seed)
    xyz = h.xyz
    nb = int(np.sum(h.elem_kind != A.ELEM_HEX))
    hexes = h.elem_nodes[h.elem_offsets[nb]:].reshape(-1, 8)
    tets = []
    for t in _KUHN:
        tets.append(hexes[:, list(t)])
    tets = np.stack(tets, axis=1).reshape(-1, 4)
    # orient positively: det(c1-c0, c2-c0, c3-c0) > 0 gives outward face normals
    p = xyz[tets]
    det = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])
    neg = det < 0
    tets[neg] = tets[neg][:, [0, 2, 1, 3]]
    # boundary triangles: split each boundary quad the same way the cube split does
    tri = {}
    for name in PATCHES:
        g = [gg for gg in h.groups if gg[0] == name][0][2]
        quads = h.elem_nodes.reshape(-1)[np.concatenate(
            [np.arange(h.elem_offsets[e], h.elem_offsets[e + 1]) for e in g])].reshape(-1, 4)
        tri[name] = quads
    # Each cube face holds one end of the cube diagonal the tets share, so exactly
    # one of the two triangulations of a boundary quad matches tet faces: keep it.
    nn = np.int64(xyz.shape[0])

    def key(tri_nodes):
        s = np.sort(tri_nodes, axis=1).astype(np.int64)
        return (s[:, 0] * nn + s[:, 1]) * nn + s[:, 2]

    tet_keys = np.unique(np.concatenate([key(np.delete(tets, q, axis=1)) for q in range(4)]))
    faces = {}
    for name, quads in tri.items():
        a, b, cc, d = quads[:, 0], quads[:, 1], quads[:, 2], quads[:, 3]
        first = np.isin(key(np.stack([a, b, cc], 1)), tet_keys)
        t1 = np.where(first[:, None], np.stack([a, b, cc], 1), np.stack([a, b, d], 1))
        t2 = np.where(first[:, None], np.stack([a, cc, d], 1), np.stack([b, cc, d], 1))
        faces[name] = np.stack([t1, t2], axis=1).reshape(-1, 3).astype(np.int64)
    return _assemble(xyz, faces, tets, A.ELEM_TETRA)


def shuffle_cells(unv, seed=0):
    """The same mesh with its volume cells listed in a random order (as an
    unstructured mesher may write them): cell ids lose their locality, the
    boundary-face elements and groups are unchanged."""
    kinds = unv.elem_kind
    is_cell = (kinds == A.ELEM_HEX) | (kinds == A.ELEM_TETRA) | (kinds == A.ELEM_WEDGE)
    first = int(np.argmax(is_cell))
    if not np.all(is_cell[first:]):
        raise ValueError("cells must follow the boundary elements")
    order = np.concatenate([np.arange(first), first + np.random.default_rng(seed).permutation(len(kinds) - first)])
    counts = np.diff(unv.elem_offsets)[order]
    offs = np.zeros(len(order) + 1, dtype=np.int64)
    np.cumsum(counts, out=offs[1:])
    src = np.repeat(unv.elem_offsets[order] - offs[:-1], counts) + np.arange(offs[-1])
    return UnvData(unv.xyz, kinds[order], offs, unv.elem_nodes[src], unv.groups)
