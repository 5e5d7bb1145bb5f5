"""The reference's own code, compiled here (oracle/_ref/libprism_ref.so) -- TEST
INFRASTRUCTURE: only tests/ and bench.py's reference arm load it, as the
checker or as the timed CPU reference, never as product code.

`available()` says whether the library was built (it is built by
oracle/ref_build.py when the reference tree is present). Meshes reach the
reference's own UnvToPMeshConverter through a binary dump of the parsed UNV
(`.unvbin`, read by the project's unvpp shim) plus fields.json and the per-field
boundary files, written to a temporary directory.
"""
import ctypes
import json
import os
import tempfile

import numpy as np

from prism_b200 import _abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libprism_ref.so")

CONV = {"Upwind": 0, "CentralDifference": 1, "LinearUpwind": 2, "SecondOrderUpwind": 2, "QUICK": 3,
        "FROMM": 4, "MINMOD": 5, "MUSCL": 6, "SMART": 7}

_lib = None
_pd = ctypes.POINTER(ctypes.c_double)
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pi = ctypes.POINTER(ctypes.c_int)


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{LIB} is not built (python -m oracle.ref_build)")
        L = ctypes.CDLL(LIB)
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_mesh_load.restype = ctypes.c_void_p
        L.ref_mesh_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.ref_mesh_free.argtypes = [ctypes.c_void_p]
        L.ref_mesh_sizes.argtypes = [ctypes.c_void_p, _pi64]
        L.ref_mesh_faces.argtypes = [ctypes.c_void_p, _pi64, _pi64, _pi64, _pd, _pd, _pd]
        L.ref_mesh_cells.argtypes = [ctypes.c_void_p, _pd, _pd]
        L.ref_poisson.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _pd]
        L.ref_advection_1d.argtypes = [ctypes.c_void_p, _pd]
        L.ref_transport.restype = ctypes.c_int64
        L.ref_transport.argtypes = [ctypes.c_void_p, ctypes.c_int, _pd, ctypes.c_double, ctypes.c_int, _pd, _pd,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, _pd,
                                    ctypes.c_int64, _pi64, _pi64, _pd, _pd]
        L.ref_simple.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 _pd, _pd, _pd, _pd, _pd, _pi, _pi, _pd]
        _lib = L
    return _lib


def _p(a, t=_pd):
    return None if a is None else a.ctypes.data_as(t)


def _check(rc):
    if rc != 0:
        raise RuntimeError("reference raised: " + lib().ref_last_error().decode())


def _shim_kind(kinds):
    """prism_b200 element kinds -> the shim's unvpp::ElementType order (Line, Triangle, Quad,
    Tetra, Wedge, Hex)."""
    table = np.full(max(A.ELEM_LINE, A.ELEM_TRIANGLE, A.ELEM_QUAD, A.ELEM_TETRA, A.ELEM_WEDGE, A.ELEM_HEX) + 1,
                    -1, np.int8)
    for k, v in ((A.ELEM_LINE, 0), (A.ELEM_TRIANGLE, 1), (A.ELEM_QUAD, 2), (A.ELEM_TETRA, 3), (A.ELEM_WEDGE, 4),
                 (A.ELEM_HEX, 5)):
        table[k] = v
    return table[np.asarray(kinds, np.int64)]


def write_unvbin(unv, path):
    """Binary dump of a parsed UNV mesh (prism_b200.io.UnvData) in the layout the shim reads."""
    with open(path, "wb") as fh:
        fh.write(b"UNVB")
        fh.write(np.int64(unv.n_nodes).tobytes())
        fh.write(np.ascontiguousarray(unv.xyz, np.float64).tobytes())
        fh.write(np.int64(unv.n_elements).tobytes())
        fh.write(_shim_kind(unv.elem_kind).tobytes())
        fh.write(np.ascontiguousarray(unv.elem_offsets, np.int64).tobytes())
        fh.write(np.ascontiguousarray(unv.elem_nodes, np.int64).tobytes())
        fh.write(np.int64(len(unv.groups)).tobytes())
        for name, is_vertex, ids in unv.groups:
            b = name.encode()
            fh.write(np.int64(len(b)).tobytes())
            fh.write(b)
            fh.write(np.int8(1 if is_vertex else 0).tobytes())
            ids = np.ascontiguousarray(ids, np.int64)
            fh.write(np.int64(len(ids)).tobytes())
            fh.write(ids.tobytes())


def case_docs(case):
    """fields.json and per-field boundary documents of a prism_b200.io.Case."""
    fields = {"fields": []}
    docs = {}
    for name, bcs in case.fields.items():
        entry = {"name": name, "type": "scalar"}
        info = case.field_info.get(name) or {}
        for k, v in info.items():
            entry[k] = v
        fields["fields"].append(entry)
        patches = []
        for pname, bc in zip(case.patch_names, bcs):
            d = {"name": pname, "type": bc.kind_str}
            if bc.value_kind == A.BCV_SCALAR:
                d["value"] = bc.value
            elif bc.value_kind == A.BCV_VECTOR:
                d["value"] = list(bc.vector)
            patches.append(d)
        docs[name] = {"patches": patches}
    return fields, docs


class Mesh:
    """A PMesh built by the reference's UnvToPMeshConverter."""

    def __init__(self, unv, case=None, fields=None, docs=None):
        if case is not None:
            fields, docs = case_docs(case)
        self._tmp = tempfile.TemporaryDirectory(prefix="prism_ref_")
        d = self._tmp.name
        path = os.path.join(d, "mesh.unvbin")
        write_unvbin(unv, path)
        with open(os.path.join(d, "fields.json"), "w") as fh:
            json.dump(fields, fh)
        for name, doc in docs.items():
            with open(os.path.join(d, name + ".json"), "w") as fh:
                json.dump(doc, fh)
        h = lib().ref_mesh_load(path.encode(), os.path.join(d, "fields.json").encode())
        if not h:
            raise RuntimeError("reference raised: " + lib().ref_last_error().decode())
        self.h = ctypes.c_void_p(h)
        s = np.zeros(6, np.int64)
        _check(lib().ref_mesh_sizes(self.h, _p(s, _pi64)))
        self.n_cells, self.n_faces, self.n_boundary, self.n_nonempty, self.n_interior, self.n_patches = map(int, s)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ref_mesh_free(self.h)
            self.h = None

    def faces(self):
        nf = self.n_faces
        owner, nbr, patch = (np.zeros(nf, np.int64) for _ in range(3))
        area = np.zeros(nf)
        normal, center = np.zeros(3 * nf), np.zeros(3 * nf)
        _check(lib().ref_mesh_faces(self.h, _p(owner, _pi64), _p(nbr, _pi64), _p(patch, _pi64), _p(area),
                                    _p(normal), _p(center)))
        return {"owner": owner, "nbr": nbr, "patch": patch, "area": area, "normal": normal.reshape(3, nf),
                "center": center.reshape(3, nf)}

    def cells(self):
        nc = self.n_cells
        center, vol = np.zeros(3 * nc), np.zeros(nc)
        _check(lib().ref_mesh_cells(self.h, _p(center), _p(vol)))
        return {"center": center.reshape(3, nc), "volume": vol}


def poisson(mesh, correctors=5, steps=15):
    """tests/test_poisson.cpp:24-50 run by the reference: the solved P."""
    P = np.zeros(mesh.n_cells)
    _check(lib().ref_poisson(mesh.h, correctors, steps, _p(P)))
    return P


def advection_1d(mesh):
    """tests/test_advection_1d.cpp:24-65 run by the reference: the solved T."""
    T = np.zeros(mesh.n_cells)
    _check(lib().ref_advection_1d(mesh.h, _p(T)))
    return T


def transport(mesh, conv=None, U=None, kappa=1.0, corrected=True, src=None, face_values=None, outer=1,
              n_iter=1, eps=0.0, method="bicgstab", T0=None, system=False):
    """Steady transport solved by the reference (see ref_transport in ref_cases.cpp). Returns T, and
    with system=True also the CSR matrix (rowptr, col, val) and rhs assembled at the final T."""
    nc = mesh.n_cells
    T = np.zeros(nc) if T0 is None else np.array(T0, dtype=np.float64)
    Uc = None if U is None else np.ascontiguousarray(U, np.float64).reshape(-1)
    srcc = None if src is None else np.ascontiguousarray(src, np.float64)
    fvc = None if face_values is None else np.ascontiguousarray(face_values, np.float64)
    cap = 0
    rp = col = val = rhs = None
    if system:
        cap = nc * 32
        rp, col, val, rhs = np.zeros(nc + 1, np.int64), np.zeros(cap, np.int64), np.zeros(cap), np.zeros(nc)
    nnz = lib().ref_transport(mesh.h, CONV[conv] if conv else 0, _p(Uc), float(kappa), 1 if corrected else 0,
                              _p(srcc), _p(fvc), int(outer), int(n_iter), float(eps),
                              1 if method == "jacobi" else 0, _p(T), cap, _p(rp, _pi64), _p(col, _pi64), _p(val),
                              _p(rhs))
    if nnz < 0:
        _check(1)
    if not system:
        return T
    return T, (rp, col[:nnz], val[:nnz]), rhs


def simple(mesh, iters, nu=1e-3, conv="LinearUpwind", symmetry=False, timings=False):
    """SIMPLE x iters run by the reference (tests/test_simple_coarse_pipe.cpp shape)."""
    nc, nf = mesh.n_cells, mesh.n_faces
    U, p = np.zeros(3 * nc), np.zeros(nc)
    flux, mflux = np.zeros(nf), np.zeros(nf)
    rep = np.zeros(48)
    nrep, needs = ctypes.c_int(0), ctypes.c_int(0)
    secs = np.zeros(max(iters, 1))
    _check(lib().ref_simple(mesh.h, float(nu), CONV[conv], 1 if symmetry else 0, int(iters), _p(U), _p(p),
                            _p(flux), _p(mflux), _p(rep), ctypes.byref(nrep), ctypes.byref(needs), _p(secs)))
    out = {"U": U.reshape(3, nc), "p": p, "flux": flux, "mdot_flux": mflux,
           "reports": rep[: 3 * nrep.value].reshape(-1, 3), "needs_ref": bool(needs.value)}
    if timings:
        out["seconds"] = secs[:iters]
    return out
