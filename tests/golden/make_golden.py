"""Generate tests/golden/*.npz from the reference's own test cases.

Run in a container where the reference checkout is available, giving the path of its
tests/cases directory:

    python tests/golden/make_golden.py <reference>/tests/cases [case names]

For each case it stores the mesh in converter form (nodes, element list,
groups; re-encoded from the case's mesh.unv), the parsed fields.json and
<field>.json documents, and the CPU oracle's results for the reference test
that uses the case (tests/test_poisson.cpp, test_advection_1d.cpp,
test_simple_coarse_pipe.cpp, test_needs_pressure_ref.cpp, test_transient_1d.cpp). The GPU tests
compare the sm_100a path with these arrays; the CPU tests re-run the oracle and
check it against the reference tests' own thresholds.

The case name "boundary" bundles the fields.json / <field>.json files of the
reference's boundary-file tests (tests/test_boundary.cpp, cases/boundary/*)
into boundary_cases.json: {case: {file name: file text}}.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from tests import cases  # noqa: E402
from prism_b200 import io  # noqa: E402

CASES = {
    "poisson_hex": ("poisson", "mesh_hex.unv"),
    "poisson_wedge": ("poisson", "mesh.unv"),
    "versteeg_advection_1d": ("versteeg_advection_1d", "mesh.unv"),
    "coarse_pipe": ("coarsePipeHex", "mesh.unv"),
    "cavity_hex": ("cavity_hex", "mesh.unv"),
    "duct_simple": ("ductSIMPLE", "mesh.unv"),
    "versteeg_trans_1d": ("versteeg_trans_1d", "mesh.unv"),
}


def boundary_files(src, out_dir):
    base = os.path.join(src, "boundary")
    bundle = {}
    for case in sorted(os.listdir(base)):
        d = os.path.join(base, case)
        bundle[case] = {}
        for f in sorted(os.listdir(d)):
            with open(os.path.join(d, f)) as fh:
                bundle[case][f] = fh.read()
    with open(os.path.join(out_dir, "boundary_cases.json"), "w") as fh:
        json.dump(bundle, fh, indent=1, sort_keys=True)
    print("boundary", {c: sorted(v) for c, v in bundle.items()})


def main(src, only=None):
    out_dir = os.path.dirname(os.path.abspath(__file__))
    if not only or "boundary" in only:
        boundary_files(src, out_dir)
    for name, (case_dir, mesh_file) in CASES.items():
        if only and name not in only:
            continue
        base = os.path.join(src, case_dir)
        unv = io.read_unv(os.path.join(base, mesh_file))
        with open(os.path.join(base, "fields.json")) as fh:
            fdoc = json.load(fh)
        docs = {}
        for f in fdoc["fields"]:
            p = os.path.join(base, f["name"] + ".json")
            if os.path.exists(p):
                with open(p) as fh:
                    docs[f["name"]] = json.load(fh)
        extra = {}
        if os.path.exists(os.path.join(base, "foam_fields.json")):
            with open(os.path.join(base, "foam_fields.json")) as fh:
                foam = json.load(fh)
            extra["foam_p"] = np.array(foam["p"], dtype=np.float64)
            extra["foam_U"] = np.array(foam["U"], dtype=np.float64)
        gnames = [g[0] for g in unv.groups]
        gvert = np.array([g[1] for g in unv.groups], dtype=np.int8)
        goff = np.cumsum([0] + [len(g[2]) for g in unv.groups]).astype(np.int64)
        gel = np.concatenate([g[2] for g in unv.groups]).astype(np.int32)
        arrays = dict(xyz=unv.xyz, elem_kind=unv.elem_kind.astype(np.int8),
                      elem_offsets=unv.elem_offsets.astype(np.int32),
                      elem_nodes=unv.elem_nodes.astype(np.int32), group_offsets=goff,
                      group_is_vertex=gvert, group_elements=gel,
                      meta=np.array(json.dumps({"groups": gnames, "fields": fdoc, "docs": docs})))
        arrays.update(extra)
        path = os.path.join(out_dir, name + ".npz")
        np.savez_compressed(path, **arrays)
        # oracle results for the reference test using the case
        lib = oracle.lib()
        res = cases.run_reference_test(name, lib)
        np.savez_compressed(os.path.join(out_dir, name + "_oracle.npz"), **res)
        print(name, os.path.getsize(path), {k: (v.shape if hasattr(v, "shape") else v) for k, v in res.items()})


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <reference tests/cases directory> [case names]")
    main(sys.argv[1], sys.argv[2:])
