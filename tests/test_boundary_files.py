"""The fields.json / <field>.json reader (prism_b200.io.read_case, the
MeshBoundary of mesh/boundary.cpp:291-319) on the reference's own boundary-file
fixtures (tests/cases/boundary/*, bundled into tests/golden/boundary_cases.json by
tests/golden/make_golden.py), with the assertions of tests/test_boundary.cpp.
The reference throws std::runtime_error where this reader raises ValueError."""
import json
import os

import pytest

from prism_b200 import _abi as A
from prism_b200 import io

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
with open(os.path.join(ROOT, "tests", "golden", "boundary_cases.json")) as _fh:
    BUNDLE = json.load(_fh)


def _case_dir(tmp_path, name):
    d = tmp_path / name
    d.mkdir()
    for fname, text in BUNDLE[name].items():
        (d / fname).write_text(text)
    return str(d / "fields.json")


def test_good_one_field(tmp_path):
    # test_boundary.cpp: "good_one_field loads correctly"
    case = io.read_case(_case_dir(tmp_path, "good_one_field"))
    assert list(case.field_info) == ["T"]
    assert case.field_info["T"]["type"] == "scalar"
    assert case.patch_names == ["Inlet", "Outlet", "Wall"]  # std::map order


def test_good_two_fields(tmp_path):
    # test_boundary.cpp: "good_two_fields parses scalar and vector"
    case = io.read_case(_case_dir(tmp_path, "good_two_fields"))
    assert list(case.field_info) == ["T", "U"]
    assert case.field_info["T"]["gradScheme"] == "greenGauss" and case.grad_scheme("T") == A.GRAD_GREEN_GAUSS
    assert len(case.field_info["T"]["units"]) == 9
    assert case.field_info["U"]["gradScheme"] == "leastSquares" and case.grad_scheme("U") == A.GRAD_LEAST_SQUARES
    assert len(case.patch_names) == 3
    inlet = case.patch_names.index("Inlet")
    t, u = case.fields["T"][inlet], case.fields["U"][inlet]
    assert (t.value_kind, t.value) == (A.BCV_SCALAR, 350.0)
    assert (u.value_kind, u.vector) == (A.BCV_VECTOR, (1.0, 0.0, 0.0))
    wall = case.fields["U"][case.patch_names.index("Wall")]
    assert wall.kind_str == "noSlip" and wall.value_kind == A.BCV_NIL


def test_good_empty_fields(tmp_path):
    # test_boundary.cpp: "good_empty_fields returns empty"
    case = io.read_case(_case_dir(tmp_path, "good_empty_fields"))
    assert not case.field_info and not case.fields and case.patch_names == []


@pytest.mark.parametrize("name", ["bad_missing_name", "bad_missing_type", "bad_missing_field_file",
                                  "bad_inconsistent_patches"])
def test_bad_files_rejected(tmp_path, name):
    # test_boundary.cpp: "bad_missing_name / bad_missing_type / bad_missing_field_file /
    # bad_inconsistent_patches throws"
    with pytest.raises(ValueError):
        io.read_case(_case_dir(tmp_path, name))


def test_missing_fields_file(tmp_path):
    # MeshBoundary::MeshBoundary: a fields.json that cannot be opened is an error
    with pytest.raises(OSError):
        io.read_case(str(tmp_path / "fields.json"))


def test_patch_lookups():
    # test_boundary.cpp BoundaryPatch cases: empty patches, direct lookup, component
    # fallback (U_x -> U), unknown fields and components rejected
    case = io.Case.from_dict(["Wall", "Inlet", "Front"],
                             {"T": {"Wall": ("fixed", 300.0), "Inlet": ("fixed", 350.0), "Front": ("empty", None)},
                              "U": {"Wall": ("noSlip", None), "Inlet": ("fixed", [1.0, 2.0, 3.0]),
                                    "Front": ("empty", None)}})
    assert case.patch_names == ["Front", "Inlet", "Wall"]
    assert case.patch_is_empty == [True, False, False]
    assert [b.kind for b in case.bcs("T")] == [A.BC_KIND_BY_NAME["empty"], A.BC_KIND_BY_NAME["fixed"],
                                               A.BC_KIND_BY_NAME["fixed"]]
    ux = case.bcs("U_x")
    assert ux[1].value_kind == A.BCV_VECTOR and list(ux[1].vector) == [1.0, 2.0, 3.0]
    for bad in ("P", "U_w"):
        with pytest.raises(KeyError):
            case.bcs(bad)
    with pytest.raises(ValueError):
        io.FieldBC("fixed", [1.0, 2.0])  # a vector value has three components
