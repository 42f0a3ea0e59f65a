"""CPU tests of the C-ABI library: it loads without a GPU, exports every function and data
symbol that include/bssn_b200.h declares, and its struct layouts equal the reference
project's (the drop-in contract)."""

import ctypes as C
import pathlib
import re

import pytest

from nrpy_b200 import lib as L

HEADER = pathlib.Path(__file__).resolve().parents[1] / "include" / "bssn_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set()
    for m in re.finditer(r"\b(?:void|int|const char \*|unsigned long long)\s+\**(\w+)\s*\(", text):
        names.add(m.group(1))
    return sorted(names)


def test_library_loads_without_gpu():
    lib = L.load()
    assert lib.bssn_b200_version().startswith(b"bssn_b200")


def test_every_declared_symbol_is_exported():
    lib = L.load()
    decl = declared_functions()
    assert len(decl) >= 40
    for name in decl:
        assert hasattr(lib, name), f"{name} declared in include/bssn_b200.h but not exported"
    for name in L.DATA_SYMBOLS:
        C.c_double.in_dll(lib, name)
    bound = {n for n, _, _ in L.SIGNATURES}
    assert set(decl) <= bound, sorted(set(decl) - bound)


def test_data_tables_match_reference_defines():
    lib = L.load()
    par = (C.c_int8 * 24).in_dll(lib, "bssn_b200_evol_gf_parity")
    assert list(par) == L.EVOL_GF_PARITY
    ws = (C.c_double * 24).in_dll(lib, "gridfunctions_wavespeed")
    fi = (C.c_double * 24).in_dll(lib, "gridfunctions_f_infinity")
    assert ws[6] == pytest.approx(2**0.5, rel=1e-12) and all(w == 1.0 for k, w in enumerate(ws) if k != 6)
    assert [k for k, v in enumerate(fi) if v != 0.0] == [6, 10]


def test_struct_layouts_match_reference_project():
    mine = {
        "sizeof_commondata": C.sizeof(L.CommondataStruct), "sizeof_params": C.sizeof(L.ParamsStruct),
        "sizeof_bc_struct": C.sizeof(L.BcStruct), "sizeof_griddata": C.sizeof(L.GriddataStruct),
        "sizeof_innerpt": C.sizeof(L.InnerptBcStruct), "sizeof_outerpt": C.sizeof(L.OuterptBcStruct),
        "offsetof_params_Nxx0": L.ParamsStruct.Nxx0.offset, "offsetof_params_invdxx0": L.ParamsStruct.invdxx0.offset,
        "offsetof_params_hash": L.ParamsStruct.CoordSystem_hash.offset,
        "offsetof_commondata_eta": L.CommondataStruct.eta.offset, "offsetof_commondata_dt": L.CommondataStruct.dt.offset,
        "offsetof_commondata_bc": L.CommondataStruct.outer_bc_type.offset,
        "offsetof_commondata_nn": L.CommondataStruct.nn.offset,
    }
    # Layout of the reference's generated BHaH_defines.h (x86-64), from oracle/ref_harness.c.
    # Its params_struct carries the CodeParameters of Spherical, SinhSpherical and SinhCylindrical.
    expected = {"sizeof_commondata": 232, "sizeof_params": 512, "sizeof_bc_struct": 552, "sizeof_griddata": 1136,
                "sizeof_innerpt": 20, "sizeof_outerpt": 10, "offsetof_params_Nxx0": 480,
                "offsetof_params_invdxx0": 152, "offsetof_params_hash": 476, "offsetof_commondata_eta": 112,
                "offsetof_commondata_dt": 104, "offsetof_commondata_bc": 160, "offsetof_commondata_nn": 216}
    assert mine == expected
    from oracle import ref

    for variant in ("sphaxi", "sph3d", "sinh3d", "sinhcyl"):
        if ref.available(variant):
            assert ref.struct_layout(variant) == expected


def test_symmetry_setting_validation():
    lib = L.load()
    assert lib.bssn_b200_set_symmetry_axes(b"2") == 0
    assert lib.bssn_b200_set_symmetry_axes(b"") == 0
    assert lib.bssn_b200_set_symmetry_axes(b"1") == 0  # SinhCylindrical, axisymmetric about z
    assert lib.bssn_b200_set_symmetry_axes(b"") == 0
    assert lib.bssn_b200_set_symmetry_axes(b"01") == -1
    assert b"only" in lib.bssn_b200_last_error()


def test_null_arguments_are_rejected_without_touching_the_gpu():
    lib = L.load()
    rc = lib.bssn_b200_rhs_eval(None, None, None, None, None, None, None)
    assert rc == -1 and b"NULL" in lib.bssn_b200_last_error()
    rc = lib.bssn_b200_mol_step(None, None, 1, 0, None)
    assert rc == -1
