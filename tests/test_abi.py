"""The C-ABI library loads and exports every entry point include/tdda.h
declares (no compute calls: this runs without a GPU)."""
import os
import re

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "tdda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tdda_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_reference_methods():
    names = _declared()
    for n in ("tdda_model_create", "tdda_model_destroy", "tdda_solve_electric_field",
              "tdda_calculate_objective", "tdda_calculate_gradients", "tdda_set_parameters",
              "tdda_get_parameters", "tdda_get_dielectrics", "tdda_get_electric_field", "tdda_matvec"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from dda_model import _lib

    lib = _lib.load()
    for name in _declared():
        assert hasattr(lib, name), name
    # the ctypes table covers the header exactly
    assert set(_declared()) == set(_lib.SIGNATURES)
    assert lib.tdda_abi_version() == 1
    assert lib.tdda_status_string(1) == b"bad argument"
