"""The C-ABI library loads on a machine without a GPU and exports every
function include/mps_capi.h declares (no compute calls here)."""
import os
import re

from helpers import HERE

ROOT = os.path.dirname(HERE)


def declared_functions():
    src = open(os.path.join(ROOT, "include", "mps_capi.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mps_[a-z_0-9]+)\s*\(", src)))


def test_header_and_binding_agree(capi):
    assert set(declared_functions()) == set(capi.EXPORTS)


def test_library_exports_every_declared_symbol(capi):
    L = capi.lib()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_status_strings_and_defaults(capi):
    L = capi.lib()
    assert L.mps_status_string(0) == b"ok"
    assert L.mps_status_string(3) == b"dt too small"
    o = capi.default_options()
    assert o.method == capi.METHOD_EXPLICIT and o.arith == capi.ARITH_EXACT
    assert o.cg_tol == 1e-8 and o.use_graph == 1


def test_native_library_has_no_oracle_dependency(capi):
    # the product library must not link or embed the CPU oracle
    data = open(capi.LIB_PATH, "rb").read()
    assert b"orc_create" not in data and b"liboracle" not in data
