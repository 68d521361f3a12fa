"""The C-ABI library loads and exports every symbol include/wilson_sm100.h
declares (no device calls: runs without a GPU)."""

import ctypes
import os
import re

from jaxqft_b200 import lib as L


def _declared():
    txt = open(L.HEADER_PATH).read()
    return set(re.findall(r"\b(wl_[a-z_0-9]+)\s*\(", txt)) - {"wl_status"}


def test_library_builds_and_loads():
    lib = L.load_library()
    assert os.path.exists(L.LIB_PATH)
    assert lib.wl_version() == 1


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(L.LIB_PATH)
    declared = _declared()
    assert declared, "no declarations parsed"
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert declared == set(L.EXPORTS)


def test_context_rejects_odd_extents_without_device_work():
    lib = L.load_library()
    g = L.WLGeometry()
    for mu, v in enumerate((4, 4, 3, 4)):
        g.dims[mu] = v
        g.bc_re[mu] = 1.0
    h = ctypes.c_void_p()
    rc = lib.wl_ctx_create(ctypes.byref(g), 0, ctypes.byref(h))
    assert rc == L.WL_ERR_ARG
    assert b"even" in lib.wl_last_error(None)


def test_release_build_reports_no_index_checks():
    """wl_bounds_errors is -1 in the release library (the checks are compiled
    only into libwilson_sm100_check.so); it makes no device call there."""
    lib = L.load_library()
    first = ctypes.c_longlong(7)
    assert lib.wl_bounds_errors(ctypes.byref(first)) == -1
    assert first.value == 0
