"""The C ABI library loads and exports every entry point include/gpsm.h declares."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gpsm.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(gpsm_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ["gpsm_init", "gpsm_graph_upload", "gpsm_match", "gpsm_match_ex", "gpsm_free"]:
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_no_device_is_an_error_not_a_fallback(lib):
    from conftest import HAS_GPU
    if HAS_GPU:
        return
    import gpsm_b200 as G
    try:
        G.init(0)
    except G.GpsmError as e:
        assert e.code == -7
    else:
        raise AssertionError("gpsm_init succeeded without a device")
