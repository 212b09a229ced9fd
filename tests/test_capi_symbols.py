"""The C-ABI library loads without a GPU and exports every entry point that include/vca.h
declares (no compute calls)."""
import os
import re

from volcano_ca_mc_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "vca.h")).read()
    return sorted(set(re.findall(r"^(?:vca_status|void|const char\*)\s+(vca_\w+)\s*\(", text, re.M)))


def test_header_lists_every_export():
    assert header_symbols() == sorted(capi.EXPORTS)


def test_library_loads_and_exports_all():
    L = capi.lib()
    for name in header_symbols():
        assert hasattr(L, name), name
    assert L.vca_version().decode().startswith("vca 2 sm_100a")


def test_errors_without_device_are_reported_not_raised_in_c():
    # a bad descriptor is rejected before any CUDA call
    d = capi.CaParams(10, 10, 1, mode="lava").desc()  # 2D lava must be the x-z section
    import ctypes
    h = ctypes.c_void_p()
    st = capi.lib().vca_ca_create(ctypes.byref(d), ctypes.byref(h))
    assert st == 1 and not h.value
    assert "x-z" in capi.lib().vca_last_error().decode()
