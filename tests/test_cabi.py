"""The C-ABI library loads, exports every entry point include/droplet_b200.h
declares, and reports errors as codes plus a message (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT
from droplet_b200 import _native as N

HEADER = os.path.join(ROOT, "include", "droplet_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dr_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "dr_render_tile" in names and "dr_upload_scene" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(N.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    assert sorted(N.SIGNATURES) == declared_functions()


def test_version_and_errors():
    L = N.lib()
    assert L.dr_version() == N.DR_VERSION == 200
    rc = L.dr_create(0, None)
    assert rc == N.DR_ERR_INVALID
    assert b"null" in L.dr_last_error()
    assert L.dr_destroy(None) == N.DR_OK
    # batch calls refuse a null batch before touching the device
    assert L.dr_batch_set_split(None, 0) == N.DR_ERR_INVALID
    assert L.dr_batch_get_split(None, None, None) == N.DR_ERR_INVALID
    assert b"null batch" in L.dr_last_error()


def test_no_device_is_an_error_not_a_fallback():
    if N.device_count() > 0:
        pytest.skip("a GPU is present")
    ctx = C.c_void_p()
    rc = N.lib().dr_create(0, C.byref(ctx))
    assert rc in (N.DR_ERR_NODEVICE, N.DR_ERR_CUDA)
    assert not ctx.value
