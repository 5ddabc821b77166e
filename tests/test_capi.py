"""The C-ABI library loads and exports every entry point its header declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(REPO, "include", "b200dwf.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(b200_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    import b200dwf
    lib = b200dwf.lib()
    names = declared_symbols()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n


def test_last_error_without_gpu_calls():
    import b200dwf
    msg = b200dwf.lib().b200_last_error()
    assert isinstance(msg, bytes)


def test_invalid_ls_rejected_before_any_device_work():
    import b200dwf
    lib = b200dwf.lib()
    h = ctypes.c_void_p()
    lat = (ctypes.c_int * 4)(4, 4, 4, 4)
    bc = (ctypes.c_int * 4)(1, 1, 1, -1)
    rc = lib.b200_dwf_create(ctypes.byref(h), lat, 5, 0.01, 1.8, None, None, 1.0, bc)
    assert rc == -1
    assert b"unsupported" in lib.b200_last_error()
    lat_odd = (ctypes.c_int * 4)(3, 4, 4, 4)
    rc = lib.b200_dwf_create(ctypes.byref(h), lat_odd, 8, 0.01, 1.8, None, None, 1.0, bc)
    assert rc == -1
