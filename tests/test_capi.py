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


def test_null_handles_are_rejected_with_einval():
    """Every entry point that takes a plan or a network validates its handle
    and sizes before touching the device (as the reference's misuse checks
    do before any work)."""
    import b200dwf
    lib = b200dwf.lib()
    vp = ctypes.c_void_p
    n = ctypes.c_int()
    d = ctypes.c_double()
    h = vp()
    assert lib.b200_lp_create(ctypes.byref(h), None, 8, 1, 0.01) == -1
    assert lib.b200_lp_nparams(None) == 0
    assert lib.b200_lp_apply(None, None, None, None) == -1
    assert lib.b200_lp_adam_step(None, 1e-3, None) == -1
    assert lib.b200_lp_train(None, 1, None, None, 1, 1e-3, 1, None, None, None) == -1
    assert lib.b200_fcg_solve(None, None, None, None, 10, 1e-20, 2, ctypes.byref(n), ctypes.byref(n),
                              ctypes.byref(d), None) == -1
    assert lib.b200_cg_snapshots(None, 0, None, None, 10, 1e-20, 0, None, None, ctypes.byref(n), None) == -1
    assert lib.b200_cg_solve(None, 0, None, None, 10, 1e-20, ctypes.byref(n), ctypes.byref(d), None) == -1
    assert lib.b200_shiftcg_solve(None, None, None, 1, None, 10, 1e-20, ctypes.byref(n), ctypes.byref(d),
                                  None) == -1
    assert lib.b200_dwf_mult(None, 0, None, None, b"D", 0, None) == -1
    assert lib.b200_field_axpby(None, 0, None, 1.0, None, 0.0, None) == -1
    assert b"invalid" in lib.b200_last_error()


def test_python_mirror_has_the_reference_operator_interface():
    """DomainWall mirrors AFopr_Domainwall_5din_eo's public methods
    (src/lib/Fopr/afopr.h:65-202) and the solvers/force/smearing mirrors
    exist with the reference's names."""
    import b200dwf
    for name in ("set_config", "set_mode", "mult", "mult_dag", "convert", "reverse", "field_nin",
                 "field_nvol", "field_nex", "needs_convert", "cg", "shiftcg", "richardson",
                 "force_udiv", "force_udiv1", "fcg", "cg_snapshots"):
        assert hasattr(b200dwf.DomainWall, name), name
    for name in ("set_config", "config", "jacobian"):
        assert hasattr(b200dwf.StoutSmear, name), name
    for name in ("apply", "loss_grad", "grad", "adam_step", "train", "weights", "set_weights"):
        assert hasattr(b200dwf.LearnedPrecond, name), name
