"""CPU tests of the product boundary: the C-ABI library loads and exports every
entry point include/mclccd_b200.h declares (no compute calls without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mclccd_b200.h")
LIB = os.path.join(ROOT, "mclccd_b200", "libmclccd_b200.so")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mclccd_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("mclccd_create", "mclccd_destroy", "mclccd_update", "mclccd_traverse", "mclccd_get_hits",
              "mclccd_get_discrete", "mclccd_narrow_phase_bulk", "mclccd_last_error"):
        assert s in syms


def test_library_loads_and_exports_all_declared():
    assert os.path.exists(LIB), "build with make -C mclccd_b200"
    L = ctypes.CDLL(LIB)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_exports_are_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (mclccd_[a-z0-9_]+)$", out, flags=re.M))
    assert set(declared_symbols()) <= exported


def test_status_strings_need_no_gpu():
    L = ctypes.CDLL(LIB)
    L.mclccd_status_string.restype = ctypes.c_char_p
    assert L.mclccd_status_string(0) == b"ok"
    assert b"invalid" in L.mclccd_status_string(1)
    L.mclccd_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    assert L.mclccd_create(5, ctypes.byref(ctypes.c_void_p())) == 1   # bad dim rejected before any CUDA call


def test_python_mirror_fails_loudly_without_library(monkeypatch, tmp_path):
    import mclccd_b200.ccd as ccd
    monkeypatch.setattr(ccd, "_lib", None)
    monkeypatch.setattr(ccd, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(ImportError):
        ccd.lib()


def test_argument_checks_need_no_gpu():
    # entry points reject a null handle or invalid arguments with a status
    # before touching the device
    L = ctypes.CDLL(LIB)
    vp, ll = ctypes.c_void_p, ctypes.c_longlong
    null = vp(0)
    assert L.mclccd_traverse_out(null, null, null, 0, null, 0, null, null, null, ll(0), null, null, ll(0), null, 0) == 1
    assert L.mclccd_update_ex(null, null, null, 0, null, 0, 3, null, 0, ctypes.c_uint(0)) == 1
    assert L.mclccd_traverse_ex(null, null, null, 0, null, 0, ctypes.c_uint(0)) == 1
    assert L.mclccd_batch_set_tuning(null, 0, 128) == 1
    assert L.mclccd_batch_wave_stats(null, null, null) == 1
    # one-sided VF with the certified form in the bulk call: unsupported
    prec_cert, one_sided = 1, 0x100
    rc = L.mclccd_narrow_phase_bulk_ex(3, null, null, 0, null, null, ll(1), ctypes.c_double(1e-3),
                                       ctypes.c_double(1e-3), null, null, 0, null, prec_cert | one_sided, null)
    assert rc == 7
    rc = L.mclccd_narrow_phase_bulk_ex(5, null, null, 0, null, null, ll(1), ctypes.c_double(1e-3),
                                       ctypes.c_double(1e-3), null, null, 0, null, 0, null)
    assert rc == 1   # bad dim
