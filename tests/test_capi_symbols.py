"""The C-ABI library loads and exports every function include/troy_b200.h declares
(no compute calls: this runs without a GPU)."""
import ctypes

import tb_capi


def test_library_exports_every_declared_symbol():
    names = tb_capi.declared_functions()
    assert "tb_context_create" in names and "tb_ntt_forward" in names
    lib = ctypes.CDLL(tb_capi.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_invalid_arguments_fail_loudly_without_touching_the_device():
    lib = tb_capi.lib()
    h = ctypes.c_void_p()
    arr = (ctypes.c_uint64 * 1)(97)  # 97 is not 1 mod 2*64
    st = lib.tb_context_create(0, ctypes.c_uint64(64), arr, 1, ctypes.c_uint64(0), ctypes.byref(h))
    assert st == 1
    assert b"1 mod 2N" in lib.tb_last_error()
    st = lib.tb_context_create(0, ctypes.c_uint64(48), arr, 1, ctypes.c_uint64(0), ctypes.byref(h))
    assert st == 1
