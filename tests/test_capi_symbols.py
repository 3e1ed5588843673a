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


def test_misaligned_buffers_and_odd_strides_are_refused_on_the_host():
    """Transform entry points take coefficient pairs as 16-byte words: a buffer off a
    16-byte boundary or an odd stride is an error status, never a device access."""
    lib = tb_capi.lib()
    base = 1 << 20   # a fake, never-dereferenced address
    v = ctypes.c_void_p
    st = lib.tb_ntt_forward(None, v(base + 8), v(base), ctypes.c_uint64(1), 0, 1, 0, None)
    assert st == 1 and b"16-byte" in lib.tb_last_error()
    st = lib.tb_rescale_to_next(None, 2, v(base), ctypes.c_uint64(3), v(base), ctypes.c_uint64(0), 2,
                                ctypes.c_uint64(1), None)
    assert st == 1 and b"even" in lib.tb_last_error()
    st = lib.tb_relinearize(None, 2, v(base), ctypes.c_uint64(0), v(base + 4), ctypes.c_uint64(1), None)
    assert st == 1 and b"16-byte" in lib.tb_last_error()


def test_butterfly_rate_refuses_bad_moduli_on_the_host():
    lib = tb_capi.lib()
    for fn in (lib.tb_measure_butterfly_rate, lib.tb_measure_slack_butterfly_rate, lib.tb_measure_wide_butterfly_rate):
        fn.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        r = ctypes.c_double(0)
        for q in (0, 2, 1 << 40, (1 << 61) + 1):
            assert fn(q, None, ctypes.byref(r)) == 1
        assert b"2^61" in lib.tb_last_error()
    lib.tb_measure_mul64_rate.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
    r = ctypes.c_double(0)
    for kind in (-1, 2):
        assert lib.tb_measure_mul64_rate(kind, None, ctypes.byref(r)) == 1
