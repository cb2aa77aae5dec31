"""The C ABI library loads and exports every entry point include/jkogb.h declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "jkogb.h")).read()
    return sorted(set(re.findall(r"\b(jk_[a-z0-9_]+)\s*\(", src)))


def test_header_and_python_agree():
    import jkogb_b200
    assert sorted(jkogb_b200.SYMBOLS) == _declared()


def test_library_exports_all_symbols():
    from jkogb_b200.build import build
    path = build()
    L = ctypes.CDLL(path)
    for name in _declared():
        assert hasattr(L, name), name


def test_argument_errors_without_gpu():
    # argument checks run before any CUDA call
    import numpy as np
    import jkogb_b200 as jk
    L = jk.lib()
    n = 4
    A = np.zeros((n, n))
    J = np.array([1, 1, -1, 2], np.int32)
    o = jk.Opts()
    d = lambda a: a.ctypes.data  # noqa: E731
    Jp = J.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    assert L.jk_dstep_loop(2, d(A), n, d(A), n, d(A), n, Jp, d(A), 0, 0, 0, ctypes.byref(o), None) == -1
    assert L.jk_dstep_loop(n, d(A), 3, d(A), n, d(A), n, Jp, d(A), 0, 0, 0, ctypes.byref(o), None) == -3
    assert L.jk_dstep_loop(n, d(A), n, d(A), 3, d(A), n, Jp, d(A), 0, 0, 0, ctypes.byref(o), None) == -5
    assert L.jk_dstep_loop(n, d(A), n, d(A), n, d(A), 2, Jp, d(A), 0, 0, 0, ctypes.byref(o), None) == -7
    assert L.jk_dstep_loop(n, d(A), n, d(A), n, d(A), n, Jp, d(A), -1, 0, 0, ctypes.byref(o), None) == -16
    assert L.jk_dstep_loop(n, d(A), n, d(A), n, d(A), n, Jp, d(A), 0, 4, 0, ctypes.byref(o), None) == -21
    assert L.jk_dstep_loop(n, d(A), n, d(A), n, d(A), n, Jp, d(A), 0, 0, 3, ctypes.byref(o), None) == -22
    assert L.jk_dstep_loop(n, d(A), n, d(A), n, d(A), n, Jp, d(A), 0, 0, 0, ctypes.byref(o), None) == -23
    assert jk.jstep_len(7, 0) == 3 and jk.jstep_len(7, 9) == 3 and jk.jstep_len(7, 2) == 2
    assert "J" in jk.strerror(-23)


def test_noalloc_argument_errors_without_gpu():
    # jk_dweights_noalloc rejects N beyond its static scratch before any CUDA call
    import numpy as np
    import jkogb_b200 as jk
    L = jk.lib()
    n = jk.NOALLOC_MAX_N + 1
    J = np.ones(n, np.int32)
    Jp = J.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    assert L.jk_dweights_noalloc(n, 16, Jp, 16, None) == -34
    assert "static scratch" in jk.strerror(-34)
    assert L.jk_dweights_noalloc(2, 16, Jp, 16, None) == -1
    assert L.jk_dweights_noalloc(8, None, Jp, 16, None) == -2
    assert L.jk_dweights_noalloc(8, 16, None, 16, None) == -8
    assert L.jk_dweights_noalloc(8, 16, Jp, None, None) == -4
    J[3] = 0
    assert L.jk_dweights_noalloc(8, 16, Jp, 16, None) == -23


def test_batched_argument_errors_without_gpu():
    # the batched plan checks orders, N_2 and J before any CUDA call
    import numpy as np
    import jkogb_b200 as jk
    L = jk.lib()
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))  # noqa: E731
    n = np.array([16, jk.BATCH_MAX_N + 2], np.int32)
    n2 = np.zeros(2, np.int32)
    J = np.ones(int(n.sum()), np.int32)
    info = ctypes.c_int(0)
    assert not L.jk_batch_create(2, ip(n), ip(n2), ip(J), None, ctypes.byref(info))
    assert info.value == -32
    n[1] = 2
    assert not L.jk_batch_create(2, ip(n), ip(n2), ip(J), None, ctypes.byref(info))
    assert info.value == -2
    n[1] = 8
    J[20] = 0
    assert not L.jk_batch_create(2, ip(n), ip(n2), ip(J), None, ctypes.byref(info))
    assert info.value == -23
    assert not L.jk_batch_create(0, ip(n), ip(n2), ip(J), None, ctypes.byref(info))
    assert info.value == -1


def test_ncp3_order_limit_without_gpu():
    # AW_NCP3 is limited to N <= 256; the check runs before any CUDA call
    import numpy as np
    import jkogb_b200 as jk
    L = jk.lib()
    n = 257
    A = np.zeros((n, n))
    J = np.ones(n, np.int32)
    o = jk.Opts()
    d = lambda a: a.ctypes.data  # noqa: E731
    Jp = J.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    assert L.jk_dstep_loop(n, d(A), n, d(A), n, d(A), n, Jp, d(A), 0, 3, 0, ctypes.byref(o), None) == -32


def test_device_buffer_checks_without_gpu():
    """NULL or misaligned device buffers are rejected with DSTEP_LOOP's argument positions
    (U -2, A -4, Z -6, SIGMA -9) before anything reaches a device.  Every call below has at
    least one such buffer, so none of them runs a kernel on the fake addresses."""
    import numpy as np
    import jkogb_b200 as jk
    L = jk.lib()
    n = 4
    J = np.array([1, 1, -1, -1], np.int32)
    Jp = J.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    o = jk.Opts()
    ok16, ok8, bad8, bad16 = 0x100000, 0x200000, 0x300004, 0x400008  # bad16: 8- but not 16-byte aligned
    V = ctypes.c_void_p
    def d(*a):  # noqa: E306
        return L.jk_dstep_loop_dev(n, V(a[0]), V(a[1]), V(a[2]), Jp, V(a[3]), 0, 0, 0, ctypes.byref(o), None, None)
    def z(*a):  # noqa: E306
        return L.jk_zstep_loop_dev(n, V(a[0]), V(a[1]), V(a[2]), Jp, V(a[3]), 0, 0, 0, ctypes.byref(o), None, None)
    assert d(None, ok8, ok8, ok8) == -2
    assert d(ok8, bad8, ok8, ok8) == -4
    assert d(ok8, ok8, None, ok8) == -6
    assert d(ok8, ok8, ok8, None) == -9
    assert d(ok8, ok8, ok8, bad8) == -9
    assert z(bad16, ok16, ok16, ok8) == -2
    assert z(ok16, bad16, ok16, ok8) == -4
    assert z(ok16, ok16, bad16, ok8) == -6
    assert z(ok16, ok16, ok16, bad8) == -9
