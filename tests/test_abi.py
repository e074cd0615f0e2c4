"""CPU: the C-ABI library loads, exports every symbol the public headers
declare, and applies the reference's host-side parameter checks (no GPU work:
only entry points that fail before touching the device are called)."""
import ctypes
import os
import re

import pytest

from sip_b200 import fft

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in ("asdsip_fft.h", "asdsip_fft_ext.h"):
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b((?:acl|asdFft)\w+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_exports_every_declared_symbol(lib):
    declared = _declared_symbols()
    assert declared, "no declarations parsed"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert declared <= set(fft.EXPORTED_SYMBOLS)


def test_symbols_are_unmangled():
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", fft.LIB_PATH], capture_output=True, text=True).stdout
    syms = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for name in fft.EXPORTED_SYMBOLS:
        assert name in syms, name


def test_invalid_handle_status_codes(lib):
    bogus = ctypes.c_void_p(0x1234)
    assert lib.asdFftSetStream(bogus, ctypes.c_void_p(1)) == fft.ACL_ERROR_INVALID_PARAM
    assert lib.asdFftSetStream(bogus, None) == fft.ACL_ERROR_INVALID_PARAM
    assert lib.asdFftMakePlan1D(bogus, 8, fft.ASCEND_FFT_C2C, fft.ASCEND_FFT_FORWARD, 1,
                                fft.ASCEND_FFT_HORIZONTAL) == fft.ACL_ERROR_INVALID_PARAM
    n = ctypes.c_size_t(0)
    assert lib.asdFftGetWorkspaceSize(bogus, ctypes.byref(n)) == fft.ACL_ERROR_INVALID_PARAM
    assert lib.asdFftSetWorkspace(bogus, None) == fft.ACL_ERROR_INVALID_PARAM
    assert lib.asdFftDestroy(bogus) == fft.ACL_ERROR_INVALID_PARAM
    # Synchronize / GetType report an unknown handle as an internal error (fft_api.cpp:963-987)
    assert lib.asdFftSynchronize(bogus) == fft.ACL_ERROR_INTERNAL_ERROR
    t = ctypes.c_int(0)
    assert lib.asdFftGetType(bogus, ctypes.byref(t)) == fft.ACL_ERROR_INTERNAL_ERROR
    assert lib.asdFftExecC2C(bogus, None, None) == fft.ACL_ERROR_INVALID_PARAM


def test_plan_parameter_checks_before_device(lib):
    h = fft.asdFftCreate()
    try:
        C2C, FWD, H = fft.ASCEND_FFT_C2C, fft.ASCEND_FFT_FORWARD, fft.ASCEND_FFT_HORIZONTAL
        assert lib.asdFftMakePlan1D(h, 0, C2C, FWD, 1, H) == fft.ACL_ERROR_INVALID_PARAM
        assert lib.asdFftMakePlan1D(h, (1 << 27) + 1, C2C, FWD, 1, H) == fft.ACL_ERROR_INVALID_PARAM
        assert lib.asdFftMakePlan1D(h, 64, C2C, FWD, 0, H) == fft.ACL_ERROR_INVALID_PARAM
        assert lib.asdFftMakePlan2D(h, 0, 8, C2C, FWD, 1) == fft.ACL_ERROR_INVALID_PARAM
        assert lib.asdFftMakePlan2D(h, 8, 8, C2C, FWD, 0) == fft.ACL_ERROR_INVALID_PARAM
        assert lib.asdFftMakePlan3D(h, 8, 8, -1, C2C, FWD, 1) == fft.ACL_ERROR_INVALID_PARAM
        assert lib.asdFftMakePlan1D(h, 64, 0x99, FWD, 1, H) == fft.ACL_ERROR_INVALID_PARAM
        assert lib.asdFftMakePlan1D(h, 64, C2C, 0x42, 1, H) == fft.ACL_ERROR_INVALID_PARAM
        # an unplanned handle has workspace 0 and refuses to execute
        st, ws = fft.asdFftGetWorkspaceSize(h)
        assert st == fft.ACL_SUCCESS and ws == 0
        assert lib.asdFftExecRaw(h, ctypes.c_void_p(8), ctypes.c_void_p(16)) == fft.ACL_ERROR_INVALID_PARAM
        st, typ = fft.asdFftGetType(h)
        assert st == fft.ACL_SUCCESS
        # precision modes 0..3; anything else (or an unknown handle) is a parameter error
        for mode in (fft.PRECISION_FP16X3, fft.PRECISION_BF16X3, fft.PRECISION_AUTO, fft.PRECISION_FP32):
            assert lib.asdFftSetPrecision(h, mode) == fft.ACL_SUCCESS
        assert lib.asdFftSetPrecision(h, 4) == fft.ACL_ERROR_INVALID_PARAM
        assert lib.asdFftSetPrecision(h, -1) == fft.ACL_ERROR_INVALID_PARAM
        assert lib.asdFftSetPrecision(ctypes.c_void_p(0x1234), 1) == fft.ACL_ERROR_INVALID_PARAM
    finally:
        assert fft.asdFftDestroy(h) == fft.ACL_SUCCESS
    assert fft.asdFftDestroy(h) == fft.ACL_ERROR_INVALID_PARAM


def test_acl_tensor_shim(lib):
    t = fft.AclTensor([4, 3, 1024], fft.ACL_COMPLEX64, 0x1000)
    dt = ctypes.c_int(-5)
    assert lib.aclGetDataType(t.ptr, ctypes.byref(dt)) == 0 and dt.value == fft.ACL_COMPLEX64
    dims = ctypes.POINTER(ctypes.c_int64)()
    nd = ctypes.c_uint64(0)
    assert lib.aclGetViewShape(t.ptr, ctypes.byref(dims), ctypes.byref(nd)) == 0
    assert nd.value == 3 and [dims[i] for i in range(3)] == [4, 3, 1024]
    assert lib.aclGetTensorAddr(t.ptr) == 0x1000
    t.close()


def test_exec_rejects_mismatched_tensors_without_device(lib):
    """A handle that never planned fails the shape match before any launch."""
    h = fft.asdFftCreate()
    try:
        a = fft.AclTensor([2, 8], fft.ACL_FLOAT, 0x1000)
        assert fft.asdFftExecC2C(h, a, a) == fft.ACL_ERROR_INVALID_PARAM
    finally:
        fft.asdFftDestroy(h)
