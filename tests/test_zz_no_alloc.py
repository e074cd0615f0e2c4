"""GPU: the allocation-free C2C entry point.

Callers that cannot allocate device memory when they need a long transform
(allocation-free real-time loops, hosts that own every allocation) use
asdFftExecC2CNoAlloc, whose scratch is a fixed __device__ array of the
library instead of a plan workspace.  This checks it, through the C ABI,
against the ordinary plan + workspace entry point on two calls in a row (the
second call reuses the array the first one wrote).  The file is collected
last so that a run stopping at its first failure has run every other test."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from sip_b200 import fft

pytestmark = pytest.mark.gpu


def _no_alloc(lib, x_ptr, y_ptr, n, batch, direction, stream):
    fn = lib.asdFftExecC2CNoAlloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int32
    return fn(x_ptr, y_ptr, n, batch, direction, ctypes.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("n,batch,direction", [(32768, 4, fft.ASCEND_FFT_FORWARD),
                                               (65536, 16, fft.ASCEND_FFT_INVERSE),
                                               (3 * 2 ** 14, 5, fft.ASCEND_FFT_FORWARD),
                                               (2 ** 20, 1, fft.ASCEND_FFT_FORWARD),
                                               # 7 * 11 * 13 * 32: passes with odd radices
                                               (7 * 11 * 13 * 32, 3, fft.ASCEND_FFT_INVERSE)])
def test_no_alloc_matches_plan_path(cuda, n, batch, direction):
    import torch

    lib = fft.load_library()
    rng = np.random.default_rng(n + batch)
    stream = torch.cuda.current_stream()
    plan = fft.FftPlan([n], fft.ASCEND_FFT_C2C, direction, batch)
    tol = oracle.tolerance(n)
    for call in range(2):
        x = (rng.uniform(-1, 1, (batch, n)) + 1j * rng.uniform(-1, 1, (batch, n))).astype(np.complex64)
        xd = torch.from_numpy(x).cuda()
        y_ref = torch.empty_like(xd)
        plan(xd, y_ref)
        y = torch.full_like(xd, float("nan"))
        assert _no_alloc(lib, xd.data_ptr(), y.data_ptr(), n, batch, direction, stream) == fft.ACL_SUCCESS
        torch.cuda.synchronize()
        got, ref = y.cpu().numpy(), y_ref.cpu().numpy()
        assert np.all(np.isfinite(got)), f"call {call}"
        assert oracle.rel_l2(got, ref) <= tol, f"call {call}: {oracle.rel_l2(got, ref)}"
        assert oracle.rel_l2(got, oracle.c2c(x, direction == fft.ASCEND_FFT_FORWARD)) <= tol
    plan.close()


def test_no_alloc_in_place_at_the_size_limit(cuda):
    """input == output, length * batch exactly at the array's 2^20 limit with batch > 1:
    the tables and the intermediate never overlap the caller's buffer."""
    import torch

    lib = fft.load_library()
    n, batch = 65536, 16
    rng = np.random.default_rng(7)
    x = (rng.uniform(-1, 1, (batch, n)) + 1j * rng.uniform(-1, 1, (batch, n))).astype(np.complex64)
    buf = torch.from_numpy(x).cuda()
    stream = torch.cuda.current_stream()
    assert _no_alloc(lib, buf.data_ptr(), buf.data_ptr(), n, batch, fft.ASCEND_FFT_FORWARD, stream) == fft.ACL_SUCCESS
    torch.cuda.synchronize()
    assert oracle.rel_l2(buf.cpu().numpy(), oracle.c2c(x, True)) <= oracle.tolerance(n)


def test_no_alloc_rejects_sizes_beyond_the_array(cuda):
    import torch

    lib = fft.load_library()
    stream = torch.cuda.current_stream()
    x = torch.zeros(2 ** 20 + 64, dtype=torch.complex64, device="cuda")
    p = x.data_ptr()
    FWD = fft.ASCEND_FFT_FORWARD
    assert _no_alloc(lib, p, p, 65536, 17, FWD, stream) == fft.ACL_ERROR_INVALID_PARAM   # 17 * 65536 > 2^20
    assert _no_alloc(lib, p, p, 2 ** 21, 1, FWD, stream) == fft.ACL_ERROR_INVALID_PARAM  # longer than 2^20
    assert _no_alloc(lib, p, p, 8192, 1, FWD, stream) == fft.ACL_ERROR_INVALID_PARAM     # below the range
    assert _no_alloc(lib, p, p, 65536, 1, 0x42, stream) == fft.ACL_ERROR_INVALID_PARAM   # bad direction
    assert _no_alloc(lib, p, p, 17 * 2048, 1, FWD, stream) == fft.ACL_ERROR_API_NOT_SUPPORT  # no 2-pass split
