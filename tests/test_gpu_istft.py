"""GPU parity of the inverse STFT (asdFftIstftMakePlan / asdFftExecIstft,
reference core/fft/istft.cpp, fftcore/fft_core_istft_any.cpp) against the FP64
restatement oracle.istft (itself checked against torch.istft on the CPU)."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from sip_b200 import fft

pytestmark = pytest.mark.gpu


def _make(x_t, n_fft, hop, win_len=None, **kw):
    import torch

    h = fft.asdFftCreate()
    a = fft.AclTensor.from_torch(x_t)
    lib = fft.load_library()
    st = lib.asdFftIstftMakePlan(h, a.ptr, n_fft, hop, win_len or n_fft, kw.get("center", True),
                                 kw.get("normalized", False), kw.get("onesided", False), kw.get("length", 0),
                                 kw.get("return_complex", True))
    a.close()
    ws = None
    if st == fft.ACL_SUCCESS:
        st2, nbytes = fft.asdFftGetWorkspaceSize(h)
        if nbytes:
            ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
            fft.asdFftSetWorkspace(h, ws.data_ptr())
    return h, st, ws


def _exec(h, x_t, w_t, y_t):
    t = [fft.AclTensor.from_torch(v) for v in (x_t, w_t, y_t)]
    try:
        return fft.load_library().asdFftExecIstft(h, *[a.ptr for a in t])
    finally:
        for a in t:
            a.close()


@pytest.mark.parametrize("n_fft,hop,frames,ch", [(64, 16, 10, 2), (400, 160, 33, 3), (512, 128, 40, 4),
                                                  (1024, 256, 9, 2), (1000, 1000, 5, 1), (96, 1, 7, 1)])
def test_istft_matches_oracle(cuda, n_fft, hop, frames, ch):
    import torch

    rng = np.random.default_rng(n_fft + hop)
    x = (rng.standard_normal((ch, n_fft, frames)) + 1j * rng.standard_normal((ch, n_fft, frames))).astype(np.complex64)
    w = (np.hanning(n_fft) + 0.05).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    h, st, ws = _make(xt, n_fft, hop)
    try:
        assert st == fft.ACL_SUCCESS
        st, typ = fft.asdFftGetType(h)
        assert typ == fft.ASCEND_FFT_C2C
        out_len = n_fft + hop * (frames - 1) - 2 * (n_fft // 2)
        y = torch.empty((ch, out_len), dtype=torch.complex64, device="cuda")
        assert _exec(h, xt, torch.from_numpy(w).cuda(), y) == fft.ACL_SUCCESS
        torch.cuda.synchronize()
        ref = oracle.istft(x, n_fft, hop, w)
        assert oracle.rel_l2(y.cpu().numpy(), ref) <= oracle.tolerance(n_fft)
    finally:
        fft.asdFftDestroy(h)


def test_istft_parameter_checks(cuda):
    import torch

    x = torch.zeros((2, 64, 8), dtype=torch.complex64, device="cuda")
    for kw, hop, win in [({}, 0, 64), ({}, 65, 64), ({}, 16, 32)]:
        h, st, _ = _make(x, 64, hop, win, **kw)
        assert st == fft.ACL_ERROR_INVALID_PARAM
        fft.asdFftDestroy(h)
    h, st, _ = _make(torch.zeros((2, 64, 1), dtype=torch.complex64, device="cuda"), 64, 16)  # one frame
    assert st == fft.ACL_ERROR_INVALID_PARAM
    fft.asdFftDestroy(h)
    h, st, _ = _make(torch.zeros((2, 2000, 4), dtype=torch.complex64, device="cuda"), 2000, 16)  # n_fft >= 1500
    assert st == fft.ACL_ERROR_INVALID_PARAM
    fft.asdFftDestroy(h)
    # unsupported options are forced (with a warning), as in the reference
    h, st, ws = _make(x, 64, 16, center=False, normalized=True, onesided=True, length=5, return_complex=False)
    try:
        assert st == fft.ACL_SUCCESS
        w = torch.ones(64, dtype=torch.float32, device="cuda")
        good = torch.empty((2, 64 + 16 * 7 - 64), dtype=torch.complex64, device="cuda")
        bad = torch.empty((2, 10), dtype=torch.complex64, device="cuda")
        assert _exec(h, x, w, bad) == fft.ACL_ERROR_INVALID_PARAM
        assert _exec(h, x, w.to(torch.complex64), good) == fft.ACL_ERROR_INVALID_PARAM
        assert _exec(h, x, w, good) == fft.ACL_SUCCESS
        # the plain exec entry points refuse an ISTFT plan
        a, b = fft.AclTensor.from_torch(good), fft.AclTensor.from_torch(good)
        assert fft.asdFftExecC2C(h, a, b) == fft.ACL_ERROR_INVALID_PARAM
        a.close()
        b.close()
    finally:
        fft.asdFftDestroy(h)
