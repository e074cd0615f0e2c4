"""GPU parity of ASCEND_FFT_C2C_SEP plans executed with asdFftExecC2CSeparated
(planar float32 real / imaginary tensors; reference fft_api.cpp:1236-1342,
planar cores ops/fft/c2c/dft_sep, fft_b_sep, c2c3d/ddd_sep) against the FP64
oracle: the result must equal the interleaved C2C of re + i im.
"""
import numpy as np
import pytest

from oracle import oracle
from sip_b200 import fft

pytestmark = pytest.mark.gpu

SEP, FWD, INV = fft.ASCEND_FFT_C2C_SEP, fft.ASCEND_FFT_FORWARD, fft.ASCEND_FFT_INVERSE


def _plan(sizes, direction, batch):
    import torch

    h = fft.asdFftCreate()
    if len(sizes) == 1:
        st = fft.asdFftMakePlan1D(h, sizes[0], SEP, direction, batch)
    elif len(sizes) == 2:
        st = fft.asdFftMakePlan2D(h, sizes[0], sizes[1], SEP, direction, batch)
    else:
        st = fft.asdFftMakePlan3D(h, *sizes, SEP, direction, batch)
    assert st == fft.ACL_SUCCESS, st
    st, ws = fft.asdFftGetWorkspaceSize(h)
    wbuf = None
    if ws:
        wbuf = torch.empty(ws, dtype=torch.uint8, device="cuda")
        fft.asdFftSetWorkspace(h, wbuf.data_ptr())
    return h, wbuf


def _exec(h, xr, xi, yr, yi):
    t = [fft.AclTensor.from_torch(v) for v in (xr, xi, yr, yi)]
    try:
        return fft.load_library().asdFftExecC2CSeparated(h, *[a.ptr for a in t])
    finally:
        for a in t:
            a.close()


CASES = [([1024], 7), ([4096], 3), ([3000], 5), ([17], 9), ([65536], 2), ([64, 96], 3), ([16, 24, 20], 2)]


@pytest.mark.parametrize("direction", [FWD, INV], ids=["fwd", "inv"])
@pytest.mark.parametrize("sizes,batch", CASES, ids=[f"{'x'.join(map(str, s))}_b{b}" for s, b in CASES])
def test_separated_matches_complex(cuda, sizes, batch, direction):
    import torch

    rng = np.random.default_rng(sum(sizes) + batch)
    shape = (batch, *sizes)
    xr = rng.uniform(-1, 1, shape).astype(np.float32)
    xi = rng.uniform(-1, 1, shape).astype(np.float32)
    h, ws = _plan(sizes, direction, batch)
    try:
        txr, txi = torch.from_numpy(xr).cuda(), torch.from_numpy(xi).cuda()
        yr, yi = torch.empty_like(txr), torch.empty_like(txi)
        assert _exec(h, txr, txi, yr, yi) == fft.ACL_SUCCESS
        torch.cuda.synchronize()
        assert fft.asdFftSynchronize(h) == fft.ACL_SUCCESS
        got = yr.cpu().numpy() + 1j * yi.cpu().numpy()
        ref = oracle.c2c((xr + 1j * xi).astype(np.complex128), direction == FWD, ndim=len(sizes))
        assert oracle.rel_l2(got, ref) <= oracle.tolerance(int(np.prod(sizes)))
    finally:
        fft.asdFftDestroy(h)


def test_separated_in_place_and_errors(cuda):
    import torch

    rng = np.random.default_rng(3)
    xr = rng.standard_normal((4, 512)).astype(np.float32)
    xi = rng.standard_normal((4, 512)).astype(np.float32)
    h, ws = _plan([512], FWD, 4)
    try:
        tr, ti = torch.from_numpy(xr).cuda(), torch.from_numpy(xi).cuda()
        assert _exec(h, tr, ti, tr, ti) == fft.ACL_SUCCESS  # in place on both planes
        torch.cuda.synchronize()
        ref = oracle.c2c(xr + 1j * xi, True)
        assert oracle.rel_l2(tr.cpu().numpy() + 1j * ti.cpu().numpy(), ref) <= oracle.tolerance(512)
        # planes of different shapes: 500000 (fft_api.cpp:1305-1336)
        short = torch.empty((4, 256), dtype=torch.float32, device="cuda")
        assert _exec(h, tr, ti, short, ti) == fft.ACL_ERROR_INTERNAL_ERROR
        # complex planes: 100000
        c = torch.empty((4, 512), dtype=torch.complex64, device="cuda")
        assert _exec(h, c, c, c, c) == fft.ACL_ERROR_INVALID_PARAM
        # interleaved exec on a separated plan: 100000
        a, b = fft.AclTensor.from_torch(c), fft.AclTensor.from_torch(c)
        assert fft.asdFftExecC2C(h, a, b) == fft.ACL_ERROR_INVALID_PARAM
        a.close()
        b.close()
    finally:
        fft.asdFftDestroy(h)
