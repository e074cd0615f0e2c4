"""GPU: the continuous-batching server — every result matches the oracle,
a request gives the same result alone and in a mix with other requests, and
the Poisson driver completes every request."""
import numpy as np
import pytest

from oracle import oracle
from sip_b200 import fft, workloads

pytestmark = pytest.mark.gpu

C2C, R2C, FWD = fft.ASCEND_FFT_C2C, fft.ASCEND_FFT_R2C, fft.ASCEND_FFT_FORWARD


def _host_buffers(torch, typ, n, rows, seed):
    if typ == C2C:
        x = workloads.chirp_noise(n, rows, snr_db=10.0, seed=seed)
        xin = torch.from_numpy(x).pin_memory()
        out = torch.empty((rows, n), dtype=torch.complex64).pin_memory()
    else:
        x = workloads.chirp_noise(n, rows, snr_db=10.0, seed=seed).real.astype(np.float32)
        xin = torch.from_numpy(x).pin_memory()
        out = torch.empty((rows, n // 2 + 1), dtype=torch.complex64).pin_memory()
    return x, xin, out


def _ref(typ, x):
    return oracle.c2c(x, True) if typ == C2C else oracle.r2c(x, True)


@pytest.mark.parametrize("device_io", [False, True])
def test_alone_vs_mix(cuda, device_io):
    import torch

    srv = fft.Server(budget_bytes=8 << 30, lanes=3, max_rows=512, device_io=device_io)
    probe = (R2C, 4096, 100)
    x, xin, out = _host_buffers(torch, *probe, seed=1)
    if device_io:
        xin, out = xin.cuda(), out.cuda()
    assert srv.submit(probe[0], FWD, probe[1], probe[2], xin.data_ptr(), out.data_ptr()) >= 0
    ids, lat = srv.drain()
    assert len(ids) == 1 and lat[0] > 0
    torch.cuda.synchronize()
    alone = out.cpu().numpy().copy()
    assert oracle.rel_l2(alone, _ref(R2C, x)) <= oracle.tolerance(4096)

    # the same request inside a mix of classes and sizes, queued while the
    # server holds admissions, then released together
    srv.hold(True)
    mix = []
    rng = np.random.default_rng(3)
    classes = [(C2C, 4096), (R2C, 4096), (C2C, 8192), (R2C, 16384), (C2C, 65536)]
    for i in range(24):
        typ, n = classes[rng.integers(len(classes))]
        rows = int(rng.integers(1, 64))
        xm, xmin, outm = _host_buffers(torch, typ, n, rows, seed=100 + i)
        if device_io:
            xmin, outm = xmin.cuda(), outm.cuda()
        mix.append((typ, n, xm, xmin, outm))
        assert srv.submit(typ, FWD, n, rows, xmin.data_ptr(), outm.data_ptr()) >= 0
        if i == 11:
            out2 = torch.empty_like(out)
            assert srv.submit(probe[0], FWD, probe[1], probe[2], xin.data_ptr(), out2.data_ptr()) >= 0
    b0 = srv.batches()
    srv.hold(False)
    ids, lat = srv.drain()
    assert len(ids) == 25 and np.all(lat > 0)
    torch.cuda.synchronize()
    in_mix = out2.cpu().numpy()
    assert np.max(np.abs(in_mix - alone)) <= 1e-6 * np.max(np.abs(alone)), "result differs alone vs in the mix"
    for typ, n, xm, _, outm in mix:
        assert oracle.rel_l2(outm.cpu().numpy(), _ref(typ, xm)) <= oracle.tolerance(n)
    assert srv.batches() - b0 < 25  # same-class requests were batched together
    srv.close()


def test_poisson_driver(cuda):
    import torch

    srv = fft.Server(budget_bytes=4 << 30, lanes=4, max_rows=256, device_io=True)
    classes = [(C2C, 4096), (R2C, 8192)]
    pin, pout, keep = [], [], []
    for typ, n in classes:
        a = torch.randn(256, n, dtype=torch.complex64 if typ == C2C else torch.float32, device="cuda")
        b = torch.empty(256, n if typ == C2C else n // 2 + 1, dtype=torch.complex64, device="cuda")
        keep += [a, b]
        pin.append(a.data_ptr())
        pout.append(b.data_ptr())
    for typ, n in classes:
        assert srv.warm(typ, FWD, n) == fft.ACL_SUCCESS
    wall, lat, rows, cls = srv.run_poisson(2000.0, 300, 7, classes, pin, pout, 16, 256)
    assert wall > 0 and np.all(lat > 0), (wall, lat.min())
    assert set(cls.tolist()) == {0, 1}
    srv.close()


def test_large_device_requests_direct_and_in_place(cuda):
    """Device requests of 8 MB or more run on their own buffers (no staging
    copies); one whose output is its input keeps the staged path.  Both against
    the oracle, batched with a small staged request of the same class."""
    import torch

    srv = fft.Server(budget_bytes=8 << 30, lanes=2, max_rows=64, device_io=True)
    n = 65536
    work = []
    for i, rows in enumerate((20, 3)):          # 10.5 MB (direct) and 1.6 MB (staged)
        x = workloads.chirp_noise(n, rows, snr_db=10.0, seed=900 + i)
        xin = torch.from_numpy(x).cuda()
        out = torch.empty_like(xin)
        work.append((x, xin, out))
    x2 = workloads.chirp_noise(n, 17, snr_db=10.0, seed=950)
    inplace = torch.from_numpy(x2).cuda()       # 8.9 MB, output over the input
    srv.hold(True)
    for x, xin, out in work:
        assert srv.submit(C2C, FWD, n, x.shape[0], xin.data_ptr(), out.data_ptr()) >= 0
    assert srv.submit(C2C, FWD, n, 17, inplace.data_ptr(), inplace.data_ptr()) >= 0
    srv.hold(False)
    ids, lat = srv.drain()
    assert len(ids) == 3 and np.all(lat > 0)
    torch.cuda.synchronize()
    for x, _, out in work:
        assert oracle.rel_l2(out.cpu().numpy(), oracle.c2c(x, True)) <= oracle.tolerance(n)
    assert oracle.rel_l2(inplace.cpu().numpy(), oracle.c2c(x2, True)) <= oracle.tolerance(n)
    srv.close()


def test_server_rejects_bad_requests(cuda):
    srv = fft.Server(budget_bytes=1 << 30, lanes=1, max_rows=8)
    assert srv.submit(C2C, FWD, 64, 9, 16, 16) == -1      # more rows than a lane holds
    assert srv.submit(0x11, FWD, 64, 1, 16, 16) == -1     # C2R is not a serving class
    assert srv.submit(R2C, FWD, 63, 1, 16, 16) == -1      # odd R2C length
    ids, _ = srv.drain()
    assert len(ids) == 0
    srv.close()


@pytest.mark.parametrize("precision", [fft.PRECISION_FP16X3, fft.PRECISION_BF16X3], ids=["fp16x3", "bf16x3"])
def test_split_precision_server(cuda, precision):
    """A server whose resident plans use the tensor-core split forms: results within the
    FP32 bar for every class (C2C 4096 takes the tensor-core row pipeline, R2C 8192 the
    tensor-core tile kernel, the other classes the FP32 kernels); the precision cannot be
    changed once plans exist."""
    import torch

    srv = fft.Server(budget_bytes=8 << 30, lanes=2, max_rows=256, device_io=True, precision=precision)
    assert fft.load_library().asdFftServerSetPrecision(srv.handle, fft.PRECISION_FP32) == fft.ACL_SUCCESS
    assert fft.load_library().asdFftServerSetPrecision(srv.handle, precision) == fft.ACL_SUCCESS
    work = []
    for i, (typ, n) in enumerate([(C2C, 4096), (R2C, 8192), (C2C, 16384), (R2C, 4096), (C2C, 4096)]):
        rows = 37 + 11 * i
        x, xin, out = _host_buffers(torch, typ, n, rows, seed=700 + i)
        xin, out = xin.cuda(), out.cuda()
        work.append((typ, n, x, xin, out))
        assert srv.submit(typ, FWD, n, rows, xin.data_ptr(), out.data_ptr()) >= 0
    ids, lat = srv.drain()
    assert len(ids) == 5 and np.all(lat > 0)
    torch.cuda.synchronize()
    for typ, n, x, _, out in work:
        assert oracle.rel_l2(out.cpu().numpy(), _ref(typ, x)) <= oracle.tolerance(n)
    assert fft.load_library().asdFftServerSetPrecision(srv.handle, fft.PRECISION_FP32) == fft.ACL_ERROR_INVALID_PARAM
    srv.close()
