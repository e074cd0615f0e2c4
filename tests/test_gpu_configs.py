"""GPU parity of the workload configurations at their stated sizes.

* C1 — 1D C2C complex64, N = 1024, batch 256, forward then inverse; against the
  FP64 oracle and the reference's dense golden vectors (their rows repeated to
  the full batch).
* C3 — 2D C2C complex64 2048 x 2048 at batch 8, and 3D C2C 256^3 at batch 1, in
  every arithmetic form: plain FP32 and the tensor-core FP16 / BF16 hi/lo
  3-product forms (a 256-point axis has a tensor-core stage too).  The relative
  L2 and max-abs error against FP64 are printed per form.
* C4 — the seeded uneven set of 20 000 1D C2C transforms (lengths 64..65536,
  7-smooth, Zipf(1.2) batches capped at 512) in one persistent launch replayed
  from a CUDA graph: every row is checked by Parseval's identity and three rows
  of every length against the FP64 oracle.

Bar: relative L2 <= 1e-6 * log2(N) for every form (N = product of the sizes).
"""
import os

import numpy as np
import pytest

from oracle import oracle
from sip_b200 import fft, workloads

pytestmark = pytest.mark.gpu

C2C = fft.ASCEND_FFT_C2C
FWD, INV = fft.ASCEND_FFT_FORWARD, fft.ASCEND_FFT_INVERSE
FORMS = {"fp32": fft.PRECISION_FP32, "fp16x3": fft.PRECISION_FP16X3, "bf16x3": fft.PRECISION_BF16X3}
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz")


def _uniform_complex(rng, shape):
    return (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(np.complex64)


def _exec(sizes, direction, batch, xd, precision=fft.PRECISION_FP32):
    import torch

    plan = fft.FftPlan(sizes, C2C, direction, batch, precision=precision)
    try:
        y = torch.empty_like(xd)
        plan(xd, y)
        torch.cuda.synchronize()
        assert fft.asdFftSynchronize(plan.handle) == fft.ACL_SUCCESS
        return y, plan.describe()
    finally:
        plan.close()


def test_c1_c2c_1024_batch_256_forward_then_inverse(cuda):
    import torch

    n, batch = 1024, 256
    rng = np.random.default_rng(1)
    x = _uniform_complex(rng, (batch, n))
    xd = torch.from_numpy(x).cuda()
    X, _ = _exec([n], FWD, batch, xd)
    y, _ = _exec([n], INV, batch, X)
    Xh = X.cpu().numpy()
    err_f = oracle.rel_l2(Xh, oracle.c2c(x, True))
    err_rt = oracle.rel_l2(y.cpu().numpy() / n, x)
    print(f"C1 forward rel_l2={err_f:.2e} max_abs={oracle.max_abs(Xh, oracle.c2c(x, True)):.2e}; "
          f"round trip rel_l2={err_rt:.2e}")
    assert err_f <= oracle.tolerance(n)
    assert err_rt <= oracle.tolerance(n)
    # the reference's dense golden at N = 1024, its rows repeated over the full batch
    z = np.load(GOLDEN)
    for direction, tag in ((FWD, "fwd"), (INV, "inv")):
        gi, go = z[f"dense_c2c_{tag}_1024__in"], z[f"dense_c2c_{tag}_1024__out"]
        reps = batch // gi.shape[0] + 1
        xg = np.ascontiguousarray(np.tile(gi, (reps, 1))[:batch])
        yg, _ = _exec([n], direction, batch, torch.from_numpy(xg).cuda())
        err = oracle.rel_l2(yg.cpu().numpy(), np.tile(go, (reps, 1))[:batch])
        assert err <= 2e-6 * np.log2(n), (tag, err)


@pytest.fixture(scope="module")
def c3_2d():
    rng = np.random.default_rng(33)
    x = _uniform_complex(rng, (8, 2048, 2048))
    return x, oracle.c2c(x, True, ndim=2)


@pytest.mark.parametrize("form", list(FORMS))
def test_c3_2d_2048x2048_batch_8(cuda, c3_2d, form):
    import torch

    x, ref = c3_2d
    y, desc = _exec([2048, 2048], FWD, 8, torch.from_numpy(x).cuda(), FORMS[form])
    if form != "fp32":
        assert "tensor-core" in desc, desc
    yh = y.cpu().numpy()
    err, mx = oracle.rel_l2(yh, ref), oracle.max_abs(yh, ref)
    print(f"C3 2D 2048^2 x 8 {form}: rel_l2={err:.2e} max_abs={mx:.2e}")
    assert err <= oracle.tolerance(2048 * 2048), (form, err)


@pytest.fixture(scope="module")
def c3_3d():
    rng = np.random.default_rng(256)
    x = _uniform_complex(rng, (1, 256, 256, 256))
    return x, oracle.c2c(x, True, ndim=3)


@pytest.mark.parametrize("form", list(FORMS))
def test_c3_3d_256_cubed(cuda, c3_3d, form):
    import torch

    x, ref = c3_3d
    y, desc = _exec([256, 256, 256], FWD, 1, torch.from_numpy(x).cuda(), FORMS[form])
    yh = y.cpu().numpy()
    err, mx = oracle.rel_l2(yh, ref), oracle.max_abs(yh, ref)
    print(f"C3 3D 256^3 {form}: rel_l2={err:.2e} max_abs={mx:.2e}\n{desc}")
    assert err <= oracle.tolerance(256 ** 3), (form, err)


def test_c4_uneven_20000_transforms_one_graph_launch(cuda):
    import torch

    groups = workloads.uneven_batch_set(total=20000, seed=2024)
    assert sum(b for _, b in groups) == 20000
    plan = fft.BatchPlan(groups, FWD)
    try:
        rng = np.random.default_rng(4)
        g = torch.Generator(device="cuda").manual_seed(4)
        xd = torch.complex(torch.rand(plan.total, device="cuda", generator=g) * 2 - 1,
                           torch.rand(plan.total, device="cuda", generator=g) * 2 - 1)
        yd = torch.zeros_like(xd)
        plan(xd, yd, use_graph=True)
        plan(xd, yd, use_graph=True)  # a replay of the captured graph
        torch.cuda.synchronize()
        for (n, b), off in zip(plan.groups, plan.offsets):
            xs = xd[off:off + n * b].view(b, n)
            ys = yd[off:off + n * b].view(b, n)
            # Parseval on every row (unnormalised forward: sum |Y|^2 = N sum |X|^2)
            ex = (xs.abs() ** 2).double().sum(dim=1)
            ey = (ys.abs() ** 2).double().sum(dim=1) / n
            assert torch.all(torch.isfinite(ey))
            assert float(((ey - ex).abs() / ex).max()) <= 10 * oracle.tolerance(n), n
            rows = sorted({0, b - 1, int(rng.integers(0, b))})
            got = ys[rows].cpu().numpy()
            ref = oracle.c2c(xs[rows].cpu().numpy(), True)
            assert oracle.rel_l2(got, ref) <= oracle.tolerance(n), (n, b)
    finally:
        plan.close()
