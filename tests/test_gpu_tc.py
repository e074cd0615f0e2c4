"""GPU parity of the tensor-core split-precision stages (asdFftSetPrecision
modes 1 = FP16 hi/lo x3 and 2 = BF16 hi/lo x3) against the FP64 oracle.

Bar: relative L2 error <= 1e-6 * log2(N), the FP32 gate of the path.  The
FP16 form must also agree with the numpy replay of the kernel
(tests/tc_model.py) to 2e-6: the tensor cores' FP32 accumulation does not
round like the replay's (measured differences about 7e-7), but a wrong operand
layout or scale would show as an O(1) difference.
"""
import numpy as np
import pytest

from oracle import oracle
from sip_b200 import fft

import tc_model

pytestmark = pytest.mark.gpu

C2C, R2C, C2R = fft.ASCEND_FFT_C2C, fft.ASCEND_FFT_R2C, fft.ASCEND_FFT_C2R
FWD, INV = fft.ASCEND_FFT_FORWARD, fft.ASCEND_FFT_INVERSE
MODES = [fft.PRECISION_FP16X3, fft.PRECISION_BF16X3]


def _rand_complex(rng, shape):
    return (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(np.complex64)


def _run(sizes, typ, direction, batch, x, precision, dim_type=fft.ASCEND_FFT_HORIZONTAL, inplace=False):
    import torch

    plan = fft.FftPlan(sizes, typ, direction, batch, dim_type, precision=precision)
    try:
        desc = plan.describe()
        xin = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        if inplace:
            out = xin
        elif typ == C2C:
            out = torch.empty_like(xin)
        elif typ == R2C:
            out = torch.empty(x.shape[:-1] + (sizes[-1] // 2 + 1,), dtype=torch.complex64, device="cuda")
        else:
            out = torch.empty(x.shape[:-1] + (sizes[-1],), dtype=torch.float32, device="cuda")
        plan(xin, out)
        torch.cuda.synchronize()
        assert fft.asdFftSynchronize(plan.handle) == fft.ACL_SUCCESS
        return out.cpu().numpy(), desc
    finally:
        plan.close()


@pytest.mark.parametrize("precision", MODES, ids=["fp16x3", "bf16x3"])
@pytest.mark.parametrize("direction", [FWD, INV], ids=["fwd", "inv"])
@pytest.mark.parametrize("n", [1024, 2048, 4096])
def test_c2c_rows(cuda, n, direction, precision):
    tb = tc_model.CONFIGS[n][2]
    batch = 37 * tb + 1  # several tiles per CTA and one partial tile
    rng = np.random.default_rng(n + precision)
    x = _rand_complex(rng, (batch, n))
    y, desc = _run([n], C2C, direction, batch, x, precision)
    assert "tensor-core" in desc and " rows " in desc, desc
    f = direction == FWD
    err = oracle.rel_l2(y, oracle.c2c(x, f))
    assert err <= oracle.tolerance(n), (err, desc)
    if precision == fft.PRECISION_FP16X3:
        rtb = tc_model.ROWS_CONFIGS[n][2]
        model = tc_model.tc_fft_rows(x[:2 * rtb], f, 0)
        assert oracle.rel_l2(y[:2 * rtb], model) <= 2e-6


@pytest.mark.parametrize("precision", MODES, ids=["fp16x3", "bf16x3"])
@pytest.mark.parametrize("n", [1024, 2048, 4096])
def test_c2c_rows_8_byte_aligned_buffers(cuda, n, precision):
    """Rows that start 8 bytes off a 16-byte boundary take the two-load path of the row pipeline."""
    import torch

    rows = 9
    rng = np.random.default_rng(n)
    x = _rand_complex(rng, (rows, n))
    plan = fft.FftPlan([n], C2C, FWD, rows, precision=precision)
    try:
        flat = torch.zeros(rows * n + 1, dtype=torch.complex64, device="cuda")
        xin = flat[1:].view(rows, n)
        xin.copy_(torch.from_numpy(x))
        out = torch.zeros(rows * n + 1, dtype=torch.complex64, device="cuda")[1:].view(rows, n)
        assert xin.data_ptr() % 16 == 8
        assert plan.exec_raw(xin.data_ptr(), out.data_ptr()) == fft.ACL_SUCCESS
        torch.cuda.synchronize()
        assert fft.asdFftSynchronize(plan.handle) == fft.ACL_SUCCESS
        assert oracle.rel_l2(out.cpu().numpy(), oracle.c2c(x, True)) <= oracle.tolerance(n)
    finally:
        plan.close()


@pytest.mark.parametrize("precision", MODES, ids=["fp16x3", "bf16x3"])
def test_c2c_inplace_and_scaled_inputs(cuda, precision):
    rng = np.random.default_rng(11)
    x = (_rand_complex(rng, (9, 1024)) * np.float32(3e4)).astype(np.complex64)
    y, _ = _run([1024], C2C, FWD, 9, x, precision, inplace=True)
    assert oracle.rel_l2(y, oracle.c2c(x, True)) <= oracle.tolerance(1024)


@pytest.mark.parametrize("precision", MODES, ids=["fp16x3", "bf16x3"])
def test_c2c_vertical_columns(cuda, precision):
    n, batch = 2048, 40
    rng = np.random.default_rng(3)
    x = _rand_complex(rng, (n, batch))
    y, desc = _run([n], C2C, FWD, batch, x, precision, fft.ASCEND_FFT_VERTICAL)
    # the strided axis is transposed into rows for the row pipeline and back
    assert "tensor-core" in desc and " rows " in desc and desc.count("transpose") == 2, desc
    assert oracle.rel_l2(y, oracle.c2c(x.T, True).T) <= oracle.tolerance(n)


@pytest.mark.parametrize("precision", MODES, ids=["fp16x3", "bf16x3"])
@pytest.mark.parametrize("direction", [FWD, INV], ids=["fwd", "inv"])
@pytest.mark.parametrize("n", [4096, 8192])
def test_real_transforms(cuda, n, direction, precision):
    rng = np.random.default_rng(n + direction)
    batch = 33
    f = direction == FWD
    xr = rng.standard_normal((batch, n)).astype(np.float32)
    y, desc = _run([n], R2C, direction, batch, xr, precision)
    assert "tensor-core" in desc, desc
    assert oracle.rel_l2(y, oracle.r2c(xr, f)) <= oracle.tolerance(n)
    h = n // 2 + 1
    xh = (rng.standard_normal((batch, h)) + 1j * rng.standard_normal((batch, h))).astype(np.complex64)
    y, desc = _run([n], C2R, direction, batch, xh, precision)
    assert "tensor-core" in desc, desc
    assert oracle.rel_l2(y, oracle.c2r(xh, n, f)) <= oracle.tolerance(n)


@pytest.mark.parametrize("precision", MODES, ids=["fp16x3", "bf16x3"])
@pytest.mark.parametrize("direction", [FWD, INV], ids=["fwd", "inv"])
def test_256_point_stage(cuda, direction, precision):
    """The 16 x 16 tensor-core DFT stage: rows, columns of a 3D volume, and the
    packed half of a 512-point real transform."""
    rng = np.random.default_rng(256 + direction)
    f = direction == FWD
    x = _rand_complex(rng, (8 * 37 + 3, 256))
    y, desc = _run([256], C2C, direction, x.shape[0], x, precision)
    assert "tensor-core" in desc, desc
    assert oracle.rel_l2(y, oracle.c2c(x, f)) <= oracle.tolerance(256)
    model = tc_model.tc_fft(x[:16], f, 0 if precision == fft.PRECISION_FP16X3 else 1)
    assert oracle.rel_l2(y[:16], model) <= 2e-6 if precision == fft.PRECISION_FP16X3 else True
    v = _rand_complex(rng, (2, 32, 256, 256))
    y, desc = _run([32, 256, 256], C2C, direction, 2, v, precision)
    assert desc.count("tensor-core") == 2, desc  # the 256-point Y and Z axes (X = 32 stays FP32)
    assert oracle.rel_l2(y, oracle.c2c(v, f, ndim=3)) <= oracle.tolerance(32 * 256 * 256)
    xr = rng.standard_normal((17, 512)).astype(np.float32)
    y, desc = _run([512], R2C, direction, 17, xr, precision)
    assert "tensor-core" in desc, desc
    assert oracle.rel_l2(y, oracle.r2c(xr, f)) <= oracle.tolerance(512)


@pytest.mark.parametrize("precision", MODES, ids=["fp16x3", "bf16x3"])
def test_2d_2048(cuda, precision):
    rng = np.random.default_rng(8)
    x = _rand_complex(rng, (2, 2048, 2048))
    y, desc = _run([2048, 2048], C2C, FWD, 2, x, precision)
    assert desc.count("tensor-core") == 2, desc
    assert oracle.rel_l2(y, oracle.c2c(x, True, ndim=2)) <= oracle.tolerance(2048 * 2048)


@pytest.mark.parametrize("precision", MODES, ids=["fp16x3", "bf16x3"])
@pytest.mark.parametrize("direction", [FWD, INV], ids=["fwd", "inv"])
def test_strided_axes_through_transposes(cuda, direction, precision):
    """Strided axes of 1024, 2048 and 4096 points run as transpose -> tensor-core
    row pipeline -> transpose (column counts that are not multiples of the 32 x 32
    transpose tile, several outer blocks, the R2C and C2R column passes)."""
    rng = np.random.default_rng(77 + direction)
    f = direction == FWD
    x = _rand_complex(rng, (3, 1024, 96))
    y, desc = _run([1024, 96], C2C, direction, 3, x, precision)
    assert desc.count("transpose") == 2 and desc.count("tensor-core") == 1, desc  # 96-point rows stay FP32
    assert oracle.rel_l2(y, oracle.c2c(x, f, ndim=2)) <= oracle.tolerance(1024 * 96)
    v = _rand_complex(rng, (2, 3, 4096, 40))
    y, desc = _run([3, 4096, 40], C2C, direction, 2, v, precision)
    assert desc.count("transpose") == 2, desc
    assert oracle.rel_l2(y, oracle.c2c(v, f, ndim=3)) <= oracle.tolerance(3 * 4096 * 40)
    xr = rng.standard_normal((2, 2048, 100)).astype(np.float32)
    y, desc = _run([2048, 100], R2C, direction, 2, xr, precision)
    assert desc.count("transpose") == 2, desc  # the 2048-point axis over 51 bins
    assert oracle.rel_l2(y, oracle.r2c(xr, f, ndim=2)) <= oracle.tolerance(2048 * 100)
    xh = _rand_complex(rng, (2, 2048, 51))
    y, desc = _run([2048, 100], C2R, direction, 2, xh, precision)
    assert desc.count("transpose") == 2, desc
    assert oracle.rel_l2(y, oracle.c2r(xh, 100, f, ndim=2)) <= oracle.tolerance(2048 * 100)


def test_fp32_default_has_no_tensor_core_step(cuda):
    rng = np.random.default_rng(1)
    x = _rand_complex(rng, (4, 1024))
    y, desc = _run([1024], C2C, FWD, 4, x, fft.PRECISION_FP32)
    assert "tensor-core" not in desc
    assert oracle.rel_l2(y, oracle.c2c(x, True)) <= oracle.tolerance(1024)


def test_set_precision_after_plan_grows_workspace(cuda):
    """A 2D plan made in FP32 needs no workspace; switched to a tensor-core form its
    1024-point strided axis runs between two transposes and needs workspace: the
    call succeeds, exec refuses until a workspace of the new size is set, then runs."""
    import torch

    plan = fft.FftPlan([1024, 64], C2C, FWD, 2)
    try:
        lib = fft.load_library()
        st, ws0 = fft.asdFftGetWorkspaceSize(plan.handle)
        assert st == fft.ACL_SUCCESS and ws0 == 0
        assert lib.asdFftSetPrecision(plan.handle, fft.PRECISION_BF16X3) == fft.ACL_SUCCESS
        st, ws1 = fft.asdFftGetWorkspaceSize(plan.handle)
        assert st == fft.ACL_SUCCESS and ws1 >= 2 * 2 * 1024 * 64 * 8, ws1
        rng = np.random.default_rng(12)
        x = _rand_complex(rng, (2, 1024, 64))
        xin = torch.from_numpy(x).cuda()
        out = torch.empty_like(xin)
        with pytest.raises(fft.FftError):
            plan(xin, out)
        wsp = torch.empty(ws1, dtype=torch.uint8, device="cuda")
        assert fft.asdFftSetWorkspace(plan.handle, wsp.data_ptr()) == fft.ACL_SUCCESS
        plan(xin, out)
        torch.cuda.synchronize()
        assert "transpose" in plan.describe()
        assert oracle.rel_l2(out.cpu().numpy(), oracle.c2c(x, True, ndim=2)) <= oracle.tolerance(1024 * 64)
    finally:
        plan.close()


def test_set_precision_after_plan_rebuilds(cuda):
    import torch

    plan = fft.FftPlan([2048], C2C, FWD, 8)
    try:
        assert "tensor-core" not in plan.describe()
        assert fft.load_library().asdFftSetPrecision(plan.handle, fft.PRECISION_FP16X3) == fft.ACL_SUCCESS
        assert "tensor-core fp16x3" in plan.describe()
        rng = np.random.default_rng(2)
        x = _rand_complex(rng, (8, 2048))
        xin = torch.from_numpy(x).cuda()
        out = torch.empty_like(xin)
        plan(xin, out)
        torch.cuda.synchronize()
        assert oracle.rel_l2(out.cpu().numpy(), oracle.c2c(x, True)) <= oracle.tolerance(2048)
    finally:
        plan.close()
