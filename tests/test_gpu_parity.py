"""GPU parity: the library's sm_100a kernels, called through the C ABI, against
the FP64 oracle and against the reference's golden vectors.

Bar: relative L2 error <= 1e-6 * log2(N) (N = product of the transform sizes),
the accuracy gate the path is specified with; the golden vectors (FP32 outputs
of the reference's FP32 matrices) get 2e-6 * log2(N).
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle
from sip_b200 import fft

pytestmark = pytest.mark.gpu

C2C, R2C, C2R = fft.ASCEND_FFT_C2C, fft.ASCEND_FFT_R2C, fft.ASCEND_FFT_C2R
FWD, INV = fft.ASCEND_FFT_FORWARD, fft.ASCEND_FFT_INVERSE
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz")


def _tol(sizes):
    return oracle.tolerance(int(np.prod(sizes)))


def _rand_complex(rng, shape):
    return (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(np.complex64)


def run(sizes, typ, direction, batch, x, dim_type=fft.ASCEND_FFT_HORIZONTAL):
    import torch

    plan = fft.FftPlan(sizes, typ, direction, batch, dim_type)
    try:
        xin = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        if typ == C2C:
            out = torch.empty_like(xin)
        elif typ == R2C:
            out = torch.empty(x.shape[:-1] + (sizes[-1] // 2 + 1,), dtype=torch.complex64, device="cuda")
        else:
            out = torch.empty(x.shape[:-1] + (sizes[-1],), dtype=torch.float32, device="cuda")
        plan(xin, out)
        torch.cuda.synchronize()
        return out.cpu().numpy()
    finally:
        plan.close()


def check(sizes, typ, fwd, batch, seed=0, vertical=False):
    rng = np.random.default_rng(seed)
    nd = len(sizes)
    f = fwd == FWD
    if typ == C2C:
        shape = (sizes[0], batch) if vertical else (batch, *sizes)
        x = _rand_complex(rng, shape)
        dim = fft.ASCEND_FFT_VERTICAL if vertical else fft.ASCEND_FFT_HORIZONTAL
        y = run(sizes, typ, fwd, batch, x, dim)
        ref = oracle.c2c(x.T, f).T if vertical else oracle.c2c(x, f, ndim=nd)
    elif typ == R2C:
        x = rng.standard_normal((batch, *sizes)).astype(np.float32)
        y = run(sizes, typ, fwd, batch, x)
        ref = oracle.r2c(x, f, ndim=nd)
    else:
        h = sizes[-1] // 2 + 1
        x = (rng.standard_normal((batch, *sizes[:-1], h)) + 1j * rng.standard_normal((batch, *sizes[:-1], h)))
        x = x.astype(np.complex64)
        y = run(sizes, typ, fwd, batch, x)
        ref = oracle.c2r(x, sizes[-1], f, ndim=nd)
    err = oracle.rel_l2(y, ref)
    assert err <= _tol(sizes), f"{sizes} type={typ:#x} dir={fwd:#x} batch={batch}: rel L2 {err:.3e}"
    return err


C2C_SIZES = [1, 2, 3, 4, 5, 7, 8, 11, 13, 16, 30, 64, 100, 128, 143, 210, 256, 343, 512, 1000, 1024, 1500,
             2048, 3000, 4096, 6561, 8192, 10000, 15000, 16384, 24576, 32768, 65536, 3 * 2 ** 15, 2 ** 20,
             # prime factors above 13: Bluestein (single-tile convolution up to M = 16384, multi-pass above)
             17, 31, 97, 202, 1021, 4099, 8191, 17 * 1024, 199 * 1000, 65537, 199 * 199 * 13]


@pytest.mark.parametrize("n", C2C_SIZES)
@pytest.mark.parametrize("fwd", [FWD, INV])
def test_c2c_1d(cuda, n, fwd):
    batch = 3 if n >= 4096 else 37
    check([n], C2C, fwd, batch, seed=n)


REAL_SIZES = [1, 2, 3, 4, 5, 6, 7, 30, 64, 100, 243, 256, 1000, 1024, 3000, 4096, 8192, 15625, 16384,
              30000, 65536, 131072,
              # prime factors above 13 (Bluestein): odd, even, and even with an odd large half;
              # multi-pass convolutions for the long ones
              17, 31, 34, 1021, 2042, 17 * 1024, 199 * 1000, 2 * 65537, 65537]


@pytest.mark.parametrize("n", REAL_SIZES)
@pytest.mark.parametrize("fwd", [FWD, INV])
@pytest.mark.parametrize("typ", [R2C, C2R])
def test_real_1d(cuda, n, fwd, typ):
    batch = 3 if n >= 4096 else 21
    check([n], typ, fwd, batch, seed=n + typ)


@pytest.mark.parametrize("n,batch", [(256, 128), (1024, 200), (60, 33), (4096, 16),
                                     # long strided axes: multi-pass column tiles (the reference's
                                     # vertical 1D takes powers of two up to 65536)
                                     (16384, 128), (65536, 128), (3 * 5 * 7 * 1024, 16), (262144, 16)])
@pytest.mark.parametrize("fwd", [FWD, INV])
def test_c2c_vertical(cuda, n, batch, fwd):
    check([n], C2C, fwd, batch, seed=n, vertical=True)


@pytest.mark.parametrize("shape,typ", [((65536, 4), C2C), ((16384, 8), C2C), ((32768, 6), R2C), ((32768, 6), C2R),
                                       ((4, 16384, 8), C2C)])
def test_long_strided_axes(cuda, shape, typ):
    """2D / 3D plans whose strided (leading) axes are too long for one column tile."""
    check(list(shape), typ, FWD, 2, seed=int(np.prod(shape)))


# (4096, 40), (1536, 33), (3000, 8): strided axes above 1024 points without a TMA column
# engine, which run through transposes into rows
SIZES_2D = [(1, 1), (3, 5), (32, 32), (64, 128), (100, 60), (2, 4096), (2048, 2048), (4096, 40), (1536, 33),
            (3000, 8)]


@pytest.mark.parametrize("xy", SIZES_2D)
@pytest.mark.parametrize("typ", [C2C, R2C, C2R])
@pytest.mark.parametrize("fwd", [FWD, INV])
def test_2d(cuda, xy, typ, fwd):
    batch = 1 if xy[0] * xy[1] > 100000 else 3
    check(list(xy), typ, fwd, batch, seed=xy[0] * 7 + xy[1])


SIZES_3D = [(2, 3, 4), (8, 16, 32), (16, 16, 16), (5, 7, 30), (256, 256, 256), (3, 4096, 8)]


@pytest.mark.parametrize("xyz", SIZES_3D)
@pytest.mark.parametrize("typ", [C2C, R2C, C2R])
@pytest.mark.parametrize("fwd", [FWD, INV])
def test_3d(cuda, xyz, typ, fwd):
    batch = 1 if np.prod(xyz) > 100000 else 2
    check(list(xyz), typ, fwd, batch, seed=int(np.prod(xyz)))


def test_golden_vectors_through_library(cuda):
    z = np.load(GOLDEN)
    for name, kind, n, f in zip(z["_names"], z["_kinds"], z["_sizes"], z["_forward"]):
        name, kind, n, f = str(name), str(kind), int(n), bool(f)
        typ = {"c2c": C2C, "r2c": R2C, "c2r": C2R}[kind]
        x = z[name + "__in"]
        y = run([n], typ, FWD if f else INV, x.shape[0], x)
        err = oracle.rel_l2(y, z[name + "__out"])
        assert err <= 2e-6 * max(1.0, np.log2(max(n, 2))), (name, err)


def test_golden_vectors_nd_through_library(cuda):
    """2D / 3D C2C, R2C and C2R against the reference's per-axis matrices
    applied in the order of its multi-dimensional plans."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors_nd.npz"))
    for name, kind, shape, nd, f in zip(z["_names"], z["_kinds"], z["_shapes"], z["_ndim"], z["_forward"]):
        sizes = [int(v) for v in shape[:nd]]
        typ = {"c2c": C2C, "r2c": R2C, "c2r": C2R}[str(kind)]
        x = z[str(name) + "__in"]
        y = run(sizes, typ, FWD if f else INV, x.shape[0], x)
        err = oracle.rel_l2(y, z[str(name) + "__out"])
        assert err <= 2e-6 * max(1.0, np.log2(int(np.prod(sizes)))), (str(name), err)


@pytest.mark.parametrize("n", [3000, 4096])
def test_round_trip_full_size(cuda, n):
    """C2R(INVERSE)(R2C(FORWARD)(x)) / N == x at the benchmark's full size (batch 4096)."""
    import torch

    rng = np.random.default_rng(n)
    x = rng.standard_normal((4096, n)).astype(np.float32)
    f = fft.FftPlan([n], R2C, FWD, 4096)
    g = fft.FftPlan([n], C2R, INV, 4096)
    xd = torch.from_numpy(x).cuda()
    X = torch.empty((4096, n // 2 + 1), dtype=torch.complex64, device="cuda")
    y = torch.empty_like(xd)
    f(xd, X)
    g(X, y)
    torch.cuda.synchronize()
    err = oracle.rel_l2(y.cpu().numpy() / n, x)
    assert err <= oracle.tolerance(n), err
    # the forward half alone against the oracle on a subset of rows
    ref = oracle.r2c(x[:64], True)
    assert oracle.rel_l2(X[:64].cpu().numpy(), ref) <= oracle.tolerance(n)
    f.close()
    g.close()


def test_in_place_c2c(cuda):
    import torch

    rng = np.random.default_rng(5)
    for n, batch in [(1024, 64), (16384, 3), (65536, 2)]:
        x = _rand_complex(rng, (batch, n))
        buf = torch.from_numpy(x).cuda()
        plan = fft.FftPlan([n], C2C, FWD, batch)
        assert plan.exec_raw(buf.data_ptr(), buf.data_ptr()) == fft.ACL_SUCCESS
        torch.cuda.synchronize()
        assert oracle.rel_l2(buf.cpu().numpy(), oracle.c2c(x, True)) <= oracle.tolerance(n)
        plan.close()


def test_many_rows_grid_loop(cuda):
    """More tiles than the launch grid: the kernel's tile loop covers the rest."""
    check([8], C2C, FWD, 300000, seed=11)
    check([64], R2C, INV, 100000, seed=12)


def test_exec_error_paths(cuda):
    import torch

    plan = fft.FftPlan([1024], C2C, FWD, 4)
    x = torch.zeros((4, 1024), dtype=torch.complex64, device="cuda")
    small = torch.zeros((3, 1024), dtype=torch.complex64, device="cuda")
    wrong = torch.zeros((4, 512), dtype=torch.complex64, device="cuda")
    real = torch.zeros((4, 1024), dtype=torch.float32, device="cuda")
    for a, b in [(small, x), (x, small), (wrong, x), (real, x)]:
        ta, tb = fft.AclTensor.from_torch(a), fft.AclTensor.from_torch(b)
        assert fft.asdFftExecC2C(plan.handle, ta, tb) == fft.ACL_ERROR_INVALID_PARAM
    # wrong exec kind for the plan type
    ta, tb = fft.AclTensor.from_torch(real), fft.AclTensor.from_torch(x)
    assert fft.asdFftExecR2C(plan.handle, ta, tb) == fft.ACL_ERROR_INVALID_PARAM
    # misaligned device pointer
    assert plan.exec_raw(x.data_ptr() + 4, x.data_ptr()) == fft.ACL_ERROR_INVALID_PARAM
    plan.close()
    # a plan that needs workspace refuses to run without it (fft_api.cpp:1008-1011)
    h = fft.asdFftCreate()
    assert fft.asdFftMakePlan1D(h, 65536, C2C, FWD, 1) == fft.ACL_SUCCESS
    st, ws = fft.asdFftGetWorkspaceSize(h)
    assert st == fft.ACL_SUCCESS and ws >= 65536 * 8
    y = torch.zeros((1, 65536), dtype=torch.complex64, device="cuda")
    assert fft.load_library().asdFftExecRaw(h, y.data_ptr(), y.data_ptr()) == fft.ACL_ERROR_INTERNAL_ERROR
    assert fft.asdFftDestroy(h) == fft.ACL_SUCCESS
    # lengths above the reference's limit (2^27) are refused at plan time
    h = fft.asdFftCreate()
    assert fft.asdFftMakePlan1D(h, 2 ** 27 + 1, C2C, FWD, 1) == fft.ACL_ERROR_INVALID_PARAM
    fft.asdFftDestroy(h)
    # a strided axis with a prime factor above 13 is not planned
    h = fft.asdFftCreate()
    assert fft.asdFftMakePlan2D(h, 17, 64, C2C, FWD, 1) == fft.ACL_ERROR_API_NOT_SUPPORT
    fft.asdFftDestroy(h)


def test_stream_and_sync(cuda):
    import torch

    s = torch.cuda.Stream()
    plan = fft.FftPlan([4096], C2C, INV, 8, stream=s)
    rng = np.random.default_rng(3)
    x = _rand_complex(rng, (8, 4096))
    xd = torch.from_numpy(x).cuda()
    y = torch.empty_like(xd)
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        plan(xd, y)
    assert fft.asdFftSynchronize(plan.handle) == fft.ACL_SUCCESS
    assert oracle.rel_l2(y.cpu().numpy(), oracle.c2c(x, False)) <= oracle.tolerance(4096)
    st, typ = fft.asdFftGetType(plan.handle)
    assert st == fft.ACL_SUCCESS and typ == C2C
    plan.close()


@pytest.mark.parametrize("typ,n", [(C2C, 1024), (C2C, 4096), (R2C, 4096), (R2C, 3000), (C2R, 3000), (C2R, 4096),
                                   (C2C, 512), (R2C, 1024), (C2R, 1024), (R2C, 256), (C2R, 128),
                                   (C2C, 16384), (R2C, 32768), (C2R, 32768)])
def test_pipelined_and_generic_kernels_agree(cuda, typ, n):
    """A 16-byte aligned source takes the TMA-pipelined row kernel; an 8-byte
    aligned one (offset by one element through the aclTensor offset) takes the
    generic tile kernel.  Both must give the oracle's result.  The 1024-point
    real transforms run the 512-point engine whose last radix-2 stage is
    warp-shuffle butterflies; 128..512-point engines use warp barriers; 16384
    points (C2C, and the packed half of 32768-point real transforms) run the
    single-buffered one-row-per-CTA engine."""
    import torch

    rng = np.random.default_rng(n + typ)
    batch = 37
    h = n // 2 + 1
    if typ == C2C:
        x = _rand_complex(rng, (batch, n))
        in_shape, out_shape, idt, odt = (batch, n), (batch, n), torch.complex64, torch.complex64
        ref = oracle.c2c(x, True)
        in_el = 8
    elif typ == R2C:
        x = rng.standard_normal((batch, n)).astype(np.float32)
        in_shape, out_shape, idt, odt = (batch, n), (batch, h), torch.float32, torch.complex64
        ref = oracle.r2c(x, True)
        in_el = 4
    else:
        x = (rng.standard_normal((batch, h)) + 1j * rng.standard_normal((batch, h))).astype(np.complex64)
        in_shape, out_shape, idt, odt = (batch, h), (batch, n), torch.complex64, torch.float32
        ref = oracle.c2r(x, n, True)
        in_el = 8
    plan = fft.FftPlan([n], typ, FWD, batch)
    outs = []
    for shift in (0, 8 // in_el):
        flat = torch.zeros(x.size + 4, dtype=idt, device="cuda")
        flat[shift:shift + x.size] = torch.from_numpy(x.reshape(-1)).cuda()
        out = torch.empty(out_shape, dtype=odt, device="cuda")
        dt = fft.ACL_COMPLEX64 if idt == torch.complex64 else fft.ACL_FLOAT
        a = fft.AclTensor(list(in_shape), dt, flat.data_ptr() + shift * in_el)
        b = fft.AclTensor.from_torch(out)
        ex = {C2C: fft.asdFftExecC2C, R2C: fft.asdFftExecR2C, C2R: fft.asdFftExecC2R}[typ]
        assert ex(plan.handle, a, b) == fft.ACL_SUCCESS
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
        assert oracle.rel_l2(outs[-1], ref) <= oracle.tolerance(n)
    assert np.max(np.abs(outs[0] - outs[1])) <= 1e-6 * np.max(np.abs(ref))
    assert fft.asdFftSynchronize(plan.handle) == fft.ACL_SUCCESS
    plan.close()


@pytest.mark.parametrize("n,batch", [(64, 33), (256, 16), (1000, 8), (4096, 4), (16384, 3), (65536, 2)])
@pytest.mark.parametrize("fwd", [FWD, INV])
def test_complex32_c2c(cuda, n, batch, fwd):
    """complex32 (FP16 pairs) in and out of a C2C plan, FP32 arithmetic: the
    reference's DftC32Kernel variant (ops/fft/c2c/dft/dft/kernel/dft_complex32.cpp).
    The result equals the FP32 path's output rounded to FP16 (to one FP16 ulp)
    and is within FP16 output rounding of the FP64 oracle."""
    import torch

    rng = np.random.default_rng(n + fwd)
    x = _rand_complex(rng, (batch, n)).astype(np.complex64)
    xh = np.stack([x.real, x.imag], axis=-1).astype(np.float16)     # [batch, n, 2]
    xd = torch.from_numpy(xh).cuda()
    yd = torch.full_like(xd, float("nan"))
    plan = fft.FftPlan([n], C2C, fwd, batch)
    a = fft.AclTensor([batch, n], fft.ACL_COMPLEX32, xd.data_ptr())
    b = fft.AclTensor([batch, n], fft.ACL_COMPLEX32, yd.data_ptr())
    assert fft.asdFftExecC2C(plan.handle, a, b) == fft.ACL_SUCCESS
    torch.cuda.synchronize()
    y = yd.cpu().numpy().astype(np.float64)
    got = y[..., 0] + 1j * y[..., 1]
    xin = xh.astype(np.float64)
    ref = oracle.c2c(xin[..., 0] + 1j * xin[..., 1], fwd == FWD)
    assert np.all(np.isfinite(got))
    assert oracle.rel_l2(got, ref) <= 1e-3, oracle.rel_l2(got, ref)
    # the FP32 path on the same (FP16-exact) input, rounded to FP16
    xc = torch.from_numpy((xin[..., 0] + 1j * xin[..., 1]).astype(np.complex64)).cuda()
    y32 = torch.empty_like(xc)
    plan(xc, y32)
    torch.cuda.synchronize()
    r = torch.view_as_real(y32).half().float().cpu().numpy()
    # one FP16 ulp, plus the FP32 paths' own rounding differences (absolute, at the
    # transform's scale), which can move a value near zero by more than its ulp
    ulp = np.abs(np.spacing(r.astype(np.float16)).astype(np.float64))
    assert np.all(np.abs(y - r) <= ulp + 1e-6 * np.log2(n) * np.abs(r).max())
    # in place
    assert fft.asdFftExecC2C(plan.handle, a, a) == fft.ACL_SUCCESS
    torch.cuda.synchronize()
    assert np.array_equal(xd.cpu().numpy(), yd.cpu().numpy())
    a.close()
    b.close()
    plan.close()


def test_complex32_refused_where_unsupported(cuda):
    import torch

    x = torch.zeros((4, 64, 64, 2), dtype=torch.float16, device="cuda")
    plan = fft.FftPlan([64, 64], C2C, FWD, 4)
    a = fft.AclTensor([4, 64, 64], fft.ACL_COMPLEX32, x.data_ptr())
    assert fft.asdFftExecC2C(plan.handle, a, a) == fft.ACL_ERROR_API_NOT_SUPPORT   # 2D
    a.close()
    plan.close()
    plan = fft.FftPlan([17], C2C, FWD, 4)  # Bluestein length
    a = fft.AclTensor([4, 17], fft.ACL_COMPLEX32, x.data_ptr())
    assert fft.asdFftExecC2C(plan.handle, a, a) == fft.ACL_ERROR_API_NOT_SUPPORT
    a.close()
    plan.close()


@pytest.mark.parametrize("n,batch", [(256, 64), (2048, 20), (65536, 6), (1024, 10)])
def test_tma_column_tiles_and_fallback_agree(cuda, n, batch):
    """A 16-byte aligned source of a strided axis takes the TMA column-tile
    kernel; an 8-byte aligned one the double-buffered element-copy kernel.
    Both give the oracle's result (vertical 1D; 65536 runs as two passes)."""
    import torch

    rng = np.random.default_rng(n + batch)
    x = _rand_complex(rng, (n, batch))
    plan = fft.FftPlan([n], C2C, FWD, batch, fft.ASCEND_FFT_VERTICAL)
    assert "TMA column tiles" in plan.describe(), plan.describe()
    ref = oracle.c2c(x.T, True).T
    outs = []
    for shift in (0, 1):
        flat = torch.zeros(x.size + 4, dtype=torch.complex64, device="cuda")
        flat[shift:shift + x.size] = torch.from_numpy(x.reshape(-1)).cuda()
        out = torch.empty((n, batch), dtype=torch.complex64, device="cuda")
        assert plan.exec_raw(flat.data_ptr() + 8 * shift, out.data_ptr()) == fft.ACL_SUCCESS
        torch.cuda.synchronize()
        assert fft.asdFftSynchronize(plan.handle) == fft.ACL_SUCCESS
        outs.append(out.cpu().numpy())
        assert oracle.rel_l2(outs[-1], ref) <= oracle.tolerance(n), shift
    assert np.max(np.abs(outs[0] - outs[1])) <= 1e-5 * np.max(np.abs(ref))
    plan.close()


def test_dependent_launches_back_to_back(cuda):
    """A chain of plans on one stream with no host synchronisation in between:
    every kernel is launched with programmatic stream serialization and must
    wait for the previous launch's results (and not overwrite what it still
    reads) before touching memory.  Each link reads the previous link's output."""
    import torch

    rng = np.random.default_rng(77)
    s = torch.cuda.Stream()
    n2, n1, rows = 2048, 4096, 96
    x = rng.standard_normal((rows, n1)).astype(np.float32)
    plans = [fft.FftPlan([n1], R2C, FWD, rows, stream=s), fft.FftPlan([n1], C2R, INV, rows, stream=s),
             fft.FftPlan([rows // 2, n1 * 2], C2C, FWD, 1, stream=s),
             fft.FftPlan([65536], C2C, INV, rows * n1 // 65536, stream=s),
             fft.FftPlan([n2], C2C, FWD, rows * n1 // n2, fft.ASCEND_FFT_VERTICAL, stream=s)]
    xd = torch.from_numpy(x).cuda()
    X = torch.empty((rows, n1 // 2 + 1), dtype=torch.complex64, device="cuda")
    y = torch.empty_like(xd)
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        for _ in range(3):  # repeated, so later launches overlap earlier ones' tails
            plans[0](xd, X)
            plans[1](X, y)
            z = torch.complex(y, torch.zeros_like(y)).reshape(rows // 2, n1 * 2)
            z1 = torch.empty_like(z)
            plans[2](z.reshape(1, rows // 2, n1 * 2), z1.reshape(1, rows // 2, n1 * 2))
            z2 = torch.empty_like(z1)
            plans[3](z1.reshape(-1, 65536), z2.reshape(-1, 65536))
            z3 = torch.empty_like(z2)
            plans[4](z2.reshape(n2, -1), z3.reshape(n2, -1))
    s.synchronize()
    for p in plans:
        assert fft.asdFftSynchronize(p.handle) == fft.ACL_SUCCESS
    X_ref = oracle.r2c(x, True)
    y_ref = oracle.c2r(X_ref, n1, False)
    z_ref = oracle.c2c(y_ref.reshape(1, rows // 2, n1 * 2).astype(np.complex128), True, ndim=2)
    z_ref = oracle.c2c(z_ref.reshape(-1, 65536), False)
    z_ref = oracle.c2c(z_ref.reshape(n2, -1).T, True).T
    assert oracle.rel_l2(z3.reshape(n2, -1).cpu().numpy(), z_ref) <= 5 * oracle.tolerance(65536)
    for p in plans:
        p.close()
