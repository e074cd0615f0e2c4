"""GPU: the largest transforms the plan API accepts (N = 2^27, the reference's
limit, fft_api.cpp:61,771) and the largest Bluestein convolution, checked by
size-independent properties rather than a full FP64 oracle: the transform of
an impulse at p is exp(-+2 pi i j p / N) at every bin j (checked on a seeded
sample of bins), and Parseval's identity holds for a random input.

Bar: relative L2 error <= 1e-6 * log2(N) over the sampled bins (impulse) and
relative energy error <= 1e-6 * log2(N) (random input)."""
import numpy as np
import pytest

from oracle import oracle
from sip_b200 import fft

pytestmark = pytest.mark.gpu

C2C, FWD, INV = fft.ASCEND_FFT_C2C, fft.ASCEND_FFT_FORWARD, fft.ASCEND_FFT_INVERSE


def _impulse_check(n, direction, p, samples=200000):
    import torch

    plan = fft.FftPlan([n], C2C, direction, 1)
    try:
        x = torch.zeros((1, n), dtype=torch.complex64, device="cuda")
        x[0, p] = 1.0
        y = torch.empty_like(x)
        plan(x, y)
        torch.cuda.synchronize()
        assert fft.asdFftSynchronize(plan.handle) == fft.ACL_SUCCESS
        rng = np.random.default_rng(n % 1000003)
        j = np.unique(np.concatenate([rng.integers(0, n, samples), [0, 1, n // 2, n - 1]]))
        got = y[0, torch.from_numpy(j).cuda()].cpu().numpy().astype(np.complex128)
        sign = -1.0 if direction == FWD else 1.0
        ref = np.exp(sign * 2j * np.pi * ((j.astype(np.int64) * p) % n) / n)
        err = oracle.rel_l2(got, ref)
        assert err <= oracle.tolerance(n), (n, err, float(np.max(np.abs(got - ref))))
        # Parseval on a random input (energy relative error)
        g = torch.Generator(device="cuda").manual_seed(5)
        x = torch.complex(torch.rand((1, n), device="cuda", generator=g) - 0.5,
                          torch.rand((1, n), device="cuda", generator=g) - 0.5)
        plan(x, y)
        torch.cuda.synchronize()
        ex = float((x.abs().double() ** 2).sum())
        ey = float((y.abs().double() ** 2).sum()) / n
        assert abs(ey - ex) / ex <= oracle.tolerance(n), (n, ex, ey)
    finally:
        plan.close()


@pytest.mark.parametrize("direction", [FWD, INV])
def test_c2c_largest_power_of_two(cuda, direction):
    """N = 2^27: three multi-pass Stockham passes."""
    _impulse_check(2 ** 27, direction, 12345)


def test_c2c_largest_bluestein(cuda):
    """N = 199 * 2^19 (a prime factor above 13): Bluestein with a 2^28-point
    multi-pass convolution, the largest the planner builds."""
    _impulse_check(199 * 2 ** 19, FWD, 777)
