"""CPU: the kernel's index arithmetic (replayed by tests/stockham_model.py)
against the oracle, for the radix sets, multi-pass splits and R2C/C2R packing
the planner emits."""
import numpy as np
import pytest

import stockham_model as sm
from oracle import oracle


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 16, 20, 27, 30, 60, 64, 81, 96, 100, 128,
                               143, 210, 216, 245, 256, 343, 360, 1000, 1024, 1500, 2048, 3000, 4096])
@pytest.mark.parametrize("fwd", [True, False])
def test_smem_stockham(n, fwd):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = sm.smem_fft(x, fwd, sm.table(n, n, fwd), 1)
    assert oracle.rel_l2(y, oracle.c2c(x, fwd)) < 1e-12


@pytest.mark.parametrize("n,passes", [(64, [8, 8]), (96, [12, 8]), (1024, [32, 32]), (4096, [16, 16, 16]),
                                      (3000, [60, 50]), (32768, [256, 128])])
@pytest.mark.parametrize("fwd", [True, False])
def test_multipass_addressing(n, passes, fwd):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = sm.multipass(x, passes, fwd)
    assert oracle.rel_l2(y, oracle.c2c(x, fwd)) < 1e-12


@pytest.mark.parametrize("n", [2, 4, 6, 30, 64, 1000, 3000, 4096])
@pytest.mark.parametrize("fwd", [True, False])
def test_packed_real(n, fwd):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    assert oracle.rel_l2(sm.r2c_packed(x, fwd), oracle.r2c(x, fwd)) < 1e-12
    xh = rng.standard_normal(n // 2 + 1) + 1j * rng.standard_normal(n // 2 + 1)
    assert oracle.rel_l2(sm.c2r_packed(xh, n, fwd), oracle.c2r(xh, n, fwd)) < 1e-12


def test_reciprocal_modulo_exact():
    """fft_tile.cuh mod_ns: j mod ns = j - umulhi(j, ceil(2^32 / ns)) * ns for every stage
    product ns of 7-smooth lengths up to 32768 and every butterfly index j < 2^15."""
    import itertools

    ns_values = sorted({2 ** a * 3 ** b * 5 ** c * 7 ** d
                        for a, b, c, d in itertools.product(range(16), range(10), range(7), range(6))
                        if 1 < 2 ** a * 3 ** b * 5 ** c * 7 ** d <= 32768})
    j = np.arange(1 << 15, dtype=np.uint64)
    for ns in ns_values:
        m = np.uint64(((1 << 32) + ns - 1) // ns)
        q = (j * m) >> np.uint64(32)
        assert np.array_equal(j - q * np.uint64(ns), j % np.uint64(ns)), ns


@pytest.mark.parametrize("n,R", [(4096, 8), (3000, 5), (256, 8), (2048, 8), (4096, 16), (1000, 5)])
@pytest.mark.parametrize("fwd", [True, False])
def test_fused_c2r_first_stage(n, R, fwd):
    """Mirror-owned first stage of a C2R engine: every packed input Z[e] built once, as C2RPre would."""
    m = n // 2
    rng = np.random.default_rng(n + R)
    xh = rng.standard_normal(m + 1) + 1j * rng.standard_normal(m + 1)
    w = np.exp((-1 if fwd else 1) * 2j * np.pi * np.arange(m) / n)
    x0, xm = xh.copy(), xh[::-1].copy()
    x0[0] = x0[0].real
    xm[0] = xm[0].real  # X[m] seen by e = 0
    xm[m] = xm[m].real
    ref = (x0[:m] + np.conj(xm[:m])) + 1j * w * (x0[:m] - np.conj(xm[:m]))
    z = sm.fused_c2r_first_stage(xh, m, R, fwd)
    assert not np.isnan(z).any()
    assert np.allclose(z, ref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("n,R", [(4096, 8), (3000, 5), (256, 8), (2048, 8), (4096, 16), (1000, 5)])
@pytest.mark.parametrize("fwd", [True, False])
def test_fused_r2c_last_stage(n, R, fwd):
    """Mirror-owned last stage of an R2C engine: all m+1 bins written, equal to the R2C of the real input."""
    rng = np.random.default_rng(n * R)
    x = rng.standard_normal(n)
    Z = np.fft.fft(x[0::2] + 1j * x[1::2]) if fwd else np.fft.ifft(x[0::2] + 1j * x[1::2]) * (n // 2)
    X = sm.fused_r2c_last_stage(Z, R, fwd)
    assert not np.isnan(X).any()
    assert oracle.rel_l2(X, oracle.r2c(x, fwd)) < 1e-12


# TMA column-kernel instantiations (col_pipe.cu col_registry): N, threads per
# column, columns per tile, ping-pong work rows
COLUMN_ENGINES = [(64, 4, 16, False), (128, 8, 16, False), (256, 16, 16, False), (512, 32, 8, False),
                  (1024, 64, 4, False), (2048, 128, 4, True)]


def _pad(i):
    return i + (i >> 4)


@pytest.mark.parametrize("n,t,tb,pp", COLUMN_ENGINES)
def test_column_kernel_buffers_and_staged_stores(n, t, tb, pp):
    """col_pipe.cu: every shared-memory index of a column tile stays inside its
    buffer (staged [row][TB] tile, padded work rows, the third ping-pong buffer),
    the dynamic shared memory fits a CTA, and the staged contiguous-column
    store (TB = 16 variants) writes each element of each column exactly once."""
    # planner.cpp choose_cfg: the column-tile pitch (bank rule P mod 32/TB = 16/TB)
    p = _pad(n - 1) + 1
    m, want = 32 // tb, 16 // tb
    while p % m != want:
        p += 1
    col_buf = (tb * max(n, p) + 15) // 16 * 16
    bufs = 3 if pp else 2
    assert 128 + bufs * col_buf * 8 <= 227 * 1024
    assert n * tb <= col_buf  # staged tile, dense [row][TB]
    assert (tb - 1) * p + _pad(n - 1) < col_buf  # work rows (and ping-pong rows in the third buffer)
    if tb >= 16:
        threads = tb * t
        seen = np.zeros((tb, n), dtype=np.int64)
        for tid in range(threads):
            for c in range(tb):
                for e in range(tid, n, threads):
                    assert c * p + _pad(e) < col_buf
                    seen[c, e] += 1
        assert (seen == 1).all()
