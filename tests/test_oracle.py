"""CPU: the oracle against the reference's own outputs (golden vectors made by
oracle/_ref, i.e. the reference's compiled coefficient generator), against the
direct long-double DFT, and against itself across the conventions."""
import os

import numpy as np
import pytest

from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.npz")


def _cases():
    z = np.load(GOLDEN)
    for name, kind, n, fwd in zip(z["_names"], z["_kinds"], z["_sizes"], z["_forward"]):
        yield str(name), str(kind), int(n), bool(fwd)


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("name,kind,n,fwd", list(_cases()))
def test_oracle_matches_reference_golden(golden, name, kind, n, fwd):
    x = golden[name + "__in"]
    ref = golden[name + "__out"]
    if kind == "c2c":
        y = oracle.c2c(x, fwd)
    elif kind == "r2c":
        y = oracle.r2c(x, fwd)
    else:
        y = oracle.c2r(x, n, fwd)
    # the golden outputs are FP32 results of FP32 reference matrices: compare
    # at FP32-table accuracy
    assert oracle.rel_l2(y, ref) < 2e-6 * max(1.0, np.log2(max(n, 2))), name


GOLDEN_ND = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors_nd.npz")


def _nd_cases():
    z = np.load(GOLDEN_ND)
    for name, kind, shape, nd, fwd in zip(z["_names"], z["_kinds"], z["_shapes"], z["_ndim"], z["_forward"]):
        yield str(name), str(kind), tuple(int(v) for v in shape[:nd]), bool(fwd)


@pytest.mark.parametrize("name,kind,shape,fwd", list(_nd_cases()))
def test_oracle_matches_reference_golden_nd(name, kind, shape, fwd):
    """2D / 3D: the oracle's axis order (R2C on the last axis, C2R last) and
    per-axis signs against the reference's matrices applied in its plans' order."""
    z = np.load(GOLDEN_ND)
    x, ref = z[name + "__in"], z[name + "__out"]
    nd = len(shape)
    if kind == "c2c":
        y = oracle.c2c(x, fwd, ndim=nd)
    elif kind == "r2c":
        y = oracle.r2c(x, fwd, ndim=nd)
    else:
        y = oracle.c2r(x, shape[-1], fwd, ndim=nd)
    assert y.shape == ref.shape
    assert oracle.rel_l2(y, ref) < 2e-6 * max(1.0, np.log2(int(np.prod(shape)))), name


@pytest.mark.parametrize("n", [1, 2, 3, 5, 6, 8, 15, 16, 30, 49, 64, 97, 128, 210, 256])
@pytest.mark.parametrize("fwd", [True, False])
def test_oracle_vs_direct_dft(n, fwd):
    rng = np.random.default_rng(n)
    x = (rng.uniform(-1, 1, (3, n)) + 1j * rng.uniform(-1, 1, (3, n))).astype(np.complex64)
    assert oracle.rel_l2(oracle.c2c(x, fwd), oracle.direct_c2c(x, fwd)) < 1e-12
    xr = rng.standard_normal((3, n)).astype(np.float32)
    assert oracle.rel_l2(oracle.r2c(xr, fwd), oracle.direct_r2c(xr, fwd)) < 1e-12
    h = n // 2 + 1
    xh = (rng.standard_normal((3, h)) + 1j * rng.standard_normal((3, h))).astype(np.complex64)
    assert oracle.rel_l2(oracle.c2r(xh, n, fwd), oracle.direct_c2r(xh, n, fwd)) < 1e-12


def test_semantics_no_normalisation_and_round_trip():
    rng = np.random.default_rng(1)
    n = 3000
    x = rng.standard_normal((2, n))
    X = oracle.r2c(x, True)
    y = oracle.c2r(X, n, False) / n
    assert np.max(np.abs(y - x)) < 1e-12
    # C2R planned FORWARD is the time-reversed inverse
    yf = oracle.c2r(X, n, True) / n
    assert np.max(np.abs(yf - x[:, (-np.arange(n)) % n])) < 1e-12


def test_multidim_orders():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((2, 6, 10))
    X = oracle.r2c(x, True, ndim=2)
    assert np.allclose(X, np.fft.rfft2(x), atol=1e-12)
    y = oracle.c2r(X, 10, False, ndim=2)
    assert np.allclose(y / 60, x, atol=1e-12)
    z = rng.standard_normal((1, 4, 6, 8)) + 1j * rng.standard_normal((1, 4, 6, 8))
    assert np.allclose(oracle.c2c(z, True, ndim=3), np.fft.fftn(z, axes=(1, 2, 3)), atol=1e-10)


@pytest.mark.skipif(oracle.ref_lib() is None, reason="oracle/_ref not built")
@pytest.mark.parametrize("n", [4, 9, 60, 128])
def test_reference_matrices_live(n):
    """Re-run the reference's compiled generator (when built) against the oracle."""
    rng = np.random.default_rng(n + 7)
    for fwd in (True, False):
        x = (rng.uniform(-1, 1, (2, n)) + 1j * rng.uniform(-1, 1, (2, n))).astype(np.complex64)
        assert oracle.rel_l2(oracle.ref_dense("c2c", x, n, fwd), oracle.c2c(x, fwd)) < 1e-6
        assert oracle.rel_l2(oracle.ref_c2c_staged(x, fwd), oracle.c2c(x, fwd)) < 1e-6
        xr = rng.standard_normal((2, n)).astype(np.float32)
        assert oracle.rel_l2(oracle.ref_dense("r2c", xr, n, fwd), oracle.r2c(xr, fwd)) < 1e-6
        xh = (rng.standard_normal((2, n // 2 + 1)) + 1j * rng.standard_normal((2, n // 2 + 1))).astype(np.complex64)
        assert oracle.rel_l2(oracle.ref_dense("c2r", xh, n, fwd), oracle.c2r(xh, n, fwd)) < 1e-6


def test_istft_oracle_matches_torch_istft():
    """The ISTFT restatement (reference center / normalized / onesided /
    return_complex limits) equals torch.istft, whose semantics the reference
    ports, for even and odd n_fft and hop < n_fft."""
    import torch

    rng = np.random.default_rng(11)
    for n_fft, hop, frames, ch in [(64, 16, 10, 2), (400, 160, 7, 3), (255, 100, 5, 1), (1024, 256, 9, 2)]:
        x = rng.standard_normal((ch, n_fft, frames)) + 1j * rng.standard_normal((ch, n_fft, frames))
        w = np.hanning(n_fft) + 0.1
        a = oracle.istft(x, n_fft, hop, w)
        b = torch.istft(torch.from_numpy(x), n_fft, hop, n_fft, torch.from_numpy(w), center=True,
                        normalized=False, onesided=False, return_complex=True).numpy()
        assert a.shape == b.shape == (ch, n_fft + hop * (frames - 1) - 2 * (n_fft // 2))
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
