"""FP64 CPU oracle for the FFT path — test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module, and only as the checker: the shipped
library never routes through it.

It restates the reference's FFT semantics (AscendSiPBoost ``core/fft``):

* direction sets the exponent sign for C2C, R2C and C2R alike —
  FORWARD ``exp(-2*pi*i*j*k/N)``, INVERSE ``exp(+2*pi*i*j*k/N)``
  (core/fft/fftcore/dft_core.cpp:88-97, dft_r2c_core.cpp:98-104,
  dft_c2r_core.cpp:98-110, core/fft/utils/rotate.cpp:80-111);
* no normalisation in either direction;
* R2C keeps bins ``0..N//2`` of the last axis; C2R reads ``N//2+1`` bins and
  uses the Hermitian extension, ignoring the imaginary part of bin 0 and of
  bin N/2 for even N (dft_c2r_core.cpp:98-110, fft_core_any.cpp:319-381);
* multi-dimensional R2C runs R2C on the last axis and then C2C on the others;
  C2R runs C2C on the leading axes first and C2R on the last axis last
  (core/fft/fft_api.cpp:527-602 init2DSteps, 604-697 init3DSteps).

Large transforms use numpy's pocketfft in complex128; the direct long-double
DFT in ``dft_oracle.c`` cross-checks it.  Parity is pinned against the
reference's own coefficient generator compiled into ``oracle/_ref`` (see
``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

FORWARD = True
INVERSE = False


def _c2c_axis(x: np.ndarray, forward: bool, axis: int) -> np.ndarray:
    x = np.asarray(x, dtype=np.complex128)
    n = x.shape[axis]
    if forward:
        return np.fft.fft(x, axis=axis)
    return np.fft.ifft(x, axis=axis) * n


def c2c(x: np.ndarray, forward: bool, ndim: int = 1) -> np.ndarray:
    """Unnormalised C2C over the last ``ndim`` axes (complex128 result)."""
    y = np.asarray(x, dtype=np.complex128)
    for ax in range(-ndim, 0):
        y = _c2c_axis(y, forward, ax)
    return y


def r2c(x: np.ndarray, forward: bool, ndim: int = 1) -> np.ndarray:
    """R2C over the last ``ndim`` axes: half spectrum on the last axis."""
    y = np.fft.rfft(np.asarray(x, dtype=np.float64), axis=-1)
    if not forward:
        y = np.conj(y)
    for ax in range(-ndim, -1):
        y = _c2c_axis(y, forward, ax)
    return y


def c2r(x: np.ndarray, n_last: int, forward: bool, ndim: int = 1) -> np.ndarray:
    """C2R over the last ``ndim`` axes; ``n_last`` is the real length."""
    y = np.asarray(x, dtype=np.complex128)
    for ax in range(-ndim, -1):
        y = _c2c_axis(y, forward, ax)
    out = np.fft.irfft(y, n=n_last, axis=-1) * n_last
    if forward:
        idx = (-np.arange(n_last)) % n_last
        out = out[..., idx]
    return out


def rel_l2(got: np.ndarray, ref: np.ndarray) -> float:
    got = np.asarray(got, dtype=np.complex128 if np.iscomplexobj(got) else np.float64)
    num = np.linalg.norm((got - ref).ravel())
    den = np.linalg.norm(np.asarray(ref).ravel())
    return float(num / den) if den > 0 else float(num)


def max_abs(got: np.ndarray, ref: np.ndarray) -> float:
    return float(np.max(np.abs(np.asarray(got) - np.asarray(ref)))) if np.size(ref) else 0.0


def tolerance(n_total: int) -> float:
    """The accuracy gate of the path: relative L2 <= 1e-6 * log2(N)."""
    return 1e-6 * max(1.0, float(np.log2(max(2, n_total))))


# --- direct long-double DFT (dft_oracle.c) ------------------------------------------------------

_lib = None


def _direct_lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "libdft_oracle.so")
        if not os.path.exists(path):
            build_c_oracle()
        lib = ctypes.CDLL(path)
        for name in ("oracle_dft_c2c", "oracle_dft_r2c", "oracle_dft_c2r"):
            fn = getattr(lib, name)
            fn.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
            fn.restype = ctypes.c_int
        _lib = lib
    return _lib


def build_c_oracle() -> str:
    """Compile dft_oracle.c into oracle/libdft_oracle.so (plain gcc)."""
    import subprocess

    out = os.path.join(_HERE, "libdft_oracle.so")
    src = os.path.join(_HERE, "dft_oracle.c")
    if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-o", out, src, "-lm"])
    return out


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def direct_c2c(x: np.ndarray, forward: bool) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex64)
    n = x.shape[-1]
    batch = x.size // n if n else 0
    out = np.empty(x.shape, dtype=np.complex128)
    _direct_lib().oracle_dft_c2c(int(forward), n, batch, _ptr(x), _ptr(out))
    return out


def direct_r2c(x: np.ndarray, forward: bool) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    n = x.shape[-1]
    batch = x.size // n if n else 0
    out = np.empty(x.shape[:-1] + (n // 2 + 1,), dtype=np.complex128)
    _direct_lib().oracle_dft_r2c(int(forward), n, batch, _ptr(x), _ptr(out))
    return out


def direct_c2r(x: np.ndarray, n: int, forward: bool) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex64)
    batch = x.size // (n // 2 + 1) if x.size else 0
    out = np.empty(x.shape[:-1] + (n,), dtype=np.float64)
    _direct_lib().oracle_dft_c2r(int(forward), n, batch, _ptr(x), _ptr(out))
    return out


# --- reference coefficient generator (oracle/_ref, built from the reference's sources) ---------

_ref = None


def ref_lib():
    """The reference's own rotate.cpp + wten compiled by oracle/Makefile, or None."""
    global _ref
    if _ref is None:
        path = os.path.join(_HERE, "_ref", "libsipref.so")
        if not os.path.exists(path):
            return None
        lib = ctypes.CDLL(path)
        lib.sipref_dense.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
                                     ctypes.c_void_p, ctypes.c_void_p]
        lib.sipref_c2c_staged.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
                                          ctypes.c_void_p, ctypes.c_void_p]
        lib.sipref_factors.argtypes = [ctypes.c_int64, ctypes.c_void_p]
        _ref = lib
    return _ref


def ref_dense(mode: str, x: np.ndarray, n: int, forward: bool) -> np.ndarray:
    """Apply the reference's single-factor matrix (mode 'c2c' | 'r2c' | 'c2r') row by row."""
    lib = ref_lib()
    if lib is None:
        raise RuntimeError("oracle/_ref/libsipref.so is not built")
    m = {"c2c": 0, "r2c": 1, "c2r": 2}[mode]
    if m == 0:
        x = np.ascontiguousarray(x, dtype=np.complex64)
        out = np.empty(x.shape, np.complex64)
    elif m == 1:
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.empty(x.shape[:-1] + (n // 2 + 1,), np.complex64)
    else:
        x = np.ascontiguousarray(x, dtype=np.complex64)
        out = np.empty(x.shape[:-1] + (n,), np.float32)
    batch = out.size // out.shape[-1]
    lib.sipref_dense(m, int(forward), n, batch, _ptr(x), _ptr(out))
    return out


def ref_c2c_staged(x: np.ndarray, forward: bool) -> np.ndarray:
    """The reference generic core's multi-factor C2C stage chain on the CPU."""
    lib = ref_lib()
    if lib is None:
        raise RuntimeError("oracle/_ref/libsipref.so is not built")
    x = np.ascontiguousarray(x, dtype=np.complex64)
    n = x.shape[-1]
    out = np.empty_like(x)
    lib.sipref_c2c_staged(int(forward), n, x.size // n, _ptr(x), _ptr(out))
    return out


def istft(x: np.ndarray, n_fft: int, hop: int, window: np.ndarray) -> np.ndarray:
    """Inverse STFT as the reference computes it (center=True, normalized=False,
    onesided=False, return_complex=True, length=None: the only values its
    checks let through, core/fft/istft.cpp:300-390).

    x: complex [channel, n_fft, n_frames] (frequency-major, as the input tensor);
    window: real [n_fft].  Steps (core/fft/fftcore/fft_core_istft_any.cpp:292-378):
    frames = IFFT_nfft(x[c, :, f]) / n_fft; y = overlap-add(frames * window, hop);
    envelope = overlap-add(window^2, hop); out = (y / envelope)[n_fft/2 : L - n_fft/2]
    with L = n_fft + hop * (n_frames - 1).
    """
    x = np.asarray(x, np.complex128)
    channel, nf, n_frames = x.shape
    assert nf == n_fft
    w = np.asarray(window, np.float64)
    frames = np.fft.ifft(x, axis=1)  # numpy ifft divides by n_fft: the BY_N normalisation
    L = n_fft + hop * (n_frames - 1)
    y = np.zeros((channel, L), np.complex128)
    env = np.zeros(L)
    for f in range(n_frames):
        y[:, f * hop:f * hop + n_fft] += frames[:, :, f] * w
        env[f * hop:f * hop + n_fft] += w * w
    start, end = n_fft // 2, L - n_fft // 2
    return (y / env)[:, start:end]
