"""Generate the golden FFT vectors in tests/golden/reference_vectors.npz.

The reference (AscendSiPBoost) ships no FFT tests, no golden vectors and no
known-answer tests, and its FFT kernels run only on an Ascend NPU.  Its
host-side coefficient generator does compile on a CPU, so the outputs here
come from the reference's own code: oracle/_ref/libsipref.so, built by
``make -C oracle REF=<reference tree>`` from core/fft/utils/rotate.cpp and the
wten tensor library, driven by oracle/ref_driver.cpp:

* ``dense``  — the single-factor transform matrix of the reference's generic
  core (rotate::OneRotateMatrix with factors {N}), for C2C, R2C and C2R in
  both directions; this pins sign, normalisation and half-spectrum packing;
* ``staged`` — the reference generic core's multi-factor C2C stage chain
  (merged factors, one matrix per stage, digit permutes);
* ``nd`` (reference_vectors_nd.npz) — 2D and 3D C2C, R2C and C2R built from
  the reference's single-factor matrices applied axis by axis in the order of
  the reference's multi-dimensional plans (core/fft/fft_api.cpp:527-602
  init2DSteps, 604-697 init3DSteps): R2C on the last axis first and then C2C on
  the leading axes (X before Y); C2R with C2C on the leading axes first and C2R
  on the last axis last; every step in the plan's direction.  The transposes
  between the steps are plain data movement (numpy); every product is the
  reference's own matrix.  This pins which axis is halved and the sign of
  every axis for the multi-dimensional types.

Inputs are seeded; every case stores its input, its output and its metadata.
Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402

DENSE_SIZES = [1, 2, 3, 4, 5, 7, 8, 12, 16, 17, 30, 31, 64, 100, 128, 210, 256, 343, 512, 1000, 1024]
BENCH_SIZES = [3000, 4096]          # the R2C/C2R round-trip workload lengths
STAGED_SIZES = [96, 360, 1024, 2048, 3000, 4096, 15000]
ND_SHAPES = [(4, 6), (5, 8), (7, 5), (16, 12), (3, 4, 6), (2, 5, 8), (6, 3, 7)]


def _along(x: np.ndarray, axis: int, fn) -> np.ndarray:
    """Apply a row transform fn ([rows, n] -> [rows, m]) along one axis of x."""
    moved = np.moveaxis(x, axis, -1)
    lead = moved.shape[:-1]
    y = fn(np.ascontiguousarray(moved.reshape(-1, moved.shape[-1])))
    return np.moveaxis(y.reshape(lead + (y.shape[-1],)), -1, axis)


def nd_reference(kind: str, x: np.ndarray, shape: tuple, forward: bool) -> np.ndarray:
    """Multi-dimensional transform from the reference's per-axis matrices, in
    the reference plans' step order.  x has a leading batch axis."""
    nd = len(shape)
    lead_axes = list(range(1, nd))  # X (and Y): the axes before the last
    if kind == "c2c":
        y = _along(x, -1, lambda r: oracle.ref_dense("c2c", r, shape[-1], forward))
        for ax in lead_axes:
            y = _along(y, ax, lambda r, n=shape[ax - 1]: oracle.ref_dense("c2c", r, n, forward))
        return y
    if kind == "r2c":
        y = _along(x, -1, lambda r: oracle.ref_dense("r2c", r, shape[-1], forward))
        for ax in lead_axes:
            y = _along(y, ax, lambda r, n=shape[ax - 1]: oracle.ref_dense("c2c", r, n, forward))
        return y
    y = x
    for ax in lead_axes:
        y = _along(y, ax, lambda r, n=shape[ax - 1]: oracle.ref_dense("c2c", r, n, forward))
    return _along(y, -1, lambda r: oracle.ref_dense("c2r", r, shape[-1], forward))


def make_nd(rng) -> None:
    arrays: dict[str, np.ndarray] = {}
    meta = []
    for shape in ND_SHAPES:
        batch = 2
        for forward in (True, False):
            d = "fwd" if forward else "inv"
            tag = "x".join(str(v) for v in shape)
            h = shape[-1] // 2 + 1
            xc = (rng.uniform(-1, 1, (batch,) + shape) + 1j * rng.uniform(-1, 1, (batch,) + shape)).astype(np.complex64)
            xr = rng.standard_normal((batch,) + shape).astype(np.float32)
            xh = (rng.standard_normal((batch,) + shape[:-1] + (h,)) +
                  1j * rng.standard_normal((batch,) + shape[:-1] + (h,))).astype(np.complex64)
            for kind, x in (("c2c", xc), ("r2c", xr), ("c2r", xh)):
                name = f"nd_{kind}_{d}_{tag}"
                arrays[name + "__in"] = x
                arrays[name + "__out"] = nd_reference(kind, x, shape, forward)
                meta.append((name, kind, shape, int(forward)))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors_nd.npz")
    shapes = np.zeros((len(meta), 3), dtype=np.int64)
    for i, m in enumerate(meta):
        shapes[i, :len(m[2])] = m[2]
    np.savez_compressed(out, _names=np.array([m[0] for m in meta]), _kinds=np.array([m[1] for m in meta]),
                        _shapes=shapes, _ndim=np.array([len(m[2]) for m in meta], dtype=np.int64),
                        _forward=np.array([m[3] for m in meta], dtype=np.int64), **arrays)
    print(f"wrote {len(meta)} cases to {out} ({os.path.getsize(out) / 1024:.0f} KiB)")


def main() -> None:
    if oracle.ref_lib() is None:
        raise SystemExit("build oracle/_ref first: make -C oracle REF=<reference tree>")
    rng = np.random.default_rng(20251203)
    arrays: dict[str, np.ndarray] = {}
    meta = []

    def add(name, kind, n, forward, x, y):
        arrays[name + "__in"] = x
        arrays[name + "__out"] = y
        meta.append((name, kind, n, int(forward)))

    for n in DENSE_SIZES + BENCH_SIZES:
        batch = 2 if n <= 256 else 1
        for forward in (True, False):
            d = "fwd" if forward else "inv"
            x = (rng.uniform(-1, 1, (batch, n)) + 1j * rng.uniform(-1, 1, (batch, n))).astype(np.complex64)
            if n <= 1024:
                add(f"dense_c2c_{d}_{n}", "c2c", n, forward, x, oracle.ref_dense("c2c", x, n, forward))
            xr = rng.standard_normal((batch, n)).astype(np.float32)
            add(f"dense_r2c_{d}_{n}", "r2c", n, forward, xr, oracle.ref_dense("r2c", xr, n, forward))
            h = n // 2 + 1
            xh = (rng.standard_normal((batch, h)) + 1j * rng.standard_normal((batch, h))).astype(np.complex64)
            add(f"dense_c2r_{d}_{n}", "c2r", n, forward, xh, oracle.ref_dense("c2r", xh, n, forward))

    for n in STAGED_SIZES:
        for forward in (True, False):
            d = "fwd" if forward else "inv"
            x = (rng.uniform(-1, 1, (1, n)) + 1j * rng.uniform(-1, 1, (1, n))).astype(np.complex64)
            add(f"staged_c2c_{d}_{n}", "c2c", n, forward, x, oracle.ref_c2c_staged(x, forward))

    names = np.array([m[0] for m in meta])
    kinds = np.array([m[1] for m in meta])
    sizes = np.array([m[2] for m in meta], dtype=np.int64)
    fwds = np.array([m[3] for m in meta], dtype=np.int64)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.npz")
    np.savez_compressed(out, _names=names, _kinds=kinds, _sizes=sizes, _forward=fwds, **arrays)
    print(f"wrote {len(meta)} cases to {out} ({os.path.getsize(out) / 1024:.0f} KiB)")
    make_nd(np.random.default_rng(20261203))


if __name__ == "__main__":
    main()
