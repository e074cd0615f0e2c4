"""CPU: the tensor-core FFT kernel's arithmetic and indexing, without a GPU.

* tc_desc.cuh's tcgen05 descriptors against CUTLASS's UMMA descriptor unions
  (host build with nvcc; skipped when no CUTLASS header tree is installed);
* every shared-memory / tensor-memory index of tc_fft_kernel inside its region;
* the numpy replay of the kernel (tests/tc_model.py) against the oracle, per
  precision form, within the FP32 tolerance 1e-6 * log2(N).
"""
import importlib.util
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import oracle

import tc_model

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _cutlass_include():
    for pkg, sub in (("flashinfer", ("data", "cutlass", "include")), ("tilelang", ("3rdparty", "cutlass", "include"))):
        spec = importlib.util.find_spec(pkg)
        if spec is None or not spec.submodule_search_locations:
            continue
        for base in spec.submodule_search_locations:
            inc = os.path.join(base, *sub)
            if os.path.exists(os.path.join(inc, "cute", "arch", "mma_sm100_desc.hpp")):
                return inc
    return None


NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not os.path.exists(NVCC) or _cutlass_include() is None, reason="nvcc or CUTLASS headers absent")
def test_descriptors_match_cutlass(tmp_path):
    exe = tmp_path / "tc_desc_check"
    src = os.path.join(ROOT, "tests", "host", "tc_desc_check.cu")
    subprocess.check_call([NVCC, "-std=c++17", "-Wno-deprecated-gpu-targets", "-I", _cutlass_include(),
                           "-I", os.path.join(ROOT, "sip_b200", "csrc"), "-o", str(exe), src])
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout


@pytest.mark.parametrize("n", sorted(tc_model.CONFIGS))
def test_kernel_indices_in_bounds(n):
    tc_model.check_bounds(n)


@pytest.mark.parametrize("n", sorted(tc_model.ROWS_CONFIGS))
def test_row_pipeline_indices_in_bounds(n):
    tc_model.check_rows_bounds(n)


@pytest.mark.parametrize("n", sorted(tc_model.ROWS_CONFIGS))
@pytest.mark.parametrize("fmt", [0, 1], ids=["fp16x3", "bf16x3"])
@pytest.mark.parametrize("forward", [True, False], ids=["fwd", "inv"])
def test_row_pipeline_model_accuracy(n, fmt, forward):
    rng = np.random.default_rng(3 * n + fmt + int(forward))
    TB = tc_model.ROWS_CONFIGS[n][2]
    x = (rng.uniform(-1, 1, (2 * TB + 1, n)) + 1j * rng.uniform(-1, 1, (2 * TB + 1, n))).astype(np.complex64)
    err = oracle.rel_l2(tc_model.tc_fft_rows(x, forward, fmt), oracle.c2c(x, forward))
    assert err <= 1e-6 * np.log2(n), err
    if fmt == 0:
        assert err <= 2e-7


@pytest.mark.parametrize("n", sorted(tc_model.CONFIGS))
@pytest.mark.parametrize("fmt", [0, 1], ids=["fp16x3", "bf16x3"])
@pytest.mark.parametrize("forward", [True, False], ids=["fwd", "inv"])
def test_model_accuracy(n, fmt, forward):
    rng = np.random.default_rng(n + 7 * fmt + int(forward))
    TB = tc_model.CONFIGS[n][2]
    rows = 2 * TB + 1  # one partial tile
    x = (rng.uniform(-1, 1, (rows, n)) + 1j * rng.uniform(-1, 1, (rows, n))).astype(np.complex64)
    ref = oracle.c2c(x, forward)
    err = oracle.rel_l2(tc_model.tc_fft(x, forward, fmt), ref)
    tol = 1e-6 * np.log2(n)
    assert err <= tol, (err, tol)
    if fmt == 0:
        assert err <= 2e-7  # the FP16 three-product form is as accurate as FP32


def test_model_fp16_scaling_handles_large_and_small_ranges():
    """The per-tile power-of-two scale keeps FP16 operands in range for tiny and huge inputs."""
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((4, 1024)) + 1j * rng.standard_normal((4, 1024))).astype(np.complex64)
    for scale in (1e-6, 1e6):
        xs = (x * scale).astype(np.complex64)
        err = oracle.rel_l2(tc_model.tc_fft(xs, True, 0), oracle.c2c(xs, True))
        assert err <= 2e-7, (scale, err)
