"""GPU: uneven batches in one persistent (graph-captured) launch, and the
autotuner cache, against the FP64 oracle."""
import json
import os

import numpy as np
import pytest

from oracle import oracle
from sip_b200 import fft, workloads

pytestmark = pytest.mark.gpu


def _run(groups, direction, use_graph=True, tune_cache=None, seed=0, reps=1):
    import torch

    rng = np.random.default_rng(seed)
    plan = fft.BatchPlan(groups, direction, tune_cache)
    x = (rng.uniform(-1, 1, plan.total) + 1j * rng.uniform(-1, 1, plan.total)).astype(np.complex64)
    xd = torch.from_numpy(x).cuda()
    outs = []
    for _ in range(reps):
        yd = torch.zeros_like(xd)
        plan(xd, yd, use_graph=use_graph)
        torch.cuda.synchronize()
        outs.append(yd.cpu().numpy())
    return plan, x, outs


def _check(plan, x, y, forward):
    for (n, b), off in zip(plan.groups, plan.offsets):
        xs = x[off:off + n * b].reshape(b, n)
        ys = y[off:off + n * b].reshape(b, n)
        err = oracle.rel_l2(ys, oracle.c2c(xs, forward))
        assert err <= oracle.tolerance(n), (n, b, err)


@pytest.mark.parametrize("use_graph", [False, True])
@pytest.mark.parametrize("direction", [fft.ASCEND_FFT_FORWARD, fft.ASCEND_FFT_INVERSE])
def test_uneven_small(cuda, use_graph, direction):
    groups = [(64, 37), (100, 5), (1024, 9), (1500, 3), (4096, 2), (17, 11), (16384, 1), (32768, 2),
              (3 * 2 ** 13, 1), (8, 400)]
    plan, x, outs = _run(groups, direction, use_graph, reps=2)
    _check(plan, x, outs[0], direction == fft.ASCEND_FFT_FORWARD)
    # graph replay and re-execution give identical results
    assert np.array_equal(outs[0], outs[1])
    assert fft.asdFftSynchronize  # API presence
    plan.close()


@pytest.mark.parametrize("direction", [fft.ASCEND_FFT_FORWARD, fft.ASCEND_FFT_INVERSE])
def test_compact_and_full_radix_kernels(cuda, direction):
    """Lengths whose radices fit 2..10 (16 and 12 split) run on the compact batch
    kernel (three CTAs per SM); a length with a factor 11 or 13 selects the kernel
    with every radix.  Both against the oracle, multi-pass lengths included."""
    fwd = direction == fft.ASCEND_FFT_FORWARD
    # 17 and 1021 are Bluestein lengths: power-of-two convolutions, radix 16 split into 4 x 4
    compact = [(17, 11), (48, 7), (144, 5), (240, 3), (1021, 3), (4096, 2), (3 * 2 ** 12, 2), (52920, 1),
               (65536, 1)]
    plan, x, outs = _run(compact, direction, seed=5)
    assert "kernel=compact" in plan.describe(), plan.describe()
    _check(plan, x, outs[0], fwd)
    plan.close()
    full = compact[:3] + [(11 * 64, 4), (13 * 13 * 16, 2)]
    plan, x, outs = _run(full, direction, seed=6)
    assert "kernel=every radix" in plan.describe(), plan.describe()
    _check(plan, x, outs[0], fwd)
    plan.close()


def test_uneven_workload_subset(cuda):
    """A slice of the seeded 20 000-transform set (lengths 64..65536, Zipf batches)."""
    groups = workloads.uneven_batch_set(total=2000, seed=7)
    plan, x, outs = _run(groups, fft.ASCEND_FFT_FORWARD)
    _check(plan, x, outs[0], True)
    plan.close()


def test_autotune_cache_round_trip(cuda, tmp_path):
    path = str(tmp_path / "tune.jsonl")
    groups = [(1500, 64), (2048, 64), (105, 64)]
    assert fft.autotune(groups, fft.ASCEND_FFT_FORWARD, path) == fft.ACL_SUCCESS
    lines = [json.loads(l) for l in open(path)]
    assert {l["n"] for l in lines} >= {1500, 2048, 105}
    for l in lines:
        assert l["type"] == "c2c" and l["precision"] in ("fp32", "fp16x3", "bf16x3") and l["gpu"]
        # a per-length winner that did not speed up the launch of all groups together
        # is recorded without a tile choice (empty radices: the planner's defaults)
        if l["radices"]:
            assert int(np.prod(l["radices"])) == l["n"]
            assert l["row_threads"] in (128, 256)
        else:
            assert l["row_threads"] == 0
    # 2048 has tensor-core stages: the whole plan was timed in every arithmetic
    assert [l for l in lines if l["n"] == 2048][0]["plan_us"] > 0
    assert fft.tune_cache_load(path) >= 3
    plan, x, outs = _run(groups, fft.ASCEND_FFT_FORWARD, tune_cache=path)
    _check(plan, x, outs[0], True)
    plan.close()


def test_precision_auto_follows_the_tuned_arithmetic(cuda, tmp_path):
    """Precision mode 3: each length runs in the arithmetic its cache entry
    names (here a tensor-core form for 2048 and FP32 for 1024), with parity."""
    import torch

    path = str(tmp_path / "tune.jsonl")
    gpu = torch.cuda.get_device_name(0)
    with open(path, "w") as f:
        f.write(json.dumps({"gpu": gpu, "type": "c2c", "precision": "fp16x3", "n": 2048, "radices": [16, 16, 8],
                            "maxe": 16, "row_threads": 256, "us": 1.0, "plan_us": 1.0}) + "\n")
        f.write(json.dumps({"gpu": gpu, "type": "c2c", "precision": "fp32", "n": 1024, "radices": [16, 16, 4],
                            "maxe": 16, "row_threads": 256, "us": 1.0, "plan_us": 1.0}) + "\n")
    assert fft.tune_cache_load(path) == 2
    rng = np.random.default_rng(9)
    for n, want_tc in ((2048, True), (1024, False)):
        x = (rng.uniform(-1, 1, (24, n)) + 1j * rng.uniform(-1, 1, (24, n))).astype(np.complex64)
        plan = fft.FftPlan([n], fft.ASCEND_FFT_C2C, fft.ASCEND_FFT_FORWARD, 24, precision=fft.PRECISION_AUTO)
        assert ("tensor-core" in plan.describe()) == want_tc, plan.describe()
        xd = torch.from_numpy(x).cuda()
        y = torch.empty_like(xd)
        plan(xd, y)
        torch.cuda.synchronize()
        assert oracle.rel_l2(y.cpu().numpy(), oracle.c2c(x, True)) <= oracle.tolerance(n)
        plan.close()
