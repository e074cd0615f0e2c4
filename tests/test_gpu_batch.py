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
        assert l["type"] == "c2c" and l["precision"] == "fp32" and l["gpu"]
        assert int(np.prod(l["radices"])) == l["n"]
    assert fft.tune_cache_load(path) >= 3
    plan, x, outs = _run(groups, fft.ASCEND_FFT_FORWARD, tune_cache=path)
    _check(plan, x, outs[0], True)
    plan.close()
