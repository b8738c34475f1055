"""GPU: the allocation-free Seed Check entry point.

wg_seed_check_noalloc serves callers that cannot call cudaMalloc — a process whose device memory
belongs to another allocator, or a latency-critical stream where cudaMalloc / cudaFree could
synchronize the device — by keeping its work lists in the library's fixed scratch array.  Here
it is called through the C ABI twice in a row (the second call must not see the first call's
leftovers in the shared array) and each result is compared with the engine entry point's
(wg_seed_check_device) on the same request: identical survivor sets, bit for bit.

This file is collected last on purpose, so a failure here cannot hide the rest of the suite.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _survivors(wg, out, n):
    got = np.frombuffer(out[:n].cpu().numpy().tobytes(), dtype=wg.CANDIDATE_DTYPE)
    return np.sort(got, order=["seed_index", "rz", "rx"])


def test_noalloc_matches_engine_two_calls(wg, engine):
    import torch

    cap = 4096
    requests = [
        # (seeds on device or None for the generator, gen_base, n_seeds, rect, max_height, preset)
        # all stay inside the entry point's limits (<= 4,096 regions per seed, ~1.7 % of the
        # regions survive the climate gates, well under the 1,048,576-entry survivor list)
        (None, 2, 8192, (-32, 32, -32, 32), -50, "NORMAL"),
        ([wg.to_signed(wg.splitmix64(7 + i)) for i in range(20000)], 0, 20000, (-20, 20, -20, 20), -50, "NORMAL"),
        # one region per seed: the engine takes its breadth-first one-region climate stage here,
        # the allocation-free entry point the ordinary climate kernel; the region of hunt.py's
        # reference hut (seed 1473884015873122059, region (-31, -34)) beside 4,095 other seeds
        ([1473884015873122059] + [wg.to_signed(wg.splitmix64(50 + i)) for i in range(4095)], 0, 4096,
         (-31, -30, -34, -33), -50, "NORMAL"),
        (None, 11, 4096, (-16, 16, -16, 16), 0, "LARGE_BIOMES"),
    ]
    counts = []
    for seeds, base, n, rect, mh, preset in requests:
        opts = wg.make_opts(preset=preset)
        d_seeds = torch.tensor(seeds, dtype=torch.int64, device="cuda") if seeds is not None else None
        ptr = d_seeds.data_ptr() if d_seeds is not None else None
        out_a = torch.zeros((cap, 4), dtype=torch.int64, device="cuda")
        out_b = torch.zeros((cap, 4), dtype=torch.int64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        n_a = wg.seed_check_noalloc(ptr, base, n, rect, mh, opts, out_a.data_ptr(), cap, stream)
        n_b, _ = engine.seed_check_device(ptr, base, n, rect, mh, opts, out_b.data_ptr(), cap, stream)
        assert n_a == n_b
        assert np.array_equal(_survivors(wg, out_a, n_a), _survivors(wg, out_b, n_b))
        counts.append(n_a)
    assert min(counts) > 0


def test_noalloc_limits(wg):
    import torch

    opts = wg.make_opts()
    out = torch.zeros((16, 4), dtype=torch.int64, device="cuda")
    with pytest.raises(wg.EngineError, match="status 4"):      # more than 65,536 seeds
        wg.seed_check_noalloc(None, 2, 65537, (-4, 5, -4, 5), -50, opts, out.data_ptr(), 16)
    with pytest.raises(wg.EngineError, match="status 4"):      # more than 4,096 regions per seed
        wg.seed_check_noalloc(None, 2, 10, (-33, 32, -32, 32), -50, opts, out.data_ptr(), 16)
    with pytest.raises(wg.EngineError, match="status 1"):      # empty rect
        wg.seed_check_noalloc(None, 2, 10, (0, 0, 0, 5), -50, opts, out.data_ptr(), 16)


def test_noalloc_full_list_then_normal_call(wg, engine):
    """A call whose climate survivors overflow the fixed list reports WG_ERR_CAPACITY (SINGLE_BIOME
    passes every region: 512 seeds x 4,096 regions = 2^21 survivors > 2^20), and the next call,
    which reuses the same array, is not disturbed by the overflow flag left in it."""
    import torch

    out = torch.zeros((4096, 4), dtype=torch.int64, device="cuda")
    single = wg.make_opts(preset="SINGLE_BIOME")
    with pytest.raises(wg.EngineError, match="status 4"):
        wg.seed_check_noalloc(None, 9, 512, (-32, 32, -32, 32), -50, single, out.data_ptr(), 4096)
    opts = wg.make_opts()
    out_b = torch.zeros((4096, 4), dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    n_a = wg.seed_check_noalloc(None, 2, 8192, (-32, 32, -32, 32), 0, opts, out.data_ptr(), 4096, stream)
    n_b, _ = engine.seed_check_device(None, 2, 8192, (-32, 32, -32, 32), 0, opts, out_b.data_ptr(), 4096, stream)
    assert n_a == n_b > 0
    assert np.array_equal(_survivors(wg, out, n_a), _survivors(wg, out_b, n_b))
