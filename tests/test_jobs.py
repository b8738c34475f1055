"""CPU: the synthetic job streams (uneven batched jobs, Poisson serving requests) follow their
stated derivation, and the vectorised seed generator equals the scalar splitmix64 stream."""
from __future__ import annotations

import math

import numpy as np


def test_splitmix64_array_equals_scalar(wg):
    for base in (0, 2, 3, (1 << 64) - 3):
        got = wg.splitmix64_array(base, 9).view(np.uint64).tolist()
        assert got == [wg.splitmix64((base + i) & 0xFFFFFFFFFFFFFFFF) for i in range(9)]


def test_uneven_jobs_derivation(wg):
    jobs = wg.uneven_jobs(n_jobs=200)
    k = 0
    for job in jobs:
        x = [wg.splitmix64(3 + k + i) for i in range(4)]
        k += 4
        n = int(4097 ** ((x[0] >> 11) / 2.0 ** 53))
        r = int(65 ** ((x[1] >> 11) / 2.0 ** 53))
        assert len(job["seeds"]) == n and 1 <= n <= 4096
        assert job["rect"] == (-r, r + 1, -r, r + 1) and 1 <= r <= 64
        assert job["max_height"] == -50 - x[2] % 5
        assert job["mode"] == ("or_lower" if x[3] & 1 else "exactly")
        assert job["seeds"].view(np.uint64).tolist() == [wg.splitmix64(3 + k + i) for i in range(n)]
        k += n


def test_uneven_jobs_distribution(wg):
    jobs = wg.uneven_jobs(n_jobs=4000)
    n = np.array([len(j["seeds"]) for j in jobs])
    r = np.array([j["rect"][1] - j["rect"][0] for j in jobs]) // 2
    # log-uniform: about half of the jobs below the geometric midpoint
    assert 0.45 < np.mean(n < 64) < 0.55
    assert 0.45 < np.mean(r < 8) < 0.55
    assert set(j["max_height"] for j in jobs) == {-50, -51, -52, -53, -54}


def test_serving_requests(wg):
    reqs = wg.serving_requests(3000, rate_per_s=50.0)
    t = np.array([q["t"] for q in reqs])
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert np.all(gaps > 0)
    assert abs(gaps.mean() * 50.0 - 1.0) < 0.06          # exponential gaps of mean 1 / rate
    assert abs(np.median(gaps) * 50.0 - math.log(2)) < 0.06
    n = np.array([q["gen"][1] for q in reqs])
    assert n.min() >= 1 and n.max() <= 10 ** 6
    assert all(1 <= (q["rect"][1] - q["rect"][0]) // 2 <= 32 for q in reqs)
