"""GPU: batched jobs (wg_seed_check_jobs) and the job server (wg_server_*).

Bar: bit-exact.  Every job's survivors, flattened into shared batches with other jobs of other
sizes, rects, floors and rules, must equal the same job run alone (wg_seed_check, itself pinned
to lysh) and, for small jobs, the C restatement in oracle/ on the same inputs.
"""
from __future__ import annotations

import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCAN_REFERENCE = 1473884015873122059   # hunt.py:86: chunk (-987, -1073) within the 40,000-block rect


def mixed_jobs(wg):
    rng = np.random.default_rng(7)
    jobs = []
    for k in range(36):
        n = int(rng.integers(1, 300))
        r = int(rng.integers(1, 9))
        job = {"rect": (-r, r + 1, -r + k % 3, r + 1 + k % 3), "max_height": int(rng.integers(-54, -44))}
        if k % 4 == 0:
            job["gen"] = (int(rng.integers(0, 1 << 62)), n)
        else:
            job["seeds"] = rng.integers(-(1 << 63), (1 << 63) - 1, n, dtype=np.int64)
        job["version"] = ("1.19.x~26.1", "26.2", "1.18.2")[k % 3] if k % 5 else "1.19.x~26.1"
        if k % 7 == 3:
            job["preset"] = "LARGE_BIOMES"
        jobs.append(job)
    # a relaxed floor, a multi-window rect holding the reference hut, a one-seed one-region job,
    # an explicit other salt and SINGLE_BIOME (every region passes the climate gates)
    jobs.append({"gen": (5, 3000), "rect": (-8, 8, -8, 8), "max_height": 100, "version": "26.2"})
    jobs.append({"seeds": [SCAN_REFERENCE], "rect": (-79, 79, -79, 79), "max_height": -50})
    jobs.append({"seeds": [0], "rect": (0, 1, 0, 1), "max_height": -50})
    jobs.append({"gen": (11, 500), "rect": (-4, 5, -4, 5), "max_height": -50, "salt": 10387312})
    jobs.append({"gen": (9, 300), "rect": (-4, 5, -4, 5), "max_height": 100, "preset": "SINGLE_BIOME"})
    return jobs


def alone(engine, job):
    kw = {k: v for k, v in job.items() if k in ("seeds", "gen", "rect", "max_height", "version", "preset", "salt")}
    return engine.seed_check(**kw).candidates


def test_jobs_equal_each_job_alone(engine, wg):
    jobs = mixed_jobs(wg)
    got, st = engine.seed_check_jobs(jobs)
    assert len(got) == len(jobs)
    total = 0
    for i, job in enumerate(jobs):
        want = alone(engine, job)
        assert np.array_equal(got[i], want), i
        total += len(want)
    assert st["accepted"] == total
    assert total >= 3
    ref = got[len(jobs) - 4]
    assert (-987, -1073) in {(int(c["chunk_x"]), int(c["chunk_z"])) for c in ref}
    assert st["scanned"] == sum(
        (len(j["seeds"]) if "seeds" in j else j["gen"][1]) * (j["rect"][1] - j["rect"][0]) * (j["rect"][3] - j["rect"][2])
        for j in jobs)


def test_jobs_vs_oracle(engine, wg, port, bind_mod):
    """Small uneven jobs against the C restatement (same seeds, rect, floor)."""
    jobs = wg.uneven_jobs(n_jobs=48, base=3, max_seeds=64, max_radius=6)
    got, _ = engine.seed_check_jobs(jobs)
    r = bind_mod.rules("1.19.x~26.1")
    for i, job in enumerate(jobs):
        want, _ = port.scan_seeds(r, job["max_height"], job["rect"], seeds=job["seeds"])
        assert np.array_equal(got[i], want), i


def test_uneven_jobs_sample(engine, wg):
    """The first 256 jobs of the uneven-jobs workload (1..4,096 seeds, radius 1..64)."""
    jobs = wg.uneven_jobs(n_jobs=256)
    got, st = engine.seed_check_jobs(jobs)
    rng = np.random.default_rng(1)
    for i in rng.choice(len(jobs), 12, replace=False):
        assert np.array_equal(got[i], alone(engine, jobs[i])), i
    assert st["accepted"] == sum(len(g) for g in got)


def test_device_queue_equals_host_loop(engine, wg):
    """The device work queue (one graph launch, slices taken off the queue on the device) and the
    host batch loop give every job the same survivors and the same funnel."""
    jobs = mixed_jobs(wg) + wg.uneven_jobs(n_jobs=64, base=5)
    engine.set_job_queue(True)
    got_q, st_q = engine.seed_check_jobs(jobs)
    engine.set_job_queue(False)
    try:
        got_h, st_h = engine.seed_check_jobs(jobs)
    finally:
        engine.set_job_queue(True)
    for i in range(len(jobs)):
        assert np.array_equal(got_q[i], got_h[i]), i
    for k in ("reject_hist", "tier_hist", "scanned", "accepted", "climate_survivors", "deep_candidates"):
        assert st_q[k] == st_h[k], k
    assert st_q["batches"] >= 1


def test_device_queue_overflow_retries(engine, wg, port, bind_mod):
    """SINGLE_BIOME jobs pass every region through the climate stage: the queue's slices overflow
    the work lists and are re-run smaller on the device; results still equal the oracle's."""
    jobs = [{"gen": (9 + k, 400), "rect": (-20, 20, -20, 20), "max_height": -50, "preset": "SINGLE_BIOME"}
            for k in range(3)]
    got, st = engine.seed_check_jobs(jobs)
    r = bind_mod.rules("1.19.x~26.1", "SINGLE_BIOME")
    for i, job in enumerate(jobs):
        want, _ = port.scan_seeds(r, -50, job["rect"], gen=job["gen"])
        assert np.array_equal(got[i], want), i


def test_tuner_picks_measured_settings(wg):
    """wg_engine_tune times each class's candidates on the device and keeps the fastest; a tuned
    engine's jobs equal the untuned engine's."""
    with wg.Engine(0) as eng:
        jobs = wg.uneven_jobs(n_jobs=96, base=11)
        before, _ = eng.seed_check_jobs(jobs)
        rep = eng.tune()
        assert len(rep["classes"]) == 4
        for c in rep["classes"]:
            ms = {x["window"]: x["ms"] for x in c["candidates"]}
            assert c["window"] in ms and ms[c["window"]] == min(ms.values()) and all(v > 0 for v in ms.values())
        assert rep["budget"] in [x["checks"] for x in rep["budget_candidates"]]
        after, _ = eng.seed_check_jobs(jobs)
        for i in range(len(jobs)):
            assert np.array_equal(before[i], after[i]), i


def test_jobs_errors(engine, wg):
    with pytest.raises(wg.EngineError):
        engine.seed_check_jobs([{"gen": (1, 10), "rect": (0, 0, 0, 1)}])
    with pytest.raises(wg.EngineError):
        engine.seed_check_jobs([{"gen": (1, 0), "rect": (0, 1, 0, 1)}])
    got, st = engine.seed_check_jobs([])
    assert got == [] and st["accepted"] == 0


def test_server_results_equal_alone_under_concurrent_arrivals(engine, wg):
    """A long job first, then jobs submitted from two threads at staggered times, so they arrive
    while others are on the device and join their batches: each result equals the job alone."""
    jobs = [{"gen": (2, 1 << 22), "rect": (-4, 5, -4, 5), "max_height": -50}] + mixed_jobs(wg)
    ids = [None] * len(jobs)
    with wg.Server(0) as srv:
        ids[0] = srv.submit(**jobs[0])

        def submit(part):
            for i in part:
                ids[i] = srv.submit(**jobs[i])
                time.sleep(0.002 * (i % 3))
        th = [threading.Thread(target=submit, args=(range(1 + p, len(jobs), 2),)) for p in (0, 1)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        statuses = [srv.wait(j, 120) for j in ids]
        results = [srv.take(j) for j in ids]
        st = srv.stats()
        with pytest.raises(wg.EngineError):   # taken results are released
            srv.take(ids[0])
    assert all(s["status"] == 0 and s["done"] for s in statuses)
    assert max(s["batch_jobs"] for s in statuses) > 1        # some batches held several jobs
    for i, job in enumerate(jobs):
        assert statuses[i]["found"] == len(results[i])
        assert statuses[i]["latency_ms"] >= statuses[i]["queue_ms"] >= 0.0
        assert np.array_equal(results[i], alone(engine, job)), i
    assert st["accepted"] == sum(len(r) for r in results)


def test_server_big_and_small_jobs_interleave(engine, wg):
    """A long job does not hold back short jobs submitted after it."""
    with wg.Server(0) as srv:
        big = srv.submit(gen=(2, 1 << 22), rect=(-4, 5, -4, 5), max_height=-50)
        time.sleep(0.01)
        small = [srv.submit(gen=(100 + k, 4), rect=(-1, 2, -1, 2), max_height=-50) for k in range(8)]
        s_small = [srv.wait(j, 120) for j in small]
        s_big = srv.wait(big, 120)
        res_big = srv.take(big)
        for j in small:
            srv.take(j)
    assert all(s["status"] == 0 for s in s_small + [s_big])
    assert max(s["latency_ms"] for s in s_small) < s_big["latency_ms"]
    assert np.array_equal(res_big, engine.seed_check(gen=(2, 1 << 22), rect=(-4, 5, -4, 5)).candidates)


def test_server_errors(wg):
    with wg.Server(0) as srv:
        with pytest.raises(wg.EngineError):
            srv.submit(gen=(1, 0), rect=(0, 1, 0, 1))
        with pytest.raises(wg.EngineError):
            srv.submit(gen=(1, 5), rect=(3, 3, 0, 1))
        with pytest.raises(wg.EngineError):
            srv.poll(12345)
        j = srv.submit(gen=(1, 5), rect=(0, 1, 0, 1))
        assert srv.wait(j, 60)["status"] == 0
    small = wg.Server(0, max_queued_seeds=10)
    try:
        with pytest.raises(wg.EngineError, match="status 4"):
            small.submit(gen=(1, 11), rect=(0, 1, 0, 1))
    finally:
        small.close()
