"""GPU: failure isolation of the job server, with faults made on the host.

No fault reaches the GPU: a batch is made to fail by the server's host-side injection hook
(wg_server_config.fail_job: every batch holding that job fails before its kernels launch), the
seed arena is capped below a job's size, and the server is closed with jobs pending.  In each case
the other jobs must finish with the results they get alone (wg_seed_check, itself pinned to lysh).
"""
from __future__ import annotations

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCAN_REFERENCE = 1473884015873122059


def jobs_mix():
    return [{"gen": (2, 5000), "rect": (-4, 5, -4, 5), "max_height": 100},
            {"seeds": [SCAN_REFERENCE], "rect": (-79, 79, -79, 79), "max_height": -50},
            {"gen": (7, 3000), "rect": (-6, 6, -6, 6), "max_height": 0, "version": "26.2"},
            {"gen": (9, 800), "rect": (-3, 3, -3, 3), "max_height": 100},
            {"gen": (13, 20000), "rect": (-2, 3, -2, 3), "max_height": 100}]


def alone(engine, job):
    kw = {k: v for k, v in job.items() if k in ("seeds", "gen", "rect", "max_height", "version", "preset", "salt")}
    return engine.seed_check(**kw).candidates


def test_failed_batch_fails_only_its_job(engine, wg):
    """The batch holding job 3 fails; the server re-runs that batch's jobs one at a time: job 3 ends
    with the injected error, every other job's survivors equal its alone-run."""
    jobs = jobs_mix()
    with wg.Server(0, fail_job=3) as srv:
        ids = [srv.submit(**j) for j in jobs]
        assert ids == [1, 2, 3, 4, 5]
        for k, (jid, job) in enumerate(zip(ids, jobs)):
            st = srv.wait(jid)
            if jid == 3:
                assert st["status"] == wg.WG_ERR_CUDA
                with pytest.raises(wg.EngineError, match="status 2"):
                    srv.take(jid)
            else:
                assert st["status"] == 0, k
                assert np.array_equal(srv.take(jid), alone(engine, job)), k
        # the server keeps working after the failure
        j = srv.submit(gen=(2, 1000), rect=(-4, 5, -4, 5), max_height=100)
        assert srv.wait(j)["status"] == 0
        assert np.array_equal(srv.take(j), alone(engine, {"gen": (2, 1000), "rect": (-4, 5, -4, 5),
                                                          "max_height": 100}))


def test_failure_mid_stream_with_small_batches(engine, wg):
    """Small batches (2^20 checks) so that the failing job shares several batches with others while
    jobs keep arriving: the others still finish with their alone-results."""
    jobs = jobs_mix() * 2
    with wg.Server(0, batch_checks=1 << 20, fail_job=7) as srv:
        ids = []
        for j in jobs:
            ids.append(srv.submit(**j))
            time.sleep(0.002)
        for jid, job in zip(ids, jobs):
            st = srv.wait(jid)
            if jid == 7:
                assert st["status"] == wg.WG_ERR_CUDA
            else:
                assert st["status"] == 0, jid
                assert np.array_equal(srv.take(jid), alone(engine, job)), jid


def test_arena_smaller_than_a_job(engine, wg):
    """A seed arena of 4,096 slots: a larger job is refused at submit; smaller jobs wait for slots
    and finish with their alone-results."""
    with wg.Server(0, arena_seeds=4096) as srv:
        with pytest.raises(wg.EngineError, match="status 4"):
            srv.submit(gen=(2, 5000), rect=(-4, 5, -4, 5), max_height=100)
        small = [{"gen": (3 + k, 3000), "rect": (-4, 5, -4, 5), "max_height": 100} for k in range(4)]
        ids = [srv.submit(**j) for j in small]
        for jid, job in zip(ids, small):
            assert srv.wait(jid)["status"] == 0
            assert np.array_equal(srv.take(jid), alone(engine, job))


def test_malformed_jobs_mid_stream(engine, wg):
    """Submits of an empty rect or an empty seed list fail at once and leave the queue intact."""
    with wg.Server(0) as srv:
        a = srv.submit(gen=(21, 2000), rect=(-4, 5, -4, 5), max_height=100)
        with pytest.raises(wg.EngineError, match="status 1"):
            srv.submit(gen=(21, 10), rect=(3, 3, 0, 5), max_height=-50)
        with pytest.raises(wg.EngineError, match="status 1"):
            srv.submit(seeds=np.zeros(0, np.int64), rect=(-4, 5, -4, 5), max_height=-50)
        b = srv.submit(gen=(22, 2000), rect=(-4, 5, -4, 5), max_height=100)
        for jid, base in ((a, 21), (b, 22)):
            assert srv.wait(jid)["status"] == 0
            assert np.array_equal(srv.take(jid), alone(engine, {"gen": (base, 2000), "rect": (-4, 5, -4, 5),
                                                                "max_height": 100}))


def test_close_with_jobs_pending(wg):
    """Closing a server whose queue still holds work returns promptly (the batch in flight finishes,
    queued jobs are dropped) and a new server on the same device works."""
    srv = wg.Server(0)
    for k in range(20):
        srv.submit(gen=(100 + k, 200000), rect=(-4, 5, -4, 5), max_height=-50)
    t0 = time.perf_counter()
    srv.close()
    assert time.perf_counter() - t0 < 30
    with wg.Server(0) as s2:
        j = s2.submit(gen=(2, 100), rect=(-4, 5, -4, 5), max_height=-50)
        assert s2.wait(j)["status"] == 0
