"""GPU: the Deep Dive solver (wg_deep_solve / wg_deep_solve_tasks) through the C ABI.

Bar: the exact hit set.  Group ranges of five plans (three layouts, regimes 22 / 00 / 21, offset
classes odd / u2 / eq) must give the reference solver's hits (tests/golden/deep_solve.npz, from
hut_lookup_v4 --solve5); explicit tasks, planted or random, must give the oracle's solutions.
"""
from __future__ import annotations

import numpy as np
import pytest

from test_deep_solve import planted

pytestmark = pytest.mark.gpu

M48 = (1 << 48) - 1


def test_groups_equal_the_reference(engine, golden):
    d = golden("deep_solve.npz")
    for k, (lay, rgx, rgz, tier, first, count) in enumerate(d["cases"]):
        hits, st = engine.deep_solve([(int(lay), (int(rgx), int(rgz)), int(tier))], int(first), int(count))
        mine = sorted((int(h["s48"]), int(h["chunk_x"]), int(h["chunk_z"])) for h in hits)
        ref = sorted((int(r[0]) & M48, int(r[1]), int(r[2])) for r in d[f"hits{k}"])
        assert mine == ref, k
        assert st["host_check_failures"] == 0 and st["hits"] == len(ref)
        assert all(int(h["layout"]) == int(lay) for h in hits)
        assert set(int(h["group"]) for h in hits) <= set(range(int(first), int(first) + int(count)))


def test_group_regions_equal_the_oracle(engine, port):
    """The regions a group covers: the solver's count against a brute-force scan of the regime."""
    lay = 231564844655014
    for g, regime in ((9, (0, 0)), (12345, (0, 0))):
        _, st = engine.deep_solve([(lay, regime, "odd")], g, 1)
        assert st["regions"] == len(port.group_regions(port.perm_group(g), *regime))
        assert st["tasks"] == st["regions"] * 288


@pytest.mark.parametrize("cls", [1, 2, 3])
def test_planted_tasks_equal_the_oracle(engine, port, cls):
    rng = np.random.default_rng(200 + cls)
    for _ in range(6):
        S, rx, rz, ox, oz, X = planted(port, rng, cls)
        got = sorted(int(h["s48"]) for h in engine.deep_solve_tasks(X, [rx], [rz], [ox], [oz]))
        assert S in got
        assert got == port.solve_task(X, rx, rz, ox, oz)


def test_many_tasks_one_call(engine, port):
    """Tasks of one layout solved together (hits keyed by task index) equal the oracle task by task;
    planted tasks of the layout guarantee hits."""
    rng = np.random.default_rng(7)
    X = 231564844655014
    rx = list(rng.integers(-58593, 58594, 40))
    rz = list(rng.integers(-58593, 58594, 40))
    ox = list(rng.integers(0, 24, 40))
    oz = list(rng.integers(1, 24, 40))
    got = sorted((int(h["group"]), int(h["s48"])) for h in engine.deep_solve_tasks(X, rx, rz, ox, oz))
    want = sorted((i, s) for i in range(40) for s in port.solve_task(X, int(rx[i]), int(rz[i]), int(ox[i]), int(oz[i])))
    assert got == want


def test_solver_errors(engine, wg):
    with pytest.raises(wg.EngineError):
        engine.deep_solve([(1, (0, 0), 4)], 0, 1)
    with pytest.raises(wg.EngineError):
        engine.deep_solve([(1, (3, 0), 1)], 0, 1)
    with pytest.raises(wg.EngineError):
        engine.deep_solve([(1, (0, 0), 1)], (1 << 20) - 1, 2)        # past the last group
    with pytest.raises(wg.EngineError):
        engine.deep_solve_tasks(1, [0], [0], [0], [0])                 # offsets (0, 0) have no class
