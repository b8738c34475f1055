"""GPU: the Deep Dive forward sweep with the layout-catalogue probe (wg_deep_sweep).

The sweep walks every hut region of a rect for each structure seed, tests each hut chunk for a
mineshaft start and probes each start's carver state in the layout catalogue, as the reference's
forward mode does (sweepProbeKernel, engine/gpu/hut_lookup_v4_source.cu:77-99, :1504-1530).
Pinned three ways: its starts equal the region walk's (itself pinned to the reference's room
walker), its matches equal the oracle's starts filtered by the catalogue, and over the whole
+-30M world its per-seed start and match counts equal the reference engine's own
(tests/golden/deep_sweep.npz, tests/golden/make_golden_sweep.py).
"""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_sweep_starts_and_matches_equal_the_walk(engine):
    """Starts per seed equal the region walk's; a catalogue of some of those starts' carver states
    (plus decoys) gives exactly those starts back, with their catalogue values."""
    rect = (-700, 700, -500, 500)
    walk = engine.deep_starts(base=31337, count=5, rect=rect)
    pick = walk[::97]
    layouts = [int(c) for c in pick["carver"]] + [1, 2, (1 << 48) - 1]
    values = list(range(7, 7 + len(pick))) + [0, 0, 0]
    matches, starts = engine.deep_sweep(layouts, values, base=31337, count=5, rect=rect)
    assert starts.tolist() == np.bincount(walk["seed_index"], minlength=5).tolist()
    keep = np.isin(walk["carver"], np.array(layouts, dtype=np.int64))
    want = walk[keep]
    assert len(matches) == len(want) >= len(pick)
    for f in ("seed_index", "s48", "rx", "rz", "chunk_x", "chunk_z", "carver"):
        assert np.array_equal(matches[f], want[f]), f
    val = dict(zip(layouts, values))
    assert [int(v) for v in matches["value"]] == [val[int(c)] for c in matches["carver"]]


def test_sweep_start_counts_when_warps_straddle_seeds(engine):
    """A rect of 33 columns x 64 rows gives each structure seed 33 tasks, so most warps hold lanes of
    two seeds: the per-seed start counts still equal the region walk's."""
    rect = (-17, 16, -40, 24)
    walk = engine.deep_starts(base=777, count=40, rect=rect)
    _, starts = engine.deep_sweep([5], base=777, count=40, rect=rect)
    assert starts.tolist() == np.bincount(walk["seed_index"], minlength=40).tolist()


def test_sweep_against_the_oracle(engine, port):
    """Matches on explicit structure seeds equal the C restatement's starts filtered by the catalogue,
    at the world border too (re-draws of the hut offsets included)."""
    s48 = [0, 1, 0xFFFFFFFFFFFF, 274264440333605]
    for rect in ((-40, 40, -40, 40), (58500, 58594, -58593, -58500)):
        want = port.deep_starts(s48, rect)
        layouts = [int(r[5]) for r in want[::3]]
        matches, starts = engine.deep_sweep(layouts, s48=s48, rect=rect)
        keep = np.isin(want[:, 5], np.array(layouts, dtype=np.int64))
        assert np.array_equal(np.stack([matches["s48"], matches["rx"], matches["rz"], matches["chunk_x"],
                                        matches["chunk_z"], matches["carver"]], 1), want[keep]), rect
        assert starts.sum() == len(want)


def test_sweep_whole_world_counts_equal_reference(engine, wg):
    """Every region of the +-30M world for three structure seeds of the reference's forward
    enumeration: starts per seed equal the reference's room walk with nextInt(24) re-drawing as
    java.util.Random does (its header built with -fwrapv); catalogue matches equal its GPU engine's.
    The reference's optimised builds drop the re-draw (a signed-overflow test), which moves one
    start of seed 1001 and two of seed 1002: the fixture lists them, and each listed region is
    checked alone."""
    g = np.load(os.path.join(GOLDEN, "deep_sweep.npz"))
    matches, starts = engine.deep_sweep([int(x) for x in g["layouts"]], g["values"], s48=[int(s) for s in g["s48"]],
                                        rect=wg.WORLD_REGIONS)
    assert starts.tolist() == g["cpu_starts_wrapv"].tolist()
    assert np.bincount(matches["seed_index"], minlength=len(g["s48"])).tolist() == g["ref_matches"].tolist()
    java = {(int(r[0]), int(r[1]), int(r[2])): (int(r[3]), int(r[4])) for r in g["redraw_starts_wrapv"]}
    for s48, rx, rz, cx, cz in g["redraw_starts_o2"]:
        _, n = engine.deep_sweep([5], s48=[int(s48)], rect=(int(rx), int(rx) + 1, int(rz), int(rz) + 1))
        assert n.tolist() == [1 if (int(s48), int(rx), int(rz)) in java else 0]
    for (s48, rx, rz), (cx, cz) in java.items():
        walk = engine.deep_starts(s48=[s48], rect=(rx, rx + 1, rz, rz + 1))
        assert [(int(w["chunk_x"]), int(w["chunk_z"])) for w in walk] == [(cx, cz)]
