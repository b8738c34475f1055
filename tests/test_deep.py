"""CPU: the Deep Dive oracle (the C restatement of the region walk) against the reference.

The fixtures (tests/golden/make_golden_deep.py) come from the reference's own room walker
(engine/gpu/room_core.h, compiled into oracle/_ref/libroom_ref.so) and from lysh.  Known
answers: hunt.py's REFERENCE hut and its four TERRAIN_REFERENCE spots are mineshaft start
chunks, and each spot's only surviving upper-bit variant is the known seed's.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
M48 = (1 << 48) - 1
KNOWN = [(3159335117276934358, -1852878, -1380275), (-5359549684776256167, -1549312, 1202688),
         (-5842228900837151037, 84992, 981504), (-7671590099420590308, 1509888, 1081344),
         (-2118812217737330443, 197632, 1145344)]


def test_known_starts(port):
    for seed, cx, cz in KNOWN:
        assert port.mineshaft_start(seed, cx, cz)[0], (seed, cx, cz)
        assert not port.mineshaft_start(seed, cx + 1, cz)[0] or not port.mineshaft_start(seed, cx, cz + 1)[0]


def test_oracle_walk_matches_reference_fixture(port):
    d = np.load(os.path.join(GOLDEN, "deep_starts.npz"))
    for k, rect in enumerate(d["rects"]):
        got = port.deep_starts(d["s48"], tuple(int(v) for v in rect))
        assert np.array_equal(got[:, :5], d[f"rows{k}"]), k


def test_spot_fixture_known_answers():
    d = np.load(os.path.join(GOLDEN, "deep_spots.npz"))
    seeds = [s for s, _, _ in KNOWN[1:]]
    passed = d["passed"]
    off = np.concatenate([[0], np.cumsum(d["counts"])])
    for i, seed in enumerate(seeds):
        assert passed[off[i]:off[i + 1]].tolist() == [(seed & ((1 << 64) - 1)) >> 48]
    assert d["start"][-1] == 0 and d["counts"][-1] == 0


def test_room_reference_pinned(bind_mod):
    if not os.path.exists(bind_mod.ROOM_LIB):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    room = bind_mod.RoomRef()
    d = np.load(os.path.join(GOLDEN, "deep_starts.npz"))
    got = room.walk(d["s48"][:3], tuple(int(v) for v in d["rects"][0]))
    want = d["rows0"][np.isin(d["rows0"][:, 0], d["s48"][:3])]
    assert np.array_equal(got, want)
