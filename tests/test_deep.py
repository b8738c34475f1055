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
    """The terrain-stage fixture: hunt.py's four TERRAIN_REFERENCE spots pass exactly their known
    seed's variant; every data/finds.tsv hut with coordinates (50, depths -55 to -59) is a start
    chunk whose known world seed is among lysh's phase-1 survivors at -54; the extra chunk is no
    start."""
    d = np.load(os.path.join(GOLDEN, "deep_spots.npz"))
    seeds = [s for s, _, _ in KNOWN[1:]]
    passed = d["passed"]
    off = np.concatenate([[0], np.cumsum(d["counts"])])
    for i, seed in enumerate(seeds):
        assert passed[off[i]:off[i + 1]].tolist() == [(seed & ((1 << 64) - 1)) >> 48]
        assert int(d["seed"][i]) == seed
    finds = [i for i in range(len(d["s48"])) if int(d["depth"][i]) != 0]
    assert len(finds) == 50 and set(int(d["depth"][i]) for i in finds) == {-55, -57, -58, -59}
    for i in finds:
        seed = int(d["seed"][i]) & ((1 << 64) - 1)
        assert d["start"][i] == 1 and int(d["s48"][i]) == seed & M48
        assert (seed >> 48) in passed[off[i]:off[i + 1]].tolist(), i
    assert d["start"][-1] == 0 and d["counts"][-1] == 0


def test_sweep_fixture_redraw_accounting():
    """The whole-world sweep fixture: the reference's room walk built on the CPU with -O2 counts
    what its GPU engine counted; built with -fwrapv (nextInt(24) re-draws as java.util.Random does)
    the counts differ only by the starts of regions that re-draw, which the fixture lists per build."""
    g = np.load(os.path.join(GOLDEN, "deep_sweep.npz"))
    assert g["cpu_starts_o2"].tolist() == g["ref_starts"].tolist()
    for i, s in enumerate(g["s48"]):
        n_o2 = int((g["redraw_starts_o2"][:, 0] == s).sum())
        n_java = int((g["redraw_starts_wrapv"][:, 0] == s).sum())
        assert int(g["cpu_starts_wrapv"][i]) - int(g["cpu_starts_o2"][i]) == n_java - n_o2
    assert len(g["redraw_starts_o2"]) + len(g["redraw_starts_wrapv"]) > 0


def test_oracle_redraw_regions_follow_java(port):
    """At each region of the sweep fixture whose hut re-draws, the oracle (whose nextInt re-draws
    like java.util.Random and lysh's rng.c:213-226) has a start exactly where the -fwrapv build has
    one; the chunks the -O2 build reports there are starts of the carver test but not the hut's."""
    g = np.load(os.path.join(GOLDEN, "deep_sweep.npz"))
    java = {(int(r[0]), int(r[1]), int(r[2])): [int(v) for v in r] for r in g["redraw_starts_wrapv"]}
    for key, row in java.items():
        got = port.deep_starts([key[0]], (key[1], key[1] + 1, key[2], key[2] + 1))
        assert got[:, :5].tolist() == [row]
    for s48, rx, rz, cx, cz in (tuple(int(v) for v in r) for r in g["redraw_starts_o2"]):
        assert port.mineshaft_start(s48, cx, cz)[0]
        got = port.deep_starts([s48], (rx, rx + 1, rz, rz + 1))
        assert (cx, cz) not in [(int(r[3]), int(r[4])) for r in got]
        assert len(got) == (1 if (s48, rx, rz) in java else 0)


def test_room_reference_pinned(bind_mod):
    if not os.path.exists(bind_mod.ROOM_LIB):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    room = bind_mod.RoomRef()
    d = np.load(os.path.join(GOLDEN, "deep_starts.npz"))
    got = room.walk(d["s48"][:3], tuple(int(v) for v in d["rects"][0]))
    want = d["rows0"][np.isin(d["rows0"][:, 0], d["s48"][:3])]
    assert np.array_equal(got, want)


def test_finisher_fixture_known_answers():
    """The finisher fixture (the reference's own tools): hunt.py's REFERENCE is accepted with the
    mineshaft floor at -58, and every located data/finds.tsv hut's listed depth lies between the
    carved floors msroom gives for the two top-layer cases (top1 <= depth <= top0); for 47 of the
    50 it is top1, the value hunt.py prints."""
    fx = np.load(os.path.join(GOLDEN, "finish_rows.npz"))
    assert (fx["verdict_ok"][0], fx["start"][0], fx["top1"][0]) == (1, 1, -58)
    d = np.load(os.path.join(GOLDEN, "deep_spots.npz"))
    finds = {(int(d["seed"][i]), int(d["chunk_x"][i]), int(d["chunk_z"][i])): int(d["depth"][i])
             for i in range(len(d["s48"])) if int(d["depth"][i]) != 0}
    seen = {}
    for i in range(len(fx["ws"])):
        key = (int(fx["ws"][i]), int(fx["cx"][i]), int(fx["cz"][i]))
        if key in finds:
            assert fx["start"][i] == 1 and int(fx["top1"][i]) <= finds[key] <= int(fx["top0"][i]), key
            seen[key] = int(fx["top1"][i]) == finds[key]
    assert len(seen) == 50 and sum(seen.values()) == 47
