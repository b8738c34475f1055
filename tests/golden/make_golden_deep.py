"""Generates the Deep Dive golden fixtures in this folder from the reference's own code.

Run from the repository root after `make -C oracle ref REF=<reference root>`:

    python tests/golden/make_golden_deep.py

  deep_starts.npz  the reference's room walk (engine/gpu/room_core.h rcWalkInit / rcWalkStep,
                   compiled into oracle/_ref/libroom_ref.so): every region whose swamp-hut chunk
                   is a mineshaft start, for 10 structure seeds (8 random, the low 48 bits of
                   hunt.py's REFERENCE and of one TERRAIN_REFERENCE seed) over a rect near the
                   origin and one in the far regime (|r| > 32,768)
  deep_spots.npz   the terrain stage of hunt.py's four TERRAIN_REFERENCE spots, every
                   data/finds.tsv hut with coordinates (50 of its 53 rows; read from the
                   reference's data/finds.tsv, found through oracle/bind.py's reference_root())
                   and one chunk that is not a start: which of the 65,536 upper-bit variants
                   (u << 48) | S48 pass lysh's phase 1 (lysh_scan_rect, oracle/_ref/liblysh_ref.so)
                   at maxHeight -54 in the spot's region; `seed` holds each spot's known world
                   seed (0 for the non-start chunk), whose variant must be among them
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import bind  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
M48 = (1 << 48) - 1
# hunt.py:83-85 (REFERENCE, TERRAIN_REFERENCE): seed, chunk x, chunk z
REFERENCE = (3159335117276934358, -1852878, -1380275)
TERRAIN_REFERENCE = [(-5359549684776256167, -1549312, 1202688), (-5842228900837151037, 84992, 981504),
                     (-7671590099420590308, 1509888, 1081344), (-2118812217737330443, 197632, 1145344)]
RECTS = [(-160, 160, -160, 160), (40000, 40120, -58593, -58473)]


def read_finds() -> list[tuple[int, int, int, int]]:
    """data/finds.tsv rows with coordinates: (depth, seed, x, z).  The coordinates lie in the hut's
    chunk (47 rows give the in-hut /tp point, chunk corner + (3, 7); three give the corner itself),
    so the chunk is (floor(x / 16), floor(z / 16))."""
    rows = []
    with open(os.path.join(bind.reference_root(), "data", "finds.tsv")) as f:
        for line in f:
            if line.startswith("#"):
                continue
            p = line.rstrip("\n").split("\t")
            if len(p) >= 5 and p[2] and p[4]:
                rows.append((int(p[0]), int(p[1]), int(p[2]), int(p[4])))
    return rows


def main() -> None:
    room = bind.RoomRef()
    rng = np.random.default_rng(11)
    s48 = [int(v) for v in rng.integers(0, 1 << 48, 8, dtype=np.uint64)]
    s48 += [REFERENCE[0] & M48, TERRAIN_REFERENCE[0][0] & M48]
    arrays = {"s48": np.array(s48, dtype=np.int64), "rects": np.array(RECTS, dtype=np.int32)}
    for k, rect in enumerate(RECTS):
        arrays[f"rows{k}"] = room.walk(s48, rect)
    np.savez_compressed(os.path.join(OUT, "deep_starts.npz"), **arrays)

    ref = bind.Ref()
    r = bind.rules("1.19.x~26.1")
    spots = [(seed, cx, cz, 0) for seed, cx, cz in TERRAIN_REFERENCE]
    for depth, seed, x, z in read_finds():
        spots.append((seed, x // 16, z // 16, depth))
    spots.append((0, spots[0][1] + 1, spots[0][2], 0))   # a chunk that is not a start (S48 of spot 0)
    s48_of = [sp[0] & M48 for sp in spots]
    s48_of[-1] = TERRAIN_REFERENCE[0][0] & M48
    rows = []
    u_all = np.arange(1 << 16, dtype=np.uint64)
    for (seed, cx, cz, depth), S in zip(spots, s48_of):
        start = room.is_start(S, cx, cz)
        passed = np.zeros(0, np.int64)
        if start:
            seeds = (u_all << np.uint64(48)) | np.uint64(S)
            rect = (cx >> 5, (cx >> 5) + 1, cz >> 5, (cz >> 5) + 1)
            _, acc = ref.phase1_seeds(seeds, r, -54, rect, threads=os.cpu_count() or 1)
            passed = np.nonzero(np.asarray(acc) > 0)[0].astype(np.int64)
        rows.append((S, cx, cz, int(start), passed, seed, depth))
        print(f"spot S={S} chunk ({cx},{cz}) start={start} passing variants={len(passed)}", flush=True)
    np.savez_compressed(os.path.join(OUT, "deep_spots.npz"),
                        s48=np.array([r_[0] for r_ in rows], dtype=np.int64),
                        chunk_x=np.array([r_[1] for r_ in rows], dtype=np.int32),
                        chunk_z=np.array([r_[2] for r_ in rows], dtype=np.int32),
                        start=np.array([r_[3] for r_ in rows], dtype=np.int8),
                        counts=np.array([len(r_[4]) for r_ in rows], dtype=np.int64),
                        passed=np.concatenate([r_[4] for r_ in rows]) if rows else np.zeros(0, np.int64),
                        seed=np.array([r_[5] for r_ in rows], dtype=np.int64),
                        depth=np.array([r_[6] for r_ in rows], dtype=np.int64),
                        max_height=np.int64(-54))


if __name__ == "__main__":
    main()
