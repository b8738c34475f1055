"""Test infrastructure only: ctypes bindings of the two CPU checkers.

* ``Port``  -- oracle/_build/libwitch_oracle.so, the C restatement (oracle/witch_oracle.c).
* ``Ref``   -- oracle/_ref/liblysh_ref.so, the reference's own lysh compiled from its sources
  (oracle/Makefile) plus the flat wrappers of oracle/ref_harness.c.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "libwitch_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "liblysh_ref.so")
REF_BIN = os.path.join(HERE, "_ref", "lysh")


def reference_root() -> str:
    """Where the reference's sources lie: $WG_REFERENCE_ROOT, else a `reference` directory beside
    this repository's root."""
    return os.environ.get("WG_REFERENCE_ROOT") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


REF_SRC = os.path.join(reference_root(), "engine", "tools", "lysh", "src")


def build(ref: bool | None = None) -> None:
    """Compile the restatement, and the reference checker when its sources are present."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    if ref is None:
        ref = os.path.isdir(REF_SRC)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", "-j8", f"REF={reference_root()}"], check=True)


class WoOpts(C.Structure):
    _fields_ = [("mc_1_18_2", C.c_int), ("single_biome", C.c_int), ("pre_26_2", C.c_int),
                ("large_biomes", C.c_int)]


CANDIDATE_DTYPE = np.dtype([("seed_index", "<u8"), ("seed", "<i8"), ("rx", "<i4"), ("rz", "<i4"),
                            ("chunk_x", "<i4"), ("chunk_z", "<i4")])

# version name -> (mc_1_18_2, pre_26_2) for the phase-1 rules (engine/tools/lysh/src/main.c:104-125)
PHASE1_RULES = {"1.19.x~26.1": (0, 1), "1.21": (0, 1), "1.21.5": (0, 1), "26.2": (0, 0), "26.2~26.3": (0, 0),
                "1.18.2": (1, 1), "1.18.x": (1, 1), "1.20.1": (0, 1), "26.1": (0, 1)}


def as_u64(seeds) -> np.ndarray:
    if isinstance(seeds, np.ndarray) and seeds.dtype in (np.int64, np.uint64):
        return np.ascontiguousarray(seeds).view(np.uint64)
    return np.array([int(s) & 0xFFFFFFFFFFFFFFFF for s in seeds], dtype=np.uint64)


def rules(version: str, preset: str = "NORMAL") -> dict:
    mc, pre = PHASE1_RULES[version]
    return {"mc_1_18_2": mc, "pre_26_2": pre, "large_biomes": int(preset == "LARGE_BIOMES"),
            "single_biome": int(preset == "SINGLE_BIOME")}


class Port:
    """The C restatement of the phase-1 path."""

    def __init__(self, path: str = PORT_LIB):
        if not os.path.exists(path):
            build(ref=False)
        lib = C.CDLL(path)
        lib.wo_splitmix64.restype = C.c_uint64
        lib.wo_splitmix64.argtypes = [C.c_uint64]
        lib.wo_orientation.argtypes = [C.c_uint64, C.c_int, C.c_int]
        lib.wo_hut_in_region.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        lib.wo_noise_dump.argtypes = [C.c_uint64, C.c_char_p] + [C.c_void_p] * 4
        lib.wo_phase1_rect.restype = C.c_longlong
        lib.wo_phase1_rect.argtypes = [C.c_uint64, C.POINTER(WoOpts)] + [C.c_int] * 6 + [C.c_void_p] * 4
        lib.wo_probe.argtypes = [C.c_uint64, C.POINTER(WoOpts), C.c_int, C.c_int, C.c_int, C.c_void_p]
        lib.wo_scan_seeds.restype = C.c_longlong
        lib.wo_scan_seeds.argtypes = [C.c_void_p, C.c_uint64, C.c_longlong, C.POINTER(WoOpts)] + [C.c_int] * 7 + \
            [C.c_void_p, C.c_longlong, C.c_void_p]
        lib.wo_mineshaft_start.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_void_p]
        lib.wo_deep_starts.restype = C.c_longlong
        lib.wo_deep_starts.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                       C.c_longlong]
        lib.wo_region_const.restype = C.c_uint64
        lib.wo_region_const.argtypes = [C.c_int, C.c_int]
        lib.wo_perm_group.restype = C.c_uint32
        lib.wo_perm_group.argtypes = [C.c_uint32]
        lib.wo_group_regions.restype = C.c_longlong
        lib.wo_group_regions.argtypes = [C.c_uint32, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_longlong]
        lib.wo_solve_task.restype = C.c_longlong
        lib.wo_solve_task.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_longlong]
        self.lib = lib

    def region_const(self, rx: int, rz: int) -> int:
        return int(self.lib.wo_region_const(rx, rz))

    def perm_group(self, g: int) -> int:
        return int(self.lib.wo_perm_group(g & 0xFFFFF))

    def group_regions(self, c20: int, regime_x: int, regime_z: int, cap: int = 1 << 14) -> np.ndarray:
        """(rx, rz) rows of the regime's regions whose region constant has low 20 bits c20."""
        rx = np.zeros(cap, np.int32)
        rz = np.zeros(cap, np.int32)
        n = self.lib.wo_group_regions(c20, regime_x, regime_z, rx.ctypes.data, rz.ctypes.data, cap)
        return np.stack([rx[:min(n, cap)], rz[:min(n, cap)]], axis=1)

    def solve_task(self, X: int, rx: int, rz: int, ox: int, oz: int, cap: int = 64) -> list[int]:
        """Structure seeds S whose hut in (rx, rz) is at offsets (ox, oz) and whose carver state at
        that chunk is X (sorted)."""
        out = np.zeros(cap, np.uint64)
        n = self.lib.wo_solve_task(X & 0xFFFFFFFFFFFF, rx, rz, ox, oz, out.ctypes.data, cap)
        return sorted(int(v) for v in out[:min(n, cap)])

    def mineshaft_start(self, s48: int, cx: int, cz: int) -> tuple[bool, int]:
        carver = C.c_uint64()
        ok = self.lib.wo_mineshaft_start(s48 & 0xFFFFFFFFFFFF, cx, cz, C.byref(carver))
        return bool(ok), carver.value

    def deep_starts(self, s48s, rect, cap: int = 1 << 16) -> np.ndarray:
        """Rows (s48, rx, rz, cx, cz, carver) of hut chunks that are mineshaft starts."""
        s = np.ascontiguousarray(np.asarray([int(v) & 0xFFFFFFFFFFFF for v in s48s], dtype=np.uint64))
        out = np.zeros((cap, 6), np.int64)
        n = self.lib.wo_deep_starts(s.ctypes.data, len(s), *rect, out.ctypes.data, cap)
        return out[:min(n, cap)].copy()

    @staticmethod
    def _o(r: dict) -> WoOpts:
        return WoOpts(r["mc_1_18_2"], r["single_biome"], r["pre_26_2"], r["large_biomes"])

    def splitmix64(self, x: int) -> int:
        return int(self.lib.wo_splitmix64(x & 0xFFFFFFFFFFFFFFFF))

    def hut_chunk(self, seed: int, rx: int, rz: int, salt: int = 14357620) -> tuple[int, int]:
        cx, cz = C.c_int(), C.c_int()
        self.lib.wo_hut_in_region(seed & 0xFFFFFFFFFFFFFFFF, rx, rz, salt, C.byref(cx), C.byref(cz))
        return cx.value, cz.value

    def orientation(self, seed: int, hut_x: int, hut_z: int) -> int:
        return int(self.lib.wo_orientation(seed & 0xFFFFFFFFFFFFFFFF, hut_x, hut_z))

    def phase1_rect(self, seed: int, r: dict, max_height: int, rect, salt: int = 0):
        n = (rect[1] - rect[0]) * (rect[3] - rect[2])
        codes, tiers = np.zeros(n, np.int8), np.zeros(n, np.int8)
        cx, cz = np.zeros(n, np.int32), np.zeros(n, np.int32)
        o = self._o(r)
        self.lib.wo_phase1_rect(seed & 0xFFFFFFFFFFFFFFFF, C.byref(o), max_height, salt, *rect,
                                codes.ctypes.data, tiers.ctypes.data, cx.ctypes.data, cz.ctypes.data)
        return codes, tiers, cx, cz

    def probe(self, seed: int, r: dict, hut_x: int, hut_z: int, max_height: int) -> np.ndarray:
        out = np.zeros(38)
        o = self._o(r)
        self.lib.wo_probe(seed & 0xFFFFFFFFFFFFFFFF, C.byref(o), hut_x, hut_z, max_height, out.ctypes.data)
        return out

    def noise_dump(self, seed: int, name: str):
        h, pr, org, pm = np.zeros(6), np.zeros(32, np.int32), np.zeros(96), np.zeros(32 * 256, np.uint8)
        self.lib.wo_noise_dump(seed & 0xFFFFFFFFFFFFFFFF, name.encode(), h.ctypes.data, pr.ctypes.data,
                               org.ctypes.data, pm.ctypes.data)
        return h, pr, org, pm

    def scan_seeds(self, r: dict, max_height: int, rect, seeds=None, gen=None, threads: int = 0, salt: int = 0,
                   cap: int = 1 << 16):
        """Phase-1 survivors of many seeds, sorted by (seed_index, rz, rx), plus the funnel."""
        if seeds is not None:
            arr = as_u64(seeds)
            ptr, base, n = arr.ctypes.data, 0, len(arr)
        else:
            arr = None
            ptr, base, n = None, gen[0] & 0xFFFFFFFFFFFFFFFF, gen[1]
        out = np.zeros(cap, CANDIDATE_DTYPE)
        hist = np.zeros(11, np.int64)
        o = self._o(r)
        found = self.lib.wo_scan_seeds(ptr, base, n, C.byref(o), max_height, salt, *rect, threads,
                                       out.ctypes.data, cap, hist.ctypes.data)
        if found > cap:
            return self.scan_seeds(r, max_height, rect, seeds, gen, threads, salt, cap=int(found))
        out = out[:found]
        out.sort(order=["seed_index", "rz", "rx"])
        return out, hist


ROOM_LIB = os.path.join(HERE, "_ref", "libroom_ref.so")


class RoomRef:
    """The reference's own Deep Dive room walk (engine/gpu/room_core.h), compiled into oracle/_ref/."""

    def __init__(self, path: str = ROOM_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing (make -C oracle ref REF=<reference root> needs the reference sources)")
        lib = C.CDLL(path)
        lib.roomh_is_start.argtypes = [C.c_int64, C.c_int, C.c_int]
        lib.roomh_walk.restype = C.c_longlong
        lib.roomh_walk.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                   C.c_longlong]
        self.lib = lib

    def is_start(self, s48: int, cx: int, cz: int) -> bool:
        return bool(self.lib.roomh_is_start(C.c_int64(s48 & 0xFFFFFFFFFFFF), cx, cz))

    def walk(self, s48s, rect, cap: int = 1 << 16) -> np.ndarray:
        """Rows (s48, rx, rz, cx, cz) of hut chunks that are mineshaft starts."""
        s = np.ascontiguousarray(np.asarray([int(v) & 0xFFFFFFFFFFFF for v in s48s], dtype=np.int64))
        out = np.zeros((cap, 5), np.int64)
        n = self.lib.roomh_walk(s.ctypes.data, len(s), *rect, out.ctypes.data, cap)
        return out[:min(n, cap)].copy()


class Ref:
    """The reference's lysh, compiled from its sources into oracle/_ref/."""

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing (make -C oracle ref REF=<reference root> needs the reference sources)")
        lib = C.CDLL(path)
        lib.refh_parse_version.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.refh_hut_in_region.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        lib.refh_hut_orientation.argtypes = [C.c_uint64, C.c_int, C.c_int]
        lib.refh_phase1_rect.restype = C.c_longlong
        lib.refh_phase1_rect.argtypes = [C.c_uint64] + [C.c_int] * 11 + [C.c_void_p] * 4
        lib.refh_probe.argtypes = [C.c_uint64] + [C.c_int] * 8 + [C.c_void_p]
        lib.refh_noise_dump.argtypes = [C.c_uint64, C.c_char_p] + [C.c_void_p] * 4
        lib.refh_ctx_new.restype = C.c_void_p
        lib.refh_ctx_new.argtypes = [C.c_uint64] + [C.c_int] * 6
        lib.refh_ctx_free.argtypes = [C.c_void_p]
        lib.refh_ctx_eval.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
        lib.refh_ctx_height.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        lib.refh_ctx_density.restype = C.c_double
        lib.refh_ctx_density.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        lib.refh_ctx_block.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        lib.refh_grade_scan.argtypes = [C.c_uint64] + [C.c_int] * 13 + [C.c_void_p, C.c_int, C.c_void_p]
        lib.refh_ctx_probe.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_longlong, C.c_void_p]
        lib.refh_phase1_seeds.restype = C.c_double
        lib.refh_phase1_seeds.argtypes = [C.c_void_p, C.c_longlong] + [C.c_int] * 12 + [C.c_void_p]
        lib.refh_cpu_count.restype = C.c_int
        self.lib = lib

    def version(self, name: str) -> tuple[int, int, int]:
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        if self.lib.refh_parse_version(name.encode(), C.byref(a), C.byref(b), C.byref(c)):
            raise ValueError(name)
        return a.value, b.value, c.value

    def phase1_rect(self, seed: int, r: dict, max_height: int, rect, salt: int = 0, tree: int = 0):
        n = (rect[1] - rect[0]) * (rect[3] - rect[2])
        codes, tiers = np.zeros(n, np.int8), np.zeros(n, np.int8)
        cx, cz = np.zeros(n, np.int32), np.zeros(n, np.int32)
        self.lib.refh_phase1_rect(seed & 0xFFFFFFFFFFFFFFFF, r["mc_1_18_2"], r["pre_26_2"], r["large_biomes"],
                                  r["single_biome"], tree, max_height, salt, *rect, codes.ctypes.data,
                                  tiers.ctypes.data, cx.ctypes.data, cz.ctypes.data)
        return codes, tiers, cx, cz

    def probe(self, seed: int, r: dict, hut_x: int, hut_z: int, max_height: int) -> np.ndarray:
        out = np.zeros(38)
        self.lib.refh_probe(seed & 0xFFFFFFFFFFFFFFFF, r["mc_1_18_2"], r["pre_26_2"], r["large_biomes"],
                            r["single_biome"], 0, hut_x, hut_z, max_height, out.ctypes.data)
        return out

    def noise_dump(self, seed: int, name: str):
        h, pr, org, pm = np.zeros(6), np.zeros(32, np.int32), np.zeros(96), np.zeros(32 * 256, np.uint8)
        self.lib.refh_noise_dump(seed & 0xFFFFFFFFFFFFFFFF, name.encode(), h.ctypes.data, pr.ctypes.data,
                                 org.ctypes.data, pm.ctypes.data)
        return h, pr, org, pm

    def ctx(self, seed: int, r: dict, max_height: int = -50, tree: int = 0) -> "RefCtx":
        """One lysh_search_ctx (phase 1 + phase 2 state of a seed; eval.c:70-107)."""
        return RefCtx(self, seed, r, max_height, tree)

    def grade_scan(self, seed: int, r: dict, max_height: int, rect, max_y: int, threads: int = 0, salt: int = 0,
                   tree: int = 0, cap: int = 4096):
        """lysh_grade_scan -> (hits [n, 12] int32, stats [7])."""
        hits = np.zeros((cap, 12), np.int32)
        st = np.zeros(7, np.int64)
        self.lib.refh_grade_scan(seed & 0xFFFFFFFFFFFFFFFF, r["mc_1_18_2"], r["pre_26_2"], r["large_biomes"],
                                 r["single_biome"], tree, max_height, *rect, salt, threads, max_y,
                                 hits.ctypes.data, cap, st.ctypes.data)
        return hits[:st[6]].copy(), st

    def phase1_seeds(self, seeds, r: dict, max_height: int, rect, threads: int = 0, salt: int = 0):
        """Times lysh's own phase-1 scan over many seeds; returns (seconds, accepted per seed)."""
        arr = as_u64(seeds)
        acc = np.zeros(len(arr), np.int64)
        secs = self.lib.refh_phase1_seeds(arr.ctypes.data, len(arr), r["mc_1_18_2"], r["pre_26_2"],
                                          r["large_biomes"], r["single_biome"], 0, max_height, salt, *rect,
                                          threads, acc.ctypes.data)
        return secs, acc

    def cpu_count(self) -> int:
        return int(self.lib.refh_cpu_count())


# lysh_hut_result fields in refh_ctx_eval's output order (ref_harness.c).
EVAL_FIELDS = ("dir", "size_x", "size_z", "avg_y", "sum_h", "wet_columns", "flooded", "ok", "reject", "biome_ok",
               "biome_winner", "biome_qx", "biome_qy", "biome_qz", "biome_occ_y", "t0", "t1", "t2", "t3", "t4", "t5",
               "rx", "rz", "all_dry")


class RefCtx:
    """A lysh search context of the compiled reference: phase-2 probes and lysh_eval_hut."""

    def __init__(self, ref: Ref, seed: int, r: dict, max_height: int, tree: int):
        self.ref = ref
        self.h = ref.lib.refh_ctx_new(seed & 0xFFFFFFFFFFFFFFFF, r["mc_1_18_2"], r["pre_26_2"], r["large_biomes"],
                                      r["single_biome"], tree, max_height)

    def probe(self, kind: int, xyz) -> np.ndarray:
        pts = np.ascontiguousarray(np.asarray(xyz, dtype=np.int32).reshape(-1, 3))
        out = np.zeros(len(pts))
        self.ref.lib.refh_ctx_probe(self.h, kind, pts.ctypes.data, len(pts), out.ctypes.data)
        return out

    def eval_hut(self, hut_x: int, hut_z: int, max_y: int) -> dict:
        out = np.zeros(24, np.int64)
        self.ref.lib.refh_ctx_eval(self.h, hut_x, hut_z, max_y, out.ctypes.data)
        return dict(zip(EVAL_FIELDS, (int(v) for v in out)))

    def close(self) -> None:
        if self.h:
            self.ref.lib.refh_ctx_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
