"""B200 Seed Check engine: Python binding of libwitchgpu.so (include/witchgpu.h).

The engine runs the reference's Seed Check phase 1 (lysh_phase1_check_ex,
engine/tools/lysh/src/phase1.c:130-200) on the GPU: world seeds -> swamp-hut region
placement -> erosion / temperature / ridge gates -> cave ladder -> continentalness ->
floodedness.  This module is a thin ctypes layer; all work happens in the CUDA library,
and every call fails loudly when the library or a GPU is missing (there is no CPU path).

The package directory name is not a Python identifier; load it with
importlib.util.spec_from_file_location (registering it in sys.modules first), as
bench.py and tests/conftest.py do.
"""
from __future__ import annotations

import ctypes as C
import functools
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwitchgpu.so")
WORKER_PATH = os.path.join(HERE, "phase1_scan")
HUT_LOOKUP_PATH = os.path.join(HERE, "hut_lookup")
BIOME_MAP_PATH = os.path.join(HERE, "biome_map")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "witchgpu.h")

WG_OK, WG_ERR_ARG, WG_ERR_CUDA, WG_ERR_NOMEM, WG_ERR_CAPACITY, WG_ERR_NODEV = 0, 1, 2, 3, 4, 5

# Reject codes (LYSH_P1_REJECT_*, engine/tools/lysh/src/phase1.h:61-74).
REJECT_NAMES = ("erosion < 0.55", "temperature", "ridge", "Entrance@50", "Entrance@60", "cave@maxHeight",
                "cave ladder (y<=0)", "cave ladder (y>0)", "continentalness < -0.11", "floodedness > 0.41",
                "ACCEPT")
ACCEPT = 10
DEFAULT_VERSION = "1.19.x~26.1"   # the hunt driver's version (hunt.py DEFAULTS)
SALT = 14357620


class Opts(C.Structure):
    """wg_opts: field-for-field lysh_phase1_opts."""
    _fields_ = [("mc_1_18_2", C.c_int), ("single_biome", C.c_int), ("pre_26_2", C.c_int),
                ("large_biomes", C.c_int), ("biome_tree", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("scanned", C.c_int64), ("accepted", C.c_int64), ("climate_survivors", C.c_int64),
                ("deep_candidates", C.c_int64), ("reject_hist", C.c_int64 * 11), ("tier_hist", C.c_int64 * 7),
                ("batches", C.c_int64), ("retries", C.c_int64), ("kernel_launches", C.c_int64 * 3),
                ("kernel_ms", C.c_double * 3), ("gpu_ms", C.c_double), ("wall_ms", C.c_double),
                ("rechecks", C.c_int64), ("records", C.c_int64)]

    def as_dict(self) -> dict:
        return {"scanned": self.scanned, "accepted": self.accepted, "climate_survivors": self.climate_survivors,
                "deep_candidates": self.deep_candidates, "reject_hist": list(self.reject_hist),
                "tier_hist": list(self.tier_hist), "batches": self.batches, "retries": self.retries,
                "kernel_launches": list(self.kernel_launches), "kernel_ms": list(self.kernel_ms),
                "gpu_ms": self.gpu_ms, "wall_ms": self.wall_ms, "rechecks": self.rechecks, "records": self.records}


# wg_engine_set_noise_core values
NOISE_FP32, NOISE_FP64, NOISE_FP32_RECHECK_ALL, NOISE_FP32_CAVES = 0, 1, 2, 3
NOISE_CORES = {"fp32": NOISE_FP32, "fp64": NOISE_FP64, "fp32_recheck_all": NOISE_FP32_RECHECK_ALL,
               "fp32_caves": NOISE_FP32_CAVES}
# wg_noise_probe noise ids (the catalog's NoiseId order)
PROBE_NOISES = {"erosion": 0, "temperature": 1, "ridge": 2, "continentalness": 3, "erosion_large": 4,
                "temperature_large": 5, "continentalness_large": 6}
# wg_noise_probe_3d noise ids: the entrance gate's cave noises
PROBE_NOISES_3D = {"cave_entrance": 7, "spaghetti_rarity": 8, "spaghetti_thickness": 9, "spaghetti_3d_1": 10,
                   "spaghetti_3d_2": 11, "roughness_modulator": 12, "roughness": 13}


CANDIDATE_DTYPE = np.dtype([("seed_index", "<u8"), ("seed", "<i8"), ("rx", "<i4"), ("rz", "<i4"),
                            ("chunk_x", "<i4"), ("chunk_z", "<i4")])

# Every symbol include/witchgpu.h declares.
EXPORTS = ("wg_engine_open", "wg_engine_close", "wg_engine_error", "wg_engine_set_noise_core", "wg_noise_probe",
           "wg_noise_probe_3d",
           "wg_parse_version", "wg_parse_preset",
           "wg_seed_check", "wg_seed_check_device", "wg_phase1_codes", "wg_seed_check_noalloc",
           "wg_eval_huts", "wg_grade_scan", "wg_p2_probe", "wg_deep_starts", "wg_deep_sweep", "wg_deep_spots",
           "wg_biome_map", "wg_biome_chunks", "wg_deep_solve", "wg_deep_solve_tasks", "wg_seed_check_jobs", "wg_engine_set_job_queue", "wg_engine_tune", "wg_engine_set_tuning",
           "wg_server_open", "wg_server_open_config", "wg_server_submit", "wg_server_poll", "wg_server_take",
           "wg_server_stats", "wg_server_close", "wg_mineshaft_tree", "wg_finish_rows")

# wg_deep_start: a swamp hut whose chunk is a mineshaft start chunk.
DEEP_START_DTYPE = np.dtype([("seed_index", "<u8"), ("s48", "<i8"), ("rx", "<i4"), ("rz", "<i4"), ("chunk_x", "<i4"), ("chunk_z", "<i4"),
                             ("carver", "<i8")])

# wg_sweep_match: a start chunk whose carver state is a catalogued layout.
SWEEP_MATCH_DTYPE = np.dtype([("seed_index", "<u8"), ("s48", "<i8"), ("rx", "<i4"), ("rz", "<i4"),
                              ("chunk_x", "<i4"), ("chunk_z", "<i4"), ("carver", "<i8"), ("value", "<u4"),
                              ("pad", "<u4")])
def _signed64(v: int) -> int:
    """A 64-bit seed given signed or unsigned, as the signed value the C ABI takes."""
    v = int(v) & 0xFFFFFFFFFFFFFFFF
    return v - (1 << 64) if v >= 1 << 63 else v


# wg_ms_piece: one piece of a mineshaft tree as mstree prints it (kind is the letter's code).
MS_PIECE_DTYPE = np.dtype([("kind", "<i4"), ("x0", "<i4"), ("y0", "<i4"), ("z0", "<i4"), ("x1", "<i4"), ("y1", "<i4"),
                           ("z1", "<i4"), ("facing", "<i4"), ("parent", "<i4"), ("rails", "<i4")])
# wg_finish_row: the mineshaft finisher's measurements of one Deep Dive survivor.
FINISH_DTYPE = np.dtype([("hut_x", "<i4"), ("hut_z", "<i4"), ("verdict_ok", "<i4"), ("avg_y", "<i4"),
                         ("tree_status", "<i4"), ("pieces", "<i4"), ("room_floor", "<i4"), ("biome", "<i4", (2,)),
                         ("nat", "<i4"), ("top", "<i4", (2,)), ("refused", "<i4", (2,)), ("no_guard", "<i4", (2,)),
                         ("sum_nat", "<i8"), ("sum_top", "<i8", (2,)), ("sum_no_guard", "<i8", (2,)),
                         ("scan_sum", "<i8"), ("scan_min", "<i4"), ("scan_max", "<i4"), ("le54", "<i4"),
                         ("lava", "<i4"), ("solid", "<i4"), ("nw", "<i4"), ("ne", "<i4"), ("sw", "<i4"), ("se", "<i4"),
                         ("above53", "<i4")])
DEEP_DARK = 183

# the +-30M world's hut regions, [rx0, rx1) x [rz0, rz1) (the reference's forward sweep: radius 58,593)
WORLD_REGIONS = (-58593, 58594, -58593, 58594)

# wg_hut_result (lysh_hut_result's fields, engine/tools/lysh/src/eval.h:63-85).
HUT_DTYPE = np.dtype([("hut_x", "<i4"), ("hut_z", "<i4"), ("rx", "<i4"), ("rz", "<i4"), ("dir", "<i4"),
                      ("axis_z", "<i4"), ("size_x", "<i4"), ("size_z", "<i4"), ("avg_y", "<i4"),
                      ("wet_columns", "<i4"), ("flooded", "<i4"), ("all_dry", "<i4"), ("ok", "<i4"),
                      ("reject", "<i4"), ("biome_ok", "<i4"), ("biome_winner", "<i4"), ("biome_qx", "<i4"),
                      ("biome_qy", "<i4"), ("biome_qz", "<i4"), ("biome_occ_y", "<i4"), ("sum_h", "<i8"),
                      ("biome_t", "<i8", (6,))])
HUT_REJECTS = ("ok", "avg_y > max_y", "flooded", "biome")
GRADE_INTS = 12   # hutX, hutZ, rx, rz, dir, avg_y, flooded, ok, wet, size_x, size_z, reject

# wg_p2_probe kinds (include/witchgpu.h).
PROBE_KINDS = {"base_noise": 0, "density_raw": 1, "column_top": 2, "continentalness": 3, "erosion": 4,
               "weirdness": 5, "offset": 6, "factor": 7, "peaks": 8, "fluid": 9, "density": 10, "block": 11,
               "height_pre": 12, "height": 13, "grid_main": 14}


class HutGrade(C.Structure):
    _fields_ = [("scanned", C.c_int64), ("evaluated", C.c_int64), ("accepted", C.c_int64),
                ("rejected_y", C.c_int64), ("rejected_flood", C.c_int64), ("rejected_biome", C.c_int64),
                ("hits_written", C.c_int32), ("ms", C.c_double), ("p2_ms", C.c_double)]



class SolveBundle(C.Structure):
    """wg_solve_bundle: one plan line (layout, regime per axis, offset class)."""
    _fields_ = [("layout", C.c_uint64), ("regime_x", C.c_int32), ("regime_z", C.c_int32), ("tier", C.c_int32),
                ("pad", C.c_int32)]


class SolveStats(C.Structure):
    _fields_ = [("groups", C.c_uint64), ("regions", C.c_uint64), ("tasks", C.c_uint64), ("candidates", C.c_uint64),
                ("hits", C.c_uint64), ("host_check_failures", C.c_uint64), ("gpu_ms", C.c_double),
                ("wall_ms", C.c_double)]


# wg_solve_hit: a structure seed whose hut chunk has the layout's carver state.
SOLVE_HIT_DTYPE = np.dtype([("s48", "<u8"), ("chunk_x", "<i4"), ("chunk_z", "<i4"), ("layout", "<u8"),
                            ("group", "<u8")])
SOLVE_TIERS = {"odd": 1, "u2": 2, "eq": 3}


class Job(C.Structure):
    """wg_job: one Seed Check job (seeds or a splitmix64 generator, rect, floor, rules)."""
    _fields_ = [("seeds", C.c_void_p), ("gen_base", C.c_uint64), ("n_seeds", C.c_uint64), ("rx0", C.c_int),
                ("rx1", C.c_int), ("rz0", C.c_int), ("rz1", C.c_int), ("max_height", C.c_int), ("salt", C.c_int),
                ("opts", Opts)]


class TuneReport(C.Structure):
    """wg_tune_report: per job class the regions-per-unit candidates and their device times."""
    _fields_ = [("max_regions", C.c_uint32 * 4), ("window", C.c_uint32 * 4),
                ("window_candidates", (C.c_uint32 * 4) * 4), ("window_ms", (C.c_double * 4) * 4),
                ("budget", C.c_uint64), ("budget_candidates", C.c_uint64 * 3), ("budget_ms", C.c_double * 3)]

    def as_dict(self) -> dict:
        classes = []
        for c in range(4):
            cands = [(int(self.window_candidates[c][q]), float(self.window_ms[c][q])) for q in range(4)
                     if self.window_candidates[c][q]]
            classes.append({"max_regions": int(self.max_regions[c]), "window": int(self.window[c]),
                            "candidates": [{"window": w, "ms": ms} for w, ms in cands]})
        return {"classes": classes, "budget": int(self.budget),
                "budget_candidates": [{"checks": int(self.budget_candidates[q]), "ms": float(self.budget_ms[q])}
                                      for q in range(3)]}


class ServerConfig(C.Structure):
    """wg_server_config: queue and arena limits, batch size, host-side fault injection."""
    _fields_ = [("max_queued_seeds", C.c_uint64), ("arena_seeds", C.c_uint64), ("batch_checks", C.c_uint64),
                ("fail_job", C.c_uint64)]


class JobStatus(C.Structure):
    _fields_ = [("done", C.c_int32), ("status", C.c_int32), ("found", C.c_uint64), ("queue_ms", C.c_double),
                ("latency_ms", C.c_double), ("batch_jobs", C.c_uint64)]

_lib = None


class EngineError(RuntimeError):
    pass


def library() -> C.CDLL:
    """The loaded CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise EngineError(f"{LIB_PATH} is missing: build the CUDA extension first (make -C {HERE})")
    lib = C.CDLL(LIB_PATH)
    vp, i64, u64, i32 = C.c_void_p, C.c_int64, C.c_uint64, C.c_int
    lib.wg_engine_open.argtypes = [i32, C.POINTER(vp)]
    lib.wg_engine_close.argtypes = [vp]
    lib.wg_engine_close.restype = None
    lib.wg_engine_error.argtypes = [vp]
    lib.wg_engine_error.restype = C.c_char_p
    lib.wg_engine_set_noise_core.argtypes = [vp, i32]
    lib.wg_noise_probe.argtypes = [vp, vp, u64, i32, vp, u64, vp, vp]
    lib.wg_noise_probe_3d.argtypes = [vp, vp, u64, i32, vp, u64, vp, vp]
    lib.wg_parse_version.argtypes = [C.c_char_p, C.POINTER(Opts)]
    lib.wg_parse_preset.argtypes = [C.c_char_p, C.POINTER(Opts)]
    common = [vp, vp, u64, u64, C.POINTER(Opts), i32, i32, i32, i32, i32, i32]
    lib.wg_seed_check.argtypes = common + [vp, u64, C.POINTER(u64), C.POINTER(Stats)]
    lib.wg_seed_check_device.argtypes = common + [vp, u64, C.POINTER(u64), C.POINTER(Stats), vp]
    lib.wg_phase1_codes.argtypes = common + [vp, vp]
    lib.wg_seed_check_noalloc.argtypes = [vp, u64, C.c_uint32, C.POINTER(Opts), i32, i32, i32, i32, i32, i32,
                                          vp, C.c_uint32, C.POINTER(C.c_uint32), vp]
    lib.wg_eval_huts.argtypes = [vp, vp, vp, vp, u64, C.POINTER(Opts), i32, vp]
    lib.wg_grade_scan.argtypes = [vp, i64, C.POINTER(Opts), i32, i32, i32, i32, i32, i32, i32, vp, C.c_int32,
                                  C.POINTER(HutGrade)]
    lib.wg_p2_probe.argtypes = [vp, i64, C.POINTER(Opts), i32, vp, u64, vp]
    lib.wg_deep_starts.argtypes = [vp, vp, i64, u64, i32, i32, i32, i32, vp, u64, C.POINTER(u64)]
    lib.wg_deep_sweep.argtypes = [vp, vp, vp, u64, vp, i64, u64, i32, i32, i32, i32, vp, u64, C.POINTER(u64), vp]
    lib.wg_deep_spots.argtypes = [vp, vp, vp, vp, u64, C.POINTER(Opts), i32, vp, u64, C.POINTER(u64),
                                  C.POINTER(u64)]
    lib.wg_biome_map.argtypes = [vp, i64, C.POINTER(Opts), i64, i64, i32, i32, i32, i32, i32, vp]
    lib.wg_mineshaft_tree.argtypes = [vp, i64, i32, i32, vp, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(i32)]
    lib.wg_finish_rows.argtypes = [vp, vp, vp, vp, u64, vp]
    lib.wg_biome_chunks.argtypes = [vp, i64, C.POINTER(Opts), vp, vp, u64, vp]
    lib.wg_deep_solve.argtypes = [vp, C.POINTER(SolveBundle), u64, u64, u64, vp, u64, C.POINTER(u64),
                                  C.POINTER(SolveStats)]
    lib.wg_deep_solve_tasks.argtypes = [vp, u64, vp, vp, vp, vp, u64, vp, u64, C.POINTER(u64)]
    lib.wg_seed_check_jobs.argtypes = [vp, C.POINTER(Job), u64, vp, u64, C.POINTER(u64), vp, C.POINTER(Stats)]
    lib.wg_server_open.argtypes = [i32, u64, C.POINTER(vp)]
    lib.wg_server_open_config.argtypes = [i32, C.POINTER(ServerConfig), C.POINTER(vp)]
    lib.wg_engine_set_job_queue.argtypes = [vp, i32]
    lib.wg_engine_tune.argtypes = [vp, C.POINTER(TuneReport)]
    lib.wg_engine_set_tuning.argtypes = [vp, vp, u64]
    lib.wg_server_submit.argtypes = [vp, C.POINTER(Job), C.POINTER(u64)]
    lib.wg_server_poll.argtypes = [vp, u64, i32, C.POINTER(JobStatus)]
    lib.wg_server_take.argtypes = [vp, u64, vp, u64, C.POINTER(u64)]
    lib.wg_server_stats.argtypes = [vp, C.POINTER(Stats)]
    lib.wg_server_close.argtypes = [vp]
    lib.wg_server_close.restype = None
    _lib = lib
    return lib


def make_opts(version: str = DEFAULT_VERSION, preset: str = "NORMAL") -> Opts:
    """lysh's --version / --preset names -> option bits (engine/tools/lysh/src/main.c:104-132)."""
    lib = library()
    o = Opts()
    if lib.wg_parse_version(version.encode(), C.byref(o)):
        raise ValueError(f"unknown version {version!r}")
    if lib.wg_parse_preset(preset.encode(), C.byref(o)):
        raise ValueError(f"unknown preset {preset!r}")
    return o


def region_rect_for_area(area_blocks: int) -> tuple[int, int, int, int]:
    """hunt.py ScanRun.rect(): a square about `area` blocks out, in hut regions."""
    r = int(area_blocks // 512) + 1
    return (-r, r, -r, r)


class ScanResult:
    """candidates: CANDIDATE_DTYPE array sorted by (seed_index, rz, rx); stats: the funnel."""

    def __init__(self, candidates: np.ndarray, stats: dict):
        self.candidates = candidates
        self.stats = stats


class Engine:
    """One engine = one device, one stream, one set of work buffers (not thread-safe)."""

    def __init__(self, device: int = 0, noise_core: str = "fp32"):
        lib = library()
        h = C.c_void_p()
        rc = lib.wg_engine_open(device, C.byref(h))
        if rc != WG_OK:
            raise EngineError(f"wg_engine_open(device={device}) failed with status {rc}"
                              + (" (no CUDA device)" if rc == WG_ERR_NODEV else ""))
        self._h = h
        self.device = device
        self.set_noise_core(noise_core)

    def set_noise_core(self, core: str) -> None:
        """'fp32' (FP32 climate samples, FP64 recheck inside the error band; the default), 'fp64',
        'fp32_caves' ('fp32' plus the entrance gate's cave samples in FP32) or 'fp32_recheck_all'
        (the check mode: 'fp32_caves' with every decision re-taken in FP64)."""
        if core not in NOISE_CORES:
            raise ValueError(f"unknown noise core {core!r}")
        rc = library().wg_engine_set_noise_core(self._h, NOISE_CORES[core])
        if rc != WG_OK:
            raise self._err(rc, "wg_engine_set_noise_core")
        self.noise_core = core

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().wg_engine_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, rc: int, what: str) -> EngineError:
        msg = library().wg_engine_error(self._h).decode(errors="replace")
        return EngineError(f"{what} failed with status {rc}: {msg}")

    @staticmethod
    def _seeds(seeds, gen):
        if seeds is not None:
            arr = as_seed_array(seeds)
            return arr, arr.ctypes.data, 0, len(arr)
        if gen is None:
            raise ValueError("give seeds or gen=(base, count)")
        base, count = gen
        return None, None, int(base) & 0xFFFFFFFFFFFFFFFF, int(count)

    def seed_check(self, seeds=None, gen=None, rect=(-4, 5, -4, 5), max_height: int = -50,
                   version: str = DEFAULT_VERSION, preset: str = "NORMAL", salt: int = 0,
                   opts: Opts | None = None) -> ScanResult:
        """Phase-1 survivors of every seed x every region of rect = (rx0, rx1, rz0, rz1)."""
        keep, ptr, base, n = self._seeds(seeds, gen)
        o = opts if opts is not None else make_opts(version, preset)
        # one survivor per 65,536 checks fits the usual floors; a fuller result re-runs once
        cap = min(1 << 26, max(1 << 12, (n * max(0, rect[1] - rect[0]) * max(0, rect[3] - rect[2])) >> 16))
        while True:
            out = np.zeros(cap, CANDIDATE_DTYPE)
            found = C.c_uint64()
            st = Stats()
            rc = library().wg_seed_check(self._h, ptr, base, n, C.byref(o), max_height, salt, *rect,
                                         out.ctypes.data, cap, C.byref(found), C.byref(st))
            if rc != WG_OK:
                raise self._err(rc, "wg_seed_check")
            if found.value <= cap:
                return ScanResult(out[:found.value].copy(), st.as_dict())
            cap = int(found.value)

    def seed_check_device(self, d_seeds_ptr, gen_base: int, n_seeds: int, rect, max_height: int,
                          opts: Opts, d_out_ptr: int, cap: int, stream_ptr: int | None = None,
                          salt: int = 0) -> tuple[int, dict]:
        """Device-buffer variant (raw CUDA pointers, e.g. torch tensor.data_ptr())."""
        found = C.c_uint64()
        st = Stats()
        rc = library().wg_seed_check_device(self._h, d_seeds_ptr, gen_base & 0xFFFFFFFFFFFFFFFF, n_seeds,
                                            C.byref(opts), max_height, salt, *rect, d_out_ptr, cap,
                                            C.byref(found), C.byref(st), stream_ptr)
        if rc != WG_OK:
            raise self._err(rc, "wg_seed_check_device")
        return int(found.value), st.as_dict()

    def noise_probe(self, seeds, noise: str, xz) -> tuple[np.ndarray, np.ndarray]:
        """(fp32, fp64) y = 0 DoublePerlin values of a climate noise, [n_seeds, n_points] float64:
        the FP32 core's value beside the reference's FP64 value at noise-space points xz [n, 2]."""
        s = as_seed_array(seeds)
        pts = np.ascontiguousarray(xz, dtype=np.float64).reshape(-1, 2)
        v32 = np.empty((len(s), len(pts)), np.float64)
        v64 = np.empty((len(s), len(pts)), np.float64)
        rc = library().wg_noise_probe(self._h, s.ctypes.data, len(s), PROBE_NOISES[noise], pts.ctypes.data,
                                      len(pts), v32.ctypes.data, v64.ctypes.data)
        if rc != WG_OK:
            raise self._err(rc, "wg_noise_probe")
        return v32, v64

    def noise_probe_3d(self, seeds, noise: str, xyz) -> tuple[np.ndarray, np.ndarray]:
        """(fp32, fp64) DoublePerlin values of a cave noise of the entrance gate, [n_seeds, n_points]
        float64: the FP32 core's samples summed as the entrance kernel sums them, beside the
        reference's FP64 value at noise-space points xyz [n, 3]."""
        s = as_seed_array(seeds)
        pts = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        v32 = np.empty((len(s), len(pts)), np.float64)
        v64 = np.empty((len(s), len(pts)), np.float64)
        rc = library().wg_noise_probe_3d(self._h, s.ctypes.data, len(s), PROBE_NOISES_3D[noise], pts.ctypes.data,
                                         len(pts), v32.ctypes.data, v64.ctypes.data)
        if rc != WG_OK:
            raise self._err(rc, "wg_noise_probe_3d")
        return v32, v64

    def phase1_codes(self, seeds=None, gen=None, rect=(-4, 5, -4, 5), max_height: int = -50,
                     version: str = DEFAULT_VERSION, preset: str = "NORMAL", salt: int = 0,
                     opts: Opts | None = None) -> tuple[np.ndarray, np.ndarray]:
        """(codes, tiers), each [n_seeds, n_regions] int8: lysh's per-region phase-1 verdicts."""
        keep, ptr, base, n = self._seeds(seeds, gen)
        o = opts if opts is not None else make_opts(version, preset)
        nreg = (rect[1] - rect[0]) * (rect[3] - rect[2])
        codes = np.empty((n, nreg), np.int8)
        tiers = np.empty((n, nreg), np.int8)
        rc = library().wg_phase1_codes(self._h, ptr, base, n, C.byref(o), max_height, salt, *rect,
                                       codes.ctypes.data, tiers.ctypes.data)
        if rc != WG_OK:
            raise self._err(rc, "wg_phase1_codes")
        return codes, tiers

    def eval_huts(self, seeds, hut_x, hut_z, max_y: int = -50, version: str = DEFAULT_VERSION,
                  preset: str = "NORMAL", opts: Opts | None = None) -> np.ndarray:
        """Phase 2 (lysh_eval_hut) for each (seed, hut_x, hut_z): a HUT_DTYPE array."""
        s = as_seed_array(seeds)
        hx = np.ascontiguousarray(hut_x, dtype=np.int32)
        hz = np.ascontiguousarray(hut_z, dtype=np.int32)
        if not (len(s) == len(hx) == len(hz)):
            raise ValueError("seeds, hut_x and hut_z differ in length")
        o = opts if opts is not None else make_opts(version, preset)
        out = np.zeros(len(s), HUT_DTYPE)
        rc = library().wg_eval_huts(self._h, s.ctypes.data, hx.ctypes.data, hz.ctypes.data, len(s), C.byref(o),
                                    max_y, out.ctypes.data)
        if rc != WG_OK:
            raise self._err(rc, "wg_eval_huts")
        return out

    def grade_scan(self, seed: int, rect, max_height: int = -50, max_y: int = -50, version: str = DEFAULT_VERSION,
                   preset: str = "NORMAL", salt: int = 0, cap: int = 4096,
                   opts: Opts | None = None) -> tuple[np.ndarray, dict]:
        """Phase 1 + phase 2 over rect for one seed (lysh_grade_scan): (hits [n, 12] int32, counts)."""
        o = opts if opts is not None else make_opts(version, preset)
        hits = np.zeros((cap, GRADE_INTS), np.int32)
        g = HutGrade()
        rc = library().wg_grade_scan(self._h, to_signed(int(seed)), C.byref(o), max_height, *rect, salt, max_y,
                                     hits.ctypes.data, cap, C.byref(g))
        if rc != WG_OK:
            raise self._err(rc, "wg_grade_scan")
        counts = {k: getattr(g, k) for k, _ in HutGrade._fields_}
        return hits[:g.hits_written].copy(), counts

    def deep_starts(self, s48=None, base: int = 0, count: int = 0, rect=(-64, 64, -64, 64)) -> np.ndarray:
        """Deep Dive region walk: huts on mineshaft start chunks (DEEP_START_DTYPE, sorted by
        (seed_index, rz, rx))."""
        if s48 is not None:
            arr = np.ascontiguousarray(np.asarray([int(v) & 0xFFFFFFFFFFFF for v in s48], dtype=np.int64))
            ptr, n = arr.ctypes.data, len(arr)
        else:
            arr, ptr, n = None, None, int(count)
        # about 0.4 % of hut chunks are start chunks: room for 1 in 200 avoids a second walk
        regions = max(0, rect[1] - rect[0]) * max(0, rect[3] - rect[2])
        cap = min(1 << 24, max(1 << 12, n * regions // 200))
        while True:
            out = np.zeros(cap, DEEP_START_DTYPE)
            found = C.c_uint64()
            rc = library().wg_deep_starts(self._h, ptr, int(base), n, *rect, out.ctypes.data, cap, C.byref(found))
            if rc != WG_OK:
                raise self._err(rc, "wg_deep_starts")
            if found.value <= cap:
                return out[:found.value]   # a view: the hits are already in order, no second copy
            cap = int(found.value)

    def deep_sweep(self, layouts, values=None, s48=None, base: int = 0, count: int = 0,
                   rect=WORLD_REGIONS) -> tuple[np.ndarray, np.ndarray]:
        """Deep Dive forward sweep with the layout-catalogue probe: (matches SWEEP_MATCH_DTYPE sorted by
        (seed_index, rz, rx), starts per structure seed uint64)."""
        keys = np.ascontiguousarray([int(v) & 0xFFFFFFFFFFFF for v in layouts], dtype=np.uint64)
        vals = None if values is None else np.ascontiguousarray(values, dtype=np.uint32)
        if s48 is not None:
            arr = np.ascontiguousarray(np.asarray([int(v) & 0xFFFFFFFFFFFF for v in s48], dtype=np.int64))
            ptr, n = arr.ctypes.data, len(arr)
        else:
            arr, ptr, n = None, None, int(count)
        cap = 1 << 12
        starts = np.zeros(n, np.uint64)
        while True:
            out = np.zeros(cap, SWEEP_MATCH_DTYPE)
            found = C.c_uint64()
            rc = library().wg_deep_sweep(self._h, keys.ctypes.data, None if vals is None else vals.ctypes.data,
                                         len(keys), ptr, int(base), n, *rect, out.ctypes.data, cap, C.byref(found),
                                         starts.ctypes.data)
            if rc != WG_OK:
                raise self._err(rc, "wg_deep_sweep")
            if found.value <= cap:
                return out[:found.value].copy(), starts
            cap = int(found.value)

    def mineshaft_tree(self, ws: int, chunk_x: int, chunk_z: int) -> tuple[np.ndarray, int]:
        """wg_mineshaft_tree: (pieces MS_PIECE_DTYPE in mstree's order, the room's floor y)."""
        out = np.zeros(512, MS_PIECE_DTYPE)
        n, floor = C.c_uint32(), C.c_int()
        rc = library().wg_mineshaft_tree(self._h, _signed64(ws), chunk_x, chunk_z, out.ctypes.data, len(out),
                                         C.byref(n), C.byref(floor))
        if rc != WG_OK:
            raise self._err(rc, "wg_mineshaft_tree")
        return out[:n.value].copy(), int(floor.value)

    def finish_rows(self, ws, chunk_x, chunk_z) -> np.ndarray:
        """wg_finish_rows: FINISH_DTYPE per survivor (world seed, hut chunk)."""
        s = np.ascontiguousarray(np.asarray([_signed64(v) for v in ws], dtype=np.int64))
        cx = np.ascontiguousarray(chunk_x, dtype=np.int32)
        cz = np.ascontiguousarray(chunk_z, dtype=np.int32)
        if not (len(s) == len(cx) == len(cz)):
            raise ValueError("ws, chunk_x, chunk_z differ in length")
        out = np.zeros(len(s), FINISH_DTYPE)
        rc = library().wg_finish_rows(self._h, s.ctypes.data, cx.ctypes.data, cz.ctypes.data, len(s), out.ctypes.data)
        if rc != WG_OK:
            raise self._err(rc, "wg_finish_rows")
        return out

    def biome_map(self, seed: int, x0: int, z0: int, w: int, h: int, step: int = 16, ss: int = 1,
                  version: str = "26.3", y: int = 63) -> np.ndarray:
        """wg_biome_map: (h, w) biome ids, as biome_map --seed ... writes them."""
        o = Opts()
        if library().wg_parse_version(version.encode(), C.byref(o)) != WG_OK:
            raise ValueError(f"unknown version {version!r}")
        out = np.zeros((h, w), np.uint8)
        rc = library().wg_biome_map(self._h, to_signed(seed), C.byref(o), x0, z0, w, h, step, ss, y, out.ctypes.data)
        if rc != WG_OK:
            raise self._err(rc, "wg_biome_map")
        return out

    def biome_chunks(self, seed: int, cx, cz, version: str = "26.3") -> np.ndarray:
        """wg_biome_chunks: the witch-hut test's biome at each chunk (biome_map --stdin)."""
        o = Opts()
        if library().wg_parse_version(version.encode(), C.byref(o)) != WG_OK:
            raise ValueError(f"unknown version {version!r}")
        x = np.ascontiguousarray(np.asarray(cx, dtype=np.int32))
        z = np.ascontiguousarray(np.asarray(cz, dtype=np.int32))
        out = np.zeros(len(x), np.uint8)
        rc = library().wg_biome_chunks(self._h, to_signed(seed), C.byref(o), x.ctypes.data, z.ctypes.data, len(x),
                                       out.ctypes.data)
        if rc != WG_OK:
            raise self._err(rc, "wg_biome_chunks")
        return out

    def deep_solve(self, bundles, first_group: int, n_groups: int) -> tuple[np.ndarray, dict]:
        """wg_deep_solve: bundles = [(layout, "XZ" regime digits or (rx, rz), "odd" | "u2" | "eq"), ...]
        (plan lines); the hits of groups [first_group, first_group + n_groups)."""
        arr = (SolveBundle * len(bundles))()
        for i, (x, regime, tier) in enumerate(bundles):
            rg = (int(regime[0]), int(regime[1]))
            arr[i] = SolveBundle(int(x) & 0xFFFFFFFFFFFF, rg[0], rg[1], SOLVE_TIERS.get(tier, tier) if isinstance(tier, str) else int(tier), 0)
        cap = max(1 << 12, 2048 * n_groups)
        while True:
            out = np.zeros(cap, SOLVE_HIT_DTYPE)
            n = C.c_uint64()
            st = SolveStats()
            rc = library().wg_deep_solve(self._h, arr, len(bundles), first_group, n_groups, out.ctypes.data, cap,
                                         C.byref(n), C.byref(st))
            if rc != WG_OK:
                raise self._err(rc, "wg_deep_solve")
            if n.value <= cap:
                return out[:n.value].copy(), {k: getattr(st, k) for k, _ in SolveStats._fields_}
            cap = int(n.value)

    def deep_solve_tasks(self, layout: int, rx, rz, ox, oz) -> np.ndarray:
        """wg_deep_solve_tasks: hits of explicit (region, chunk offset) tasks; group = task index."""
        a = [np.ascontiguousarray(np.asarray(v, dtype=np.int32)) for v in (rx, rz, ox, oz)]
        n = len(a[0])
        cap = max(1 << 10, 4 * n)
        while True:
            out = np.zeros(cap, SOLVE_HIT_DTYPE)
            got = C.c_uint64()
            rc = library().wg_deep_solve_tasks(self._h, int(layout) & 0xFFFFFFFFFFFF, *(v.ctypes.data for v in a), n,
                                               out.ctypes.data, cap, C.byref(got))
            if rc != WG_OK:
                raise self._err(rc, "wg_deep_solve_tasks")
            if got.value <= cap:
                return out[:got.value].copy()
            cap = int(got.value)

    def seed_check_jobs(self, jobs) -> tuple[list[np.ndarray], dict]:
        """wg_seed_check_jobs: many jobs (dicts with seeds= or gen=(base, count), rect=, max_height=,
        and version= / preset= / opts= / salt=) flattened into shared batches.  Returns each job's
        survivors (CANDIDATE_DTYPE, seed_index = position in the job) and the funnel."""
        arr = (Job * max(len(jobs), 1))()
        keep = [_fill_job(arr[i], j) for i, j in enumerate(jobs)]
        per = np.zeros(max(len(jobs), 1), np.uint64)
        # room for one survivor per 65,536 checks (about 500 x the rate at floor -50), so the
        # call normally runs once; a fuller result re-runs it with the exact size
        checks = sum(int(arr[i].n_seeds) * (arr[i].rx1 - arr[i].rx0) * (arr[i].rz1 - arr[i].rz0)
                     for i in range(len(jobs)))
        cap = min(1 << 26, max(1 << 12, checks >> 16))
        while True:
            out = np.zeros(cap, CANDIDATE_DTYPE)
            found = C.c_uint64()
            st = Stats()
            rc = library().wg_seed_check_jobs(self._h, arr, len(jobs), out.ctypes.data, cap, C.byref(found),
                                              per.ctypes.data, C.byref(st))
            if rc != WG_OK:
                raise self._err(rc, "wg_seed_check_jobs")
            if found.value <= cap:
                break
            cap = int(found.value)
        del keep
        bounds = np.concatenate([[0], np.cumsum(per[:len(jobs)].astype(np.int64))])
        return [out[bounds[i]:bounds[i + 1]].copy() for i in range(len(jobs))], st.as_dict()

    def set_job_queue(self, device_queue: bool) -> None:
        """seed_check_jobs through the device work queue (True, the default) or the host batch loop."""
        rc = library().wg_engine_set_job_queue(self._h, 1 if device_queue else 0)
        if rc != WG_OK:
            raise self._err(rc, "wg_engine_set_job_queue")

    def tune(self) -> dict:
        """wg_engine_tune: times the job settings' candidates on this GPU and keeps the fastest."""
        r = TuneReport()
        rc = library().wg_engine_tune(self._h, C.byref(r))
        if rc != WG_OK:
            raise self._err(rc, "wg_engine_tune")
        return r.as_dict()

    def set_tuning(self, windows=None, budget: int = 0) -> None:
        """wg_engine_set_tuning: regions per unit per job class (None = the default rule) and checks
        per queue slice (0 = the default)."""
        w = None if windows is None else (C.c_uint32 * 4)(*[int(v) for v in windows])
        rc = library().wg_engine_set_tuning(self._h, None if w is None else C.cast(w, C.c_void_p), int(budget))
        if rc != WG_OK:
            raise self._err(rc, "wg_engine_set_tuning")

    def deep_spots(self, s48, chunk_x, chunk_z, max_height: int = -54, version: str = DEFAULT_VERSION,
                   preset: str = "NORMAL", opts: Opts | None = None) -> tuple[np.ndarray, int]:
        """Deep Dive terrain stage: (survivors CANDIDATE_DTYPE with seed_index = spot * 65536 + u,
        number of spots that are not mineshaft start chunks)."""
        s = np.ascontiguousarray(np.asarray([int(v) & 0xFFFFFFFFFFFF for v in s48], dtype=np.int64))
        cx = np.ascontiguousarray(chunk_x, dtype=np.int32)
        cz = np.ascontiguousarray(chunk_z, dtype=np.int32)
        o = opts if opts is not None else make_opts(version, preset)
        cap = 1 << 12
        while True:
            out = np.zeros(cap, CANDIDATE_DTYPE)
            found, bad = C.c_uint64(), C.c_uint64()
            rc = library().wg_deep_spots(self._h, s.ctypes.data, cx.ctypes.data, cz.ctypes.data, len(s), C.byref(o),
                                         max_height, out.ctypes.data, cap, C.byref(found), C.byref(bad))
            if rc != WG_OK:
                raise self._err(rc, "wg_deep_spots")
            if found.value <= cap:
                return out[:found.value].copy(), int(bad.value)
            cap = int(found.value)

    def p2_probe(self, seed: int, kind, xyz, version: str = DEFAULT_VERSION, preset: str = "NORMAL",
                 opts: Opts | None = None) -> np.ndarray:
        """Phase-2 parity probes (wg_p2_probe) at block points xyz [n, 3]."""
        k = PROBE_KINDS[kind] if isinstance(kind, str) else int(kind)
        pts = np.ascontiguousarray(np.asarray(xyz, dtype=np.int32).reshape(-1, 3))
        o = opts if opts is not None else make_opts(version, preset)
        out = np.zeros(len(pts), np.float64)
        rc = library().wg_p2_probe(self._h, to_signed(int(seed)), C.byref(o), k, pts.ctypes.data, len(pts),
                                   out.ctypes.data)
        if rc != WG_OK:
            raise self._err(rc, "wg_p2_probe")
        return out


def as_seed_array(seeds) -> np.ndarray:
    """Seeds as contiguous int64 (Java longs); accepts signed or unsigned 64-bit spellings."""
    if isinstance(seeds, np.ndarray) and seeds.dtype in (np.int64, np.uint64):
        return np.ascontiguousarray(seeds).view(np.int64)
    return np.array([int(s) & 0xFFFFFFFFFFFFFFFF for s in seeds], dtype=np.uint64).view(np.int64)


def splitmix64(x: int) -> int:
    """The --seed-gen stream: splitmix64(base + i) with the golden-gamma pre-add."""
    m = 0xFFFFFFFFFFFFFFFF
    x = (x + 0x9E3779B97F4A7C15) & m
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31)


def to_signed(v: int) -> int:
    v &= 0xFFFFFFFFFFFFFFFF
    return v - (1 << 64) if v >= (1 << 63) else v


def shard(n_total: int, rank: int, world: int) -> tuple[int, int]:
    """Seed-index range [lo, hi) of rank `rank` out of `world`: contiguous, disjoint, covering
    [0, n_total), sizes differing by at most one.  Seeds are independent units, so a
    multi-GPU run shards seeds with no exchange beyond concatenating survivor lists."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    return (n_total * rank) // world, (n_total * (rank + 1)) // world


def seed_check_noalloc(d_seeds_ptr, gen_base: int, n_seeds: int, rect, max_height: int, opts: Opts,
                       d_out_ptr: int, cap: int, stream_ptr: int | None = None, salt: int = 0) -> int:
    """wg_seed_check_noalloc on the current CUDA device: no engine, no device allocation (the work
    lists live in the library's fixed scratch array).  Returns the number of survivors."""
    n = C.c_uint32()
    rc = library().wg_seed_check_noalloc(d_seeds_ptr, gen_base & 0xFFFFFFFFFFFFFFFF, n_seeds, C.byref(opts),
                                         max_height, salt, *rect, d_out_ptr, cap, C.byref(n), stream_ptr)
    if rc != WG_OK:
        raise EngineError(f"wg_seed_check_noalloc failed with status {rc}")
    return int(n.value)


@functools.lru_cache(maxsize=64)
def _cached_opts(version: str, preset: str) -> Opts:
    return make_opts(version, preset)


def _fill_job(dst: Job, job: dict):
    """Fills a wg_job from a job dict; returns the seed array the struct points into."""
    keep, ptr, base, n = Engine._seeds(job.get("seeds"), job.get("gen"))
    rect = job.get("rect", (-4, 5, -4, 5))
    o = job.get("opts") or _cached_opts(job.get("version", DEFAULT_VERSION), job.get("preset", "NORMAL"))
    dst.seeds = ptr
    dst.gen_base = base
    dst.n_seeds = n
    dst.rx0, dst.rx1, dst.rz0, dst.rz1 = (int(v) for v in rect)
    dst.max_height = int(job.get("max_height", -50))
    dst.salt = int(job.get("salt", 0))
    dst.opts = o
    return keep


class Server:
    """wg_server: a job server on one device.  submit() queues a job and returns at once; the
    library's worker thread admits queued jobs as device seed slots free up and runs them in
    shared batches; poll() / take() return a job's status and survivors."""

    def __init__(self, device: int = 0, max_queued_seeds: int = 0, arena_seeds: int = 0, batch_checks: int = 0,
                 fail_job: int = 0):
        lib = library()
        h = C.c_void_p()
        cfg = ServerConfig(max_queued_seeds, arena_seeds, batch_checks, fail_job)
        rc = lib.wg_server_open_config(device, C.byref(cfg), C.byref(h))
        if rc != WG_OK:
            raise EngineError(f"wg_server_open_config(device={device}) failed with status {rc}")
        self._h = h

    def submit(self, **job) -> int:
        j = Job()
        keep = _fill_job(j, job)
        jid = C.c_uint64()
        rc = library().wg_server_submit(self._h, C.byref(j), C.byref(jid))
        del keep
        if rc != WG_OK:
            raise EngineError(f"wg_server_submit failed with status {rc}")
        return int(jid.value)

    def poll(self, job_id: int, wait_ms: int = 0) -> dict:
        st = JobStatus()
        rc = library().wg_server_poll(self._h, job_id, wait_ms, C.byref(st))
        if rc != WG_OK:
            raise EngineError(f"wg_server_poll({job_id}) failed with status {rc}")
        return {"done": bool(st.done), "status": st.status, "found": st.found, "queue_ms": st.queue_ms,
                "latency_ms": st.latency_ms, "batch_jobs": st.batch_jobs}

    def wait(self, job_id: int, timeout_s: float = 600.0) -> dict:
        import time
        end = time.monotonic() + timeout_s
        while True:
            st = self.poll(job_id, 200)
            if st["done"]:
                return st
            if time.monotonic() > end:
                raise EngineError(f"job {job_id} not done after {timeout_s} s")

    def take(self, job_id: int) -> np.ndarray:
        cap = 1 << 10
        while True:
            out = np.zeros(cap, CANDIDATE_DTYPE)
            n = C.c_uint64()
            rc = library().wg_server_take(self._h, job_id, out.ctypes.data, cap, C.byref(n))
            if rc != WG_OK:
                raise EngineError(f"wg_server_take({job_id}) failed with status {rc}")
            if n.value <= cap:
                return out[:n.value].copy()
            cap = int(n.value)

    def stats(self) -> dict:
        st = Stats()
        rc = library().wg_server_stats(self._h, C.byref(st))
        if rc != WG_OK:
            raise EngineError(f"wg_server_stats failed with status {rc}")
        return st.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().wg_server_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------------------------
# Synthetic job streams (the reference measures on no public dataset).  Every draw is one step
# of the splitmix64 stream x_k = splitmix64(base + k), k = 0, 1, 2, ...; U(x) = (x >> 11) * 2^-53.
# ---------------------------------------------------------------------------------------------

def _u01(x: int) -> float:
    return (x >> 11) * (1.0 / (1 << 53))


def splitmix64_array(base: int, count: int) -> np.ndarray:
    """splitmix64(base + i) for i < count, vectorised (uint64 wrap-around arithmetic)."""
    with np.errstate(over="ignore"):
        x = (np.uint64(base & 0xFFFFFFFFFFFFFFFF) + np.arange(count, dtype=np.uint64)) + np.uint64(0x9E3779B97F4A7C15)
        z = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return (z ^ (z >> np.uint64(31))).view(np.int64)


def uneven_jobs(n_jobs: int = 65536, base: int = 3, max_seeds: int = 4096, max_radius: int = 64) -> list[dict]:
    """The uneven batched-jobs workload.  Per job, four draws then its seeds:
    n = floor((max_seeds + 1) ** U) seeds (log-uniform 1..max_seeds), radius r = floor((max_radius + 1) ** U)
    (1..max_radius, rect [-r, r + 1)^2), floor g = -50 - (x mod 5), mode = x & 1 (1 = "or lower",
    0 = "exactly": phase 1 gates on maxHeight = g in both modes), then the n seeds are the next n
    values of the stream."""
    jobs = []
    k = 0
    for _ in range(n_jobs):
        x = [splitmix64(base + k + i) for i in range(4)]
        k += 4
        n = max(1, min(max_seeds, int((max_seeds + 1) ** _u01(x[0]))))
        r = max(1, min(max_radius, int((max_radius + 1) ** _u01(x[1]))))
        g = -50 - (x[2] % 5)
        jobs.append({"seeds": splitmix64_array(base + k, n), "rect": (-r, r + 1, -r, r + 1), "max_height": g,
                     "mode": "or_lower" if x[3] & 1 else "exactly"})
        k += n
    return jobs


def serving_requests(n_req: int, rate_per_s: float, base: int = 5, max_seeds: int = 10 ** 6,
                     max_radius: int = 32) -> list[dict]:
    """The serving workload: Poisson arrivals at rate_per_s.  Per request, four draws: the
    inter-arrival gap -ln(1 - U) / rate, n = floor((max_seeds + 1) ** U) seeds, radius
    r = floor((max_radius + 1) ** U), floor g = -50 - (x mod 5); the seeds are
    splitmix64(gen_base + i) with gen_base the request's last draw (a generator job)."""
    import math
    reqs = []
    t = 0.0
    for i in range(n_req):
        x = [splitmix64(base + 4 * i + q) for q in range(4)]
        t += -math.log(1.0 - _u01(x[0])) / rate_per_s
        n = max(1, min(max_seeds, int((max_seeds + 1) ** _u01(x[1]))))
        r = max(1, min(max_radius, int((max_radius + 1) ** _u01(x[2]))))
        reqs.append({"t": t, "gen": (x[3], n), "rect": (-r, r + 1, -r, r + 1), "max_height": -50 - (x[3] % 5)})
    return reqs
