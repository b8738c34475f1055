"""Seed Check benchmark (config 2: 2^24 splitmix64(2 + i) world seeds x 9x9 swamp-hut regions,
phase-1 gate at floor -50, version rules 1.19.x~26.1).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = the whole phase-1 Seed Check of one rank's 2^24 seeds (1.36e9 (seed, region)
checks).  Multi-GPU runs shard seeds (weak scaling: every rank checks its own 2^24 seeds of
the stream); the only exchange is a max-reduce of the timings.  Prints one JSON line.

`value` is measured with the seeds already resident in HBM (wg_seed_check_device on torch's
stream, CUDA events around each step); `e2e` goes through the public host API
(wg_seed_check) with the seeds in pinned host memory, so the host->device copy of the seeds and
the device->host read of the survivors are inside the timed region.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
N_SEEDS = 1 << 24
RECT = (-4, 5, -4, 5)
MAX_HEIGHT = -50
VERSION = "1.19.x~26.1"
GEN_BASE = 2
METRIC = "seeds/s"


def load_package():
    name = "low_witch_finder_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "low-witch-finder_b200", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


# ------------------------------------------------------------------------------------------
# algorithmic work model of the phase-1 kernels (lane-operations, counted from the source)
# ------------------------------------------------------------------------------------------
OPS_PERLIN_BUILD = 7160      # 259 Xoroshiro128++ steps, 256 Lemire draws + byte swaps, RNG derivation
OPS_Y0_SAMPLE = 244          # FP64 y=0 sample: 14 table lookups, 62 FP64 ops (x2 issue slots), bit-op gradients
# FP32-core y=0 sample: 14 table lookups (x4), the FP64 coordinate reduction (16 FP64 ops x2 issue
# slots), 24 gradient-component loads, 51 FP32 ops (3 offsets, 8 gradients x3, 2 fades x5, 7 lerps x2)
# and the FMA into the running sum
OPS_Y0_SAMPLE_F32 = 56 + 32 + 24 + 51 + 1
# 3-D FP64 sample of the cave noises: 14 lookups (x4), 96 FP64 ops (x2), 24 gradient-component loads
OPS_3D_SAMPLE = 56 + 192 + 24
# the same in the FP32 core: 14 lookups (x4), the FP64 coordinate scaling and reduction (27 FP64 ops
# x2), 24 gradient-component loads, 56 FP32 ops (3 offsets, 8 gradients x3, 3 fades x5, 7 lerps x2)
OPS_3D_SAMPLE_F32 = 56 + 54 + 24 + 56
OPS_REGION = 40              # java.util.Random placement (2 x nextInt(24)) + coordinates
# dram__bytes_read.sum + dram__bytes_write.sum per launch, from ncu on `bench.py --profile 1048576`
# (one launch of each kernel on 2^20 seeds read from a list in HBM; a 2^24-seed step runs 16 such
# launches, each over its own 2^20 seeds, so the per-launch figure is the full step's per launch)
TRAFFIC = {"climate_kernel": 8473088 + 256, "entrance_kernel": 20939520 + 0,
           "source": "climate: ncu --set full --clock-control none -k regex:climate_kernel -s 1 -c 1 python bench.py "
                     "--profile 1048576 --warmup 1 --steps 1; entrance: ncu --metrics "
                     "dram__bytes_read.sum,dram__bytes_write.sum --clock-control none -k "
                     "regex:'climate_kernel|entrance_kernel|ladder_kernel' -s 3 -c 3 python bench.py --profile "
                     "1048576 --warmup 1 --steps 1 (the timed step's launch; read + write bytes)"}
# ncu pipe utilisation of the same launches (the --set full captures of one climate and one entrance
# launch on 2^20 seeds kept under profiles/): the counters behind the issue-rate roofline.  The integer
# ALU pipe issues 64 lanes per clock per SM, half the 128-lane issue rate the roofline divides by,
# and carries most of the table builds.
PIPES = {"climate_kernel": {"issue_active": 0.667, "alu": 0.589, "fma": 0.226, "fp64": 0.021,
                            "shared_wavefronts": 0.736, "warps_active": 0.275},
         "entrance_kernel": {"issue_active": 0.574, "alu": 0.553, "fma": 0.153, "fp64": 0.079,
                             "shared_wavefronts": 0.723, "warps_active": 0.278},
         "unit": "fraction of peak, ncu --set full of one launch on 2^20 seeds"}
BYTES_PER_SEED_IN = 8        # the int64 seed read from HBM
BYTES_PER_RECORD = 12        # (unit, offset, count) per seed with climate survivors
BYTES_PER_SURVIVOR = 4       # region offset per climate survivor


def climate_work(st: dict, n_seeds: int, n_regions: int, fp32: bool) -> tuple[float, float]:
    """(lane-ops, algorithmic bytes) of the climate kernel over a request, from its funnel."""
    th = st["tier_hist"]
    rh = st["reject_hist"]
    y0 = sum((t + 2) * th[t] for t in range(7)) + 12 * rh[1] + 18 * (rh[2] + st["climate_survivors"])
    ops = (18 * n_seeds * OPS_PERLIN_BUILD + y0 * (OPS_Y0_SAMPLE_F32 if fp32 else OPS_Y0_SAMPLE)
           + n_seeds * n_regions * OPS_REGION)
    nbytes = n_seeds * BYTES_PER_SEED_IN + st["climate_survivors"] * BYTES_PER_SURVIVOR
    return float(ops), float(nbytes)


def entrance_work(st: dict, fp32: bool) -> float:
    """Lane-ops of the entrance kernel: 18 tables per record (a seed unit with climate survivors),
    36 3-D samples per survivor (18 slots at y = 50 and 60) plus its 12 octave sums and decision."""
    n_rec, n_surv = st["records"], st["climate_survivors"]
    sample = OPS_3D_SAMPLE_F32 if fp32 else OPS_3D_SAMPLE
    return float(n_rec * 18 * OPS_PERLIN_BUILD + n_surv * (36 * sample + 12 * 40 + 120))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows: list[list[str]] = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(n_sample: int) -> dict:
    """The reference's own lysh (oracle/_ref, compiled from its sources) on the host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bind
    wg = load_package()
    seeds = np.array([wg.splitmix64(GEN_BASE + i) for i in range(n_sample)], dtype=np.uint64)
    r = bind.rules(VERSION)
    cores = os.cpu_count() or 1
    if os.path.exists(bind.REF_LIB):
        ref = bind.Ref()
        secs, _ = ref.phase1_seeds(seeds, r, MAX_HEIGHT, RECT, threads=cores)
        kind = "reference"
    else:
        port = bind.Port()
        t0 = time.perf_counter()
        port.scan_seeds(r, MAX_HEIGHT, RECT, seeds=seeds, threads=cores)
        secs = time.perf_counter() - t0
        kind = "port"
    out = {"value": n_sample / secs, "unit": METRIC, "cores": cores, "kind": kind,
           "sample": f"first {n_sample} seeds of config 2 (splitmix64(2 + i)), 9x9 regions, lysh phase-1 scan "
                     f"(lysh_scan_rect per seed, one seed per thread)", "seconds": secs}
    if os.path.exists(bind.REF_BIN):
        out["process_per_seed"] = process_per_seed_baseline(bind.REF_BIN, seeds[:256], cores)
    return out


def process_per_seed_baseline(lysh: str, seeds, cores: int) -> dict:
    """The mode hunt.py's CPU scan uses (hunt.py:1390-1392): one `lysh scan` process per seed (phase 1
    and lysh's own phase 2 at the ceiling, hits listed), here with `cores` processes at a time."""
    import subprocess
    from concurrent.futures import ThreadPoolExecutor
    rect = [str(v) for v in (RECT[0], RECT[1], RECT[2], RECT[3])]

    def one(seed):
        cmd = [lysh, "scan", "--seed", str(int(seed)), "--rx0", rect[0], "--rx1", rect[1], "--rz0", rect[2],
               "--rz1", rect[3], "--threads", "1", "--max-y", str(MAX_HEIGHT), "--phase2-max-y", str(MAX_HEIGHT),
               "--version", VERSION, "--list", "--no-stats"]
        return subprocess.run(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL).returncode

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=cores) as ex:
        rcs = list(ex.map(one, seeds))
    secs = time.perf_counter() - t0
    return {"value": len(seeds) / secs, "unit": METRIC, "cores": cores, "failed": sum(1 for r in rcs if r),
            "sample": f"first {len(seeds)} seeds of config 2, one `lysh scan --list --no-stats` process per seed "
                      f"(hunt.py's CPU mode), {cores} at a time", "seconds": secs}


def phase2_measure(eng, cands, opts, cpu: bool) -> dict:
    """Phase 2 (lysh_eval_hut: biome gate, aquifer flood, carvers, footprint heights) of the step's
    phase-1 survivors through wg_eval_huts, host buffers in and out (wall clock, 3 timed calls
    after one warm-up); beside it the reference lysh on one host core for the same huts."""
    if len(cands) == 0:
        return {"huts": 0}
    seeds = cands["seed"]
    hx = cands["chunk_x"].astype(np.int64) * 16
    hz = cands["chunk_z"].astype(np.int64) * 16
    eng.eval_huts(seeds[:8], hx[:8], hz[:8], max_y=MAX_HEIGHT, opts=opts)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        res = eng.eval_huts(seeds, hx, hz, max_y=MAX_HEIGHT, opts=opts)
        times.append(time.perf_counter() - t0)
    secs = statistics.median(times)
    out = {"huts": int(len(cands)), "unit": "huts/s", "value": len(cands) / secs, "ms": 1e3 * secs,
           "accepted": int(res["ok"].sum()), "rejected_biome": int((res["reject"] == 3).sum()),
           "rejected_flood": int((res["reject"] == 2).sum()), "rejected_y": int((res["reject"] == 1).sum()),
           "timing": "wall clock around wg_eval_huts (host arrays in and out), median of 3"}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import bind
        if os.path.exists(bind.REF_LIB):
            ref = bind.Ref()
            r = bind.rules(VERSION)
            n = min(64, len(cands))
            t0 = time.perf_counter()
            for i in range(n):
                with ref.ctx(int(seeds[i]), r, MAX_HEIGHT, 0) as ctx:
                    ctx.eval_hut(int(hx[i]), int(hz[i]), MAX_HEIGHT)
            dt = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": n / dt, "unit": "huts/s", "cores": 1, "kind": "reference",
                                   "sample": f"first {n} huts: lysh_search_ctx_init + lysh_eval_hut per hut"}
    return out


# hunt.py's per-seed GPU workload: one world seed over every swamp-hut region of the +-30M world
# (hunt.py:72 WORLD = [-58594, 58594) in both axes) at floor -50; the seed is hunt.py's
# SCAN_REFERENCE (hunt.py:86), whose hut is chunk (-987, -1073)
WHOLE_WORLD_SEED = 1473884015873122059
WHOLE_WORLD_RECT = (-58594, 58594, -58594, 58594)


def whole_world_measure(eng, opts) -> dict:
    """One seed over the whole world through wg_seed_check (host API, survivors back to the host),
    wall clock around the call after one warm-up call on a small rect."""
    eng.seed_check(seeds=[WHOLE_WORLD_SEED], rect=(-64, 64, -64, 64), max_height=MAX_HEIGHT, opts=opts)
    t0 = time.perf_counter()
    res = eng.seed_check(seeds=[WHOLE_WORLD_SEED], rect=WHOLE_WORLD_RECT, max_height=MAX_HEIGHT, opts=opts)
    secs = time.perf_counter() - t0
    r = WHOLE_WORLD_RECT
    n = (r[1] - r[0]) * (r[3] - r[2])
    got = {(int(c["chunk_x"]), int(c["chunk_z"])) for c in res.candidates}
    return {"seed": WHOLE_WORLD_SEED, "rect": list(r), "regions": n, "seconds": secs, "checks_per_s": n / secs,
            "phase1_survivors": len(res.candidates), "reference_hut_found": (-987, -1073) in got,
            "gpu_ms": res.stats.get("gpu_ms") if isinstance(res.stats, dict) else None,
            "reference": "the reference's GPU stage on this workload: 58.4 s on a 20-SM laptop GPU "
                         "(docs/HUNT54.txt), about 9.7 s per seed on a 188-SM GPU "
                         "(docs/OPTIMIZATION_NOTES.txt as docs/HUNT54.txt quotes it)",
            "timing": "wall clock around wg_seed_check (host seed in, phase-1 survivors out)"}


def deep_measure(eng, opts) -> dict:
    """Deep Dive: the region walk (structure seeds x regions -> huts on mineshaft start chunks)
    and the terrain stage (each spot's 65,536 upper-bit world seeds through phase 1 at -54),
    wall clock around the public calls after one warm-up, the median of three calls each, so one
    host stall does not set a figure."""

    def median_wall(fn, reps=3):
        times, out = [], None
        for _ in range(reps):
            t0 = time.perf_counter()
            out = fn()
            times.append(time.perf_counter() - t0)
        return out, sorted(times)[reps // 2]

    rect = (-2048, 2048, -2048, 2048)
    n_s48 = 16
    eng.deep_starts(base=1, count=1, rect=(-64, 64, -64, 64))
    hits, walk_s = median_wall(lambda: eng.deep_starts(base=0x5EED0000, count=n_s48, rect=rect))
    regions = n_s48 * (rect[1] - rect[0]) * (rect[3] - rect[2])
    spots = hits[:256]
    eng.deep_spots(spots["s48"][:2], spots["chunk_x"][:2], spots["chunk_z"][:2], max_height=-54, opts=opts)
    (surv, bad), spot_s = median_wall(
        lambda: eng.deep_spots(spots["s48"], spots["chunk_x"], spots["chunk_z"], max_height=-54, opts=opts))
    # config 4, a stated slice: structure seeds (hi16 << 32) | lo32, hi16 = the top 16 bits of
    # splitmix64(4), lo32 = 0, 1, 2, 3; each swept over the whole +-30M world with the catalogued
    # layouts of the -58 / -59 hunts (data/hunt/58, data/hunt/59) probed at every start
    wg = load_package()
    hi16 = wg.splitmix64(4) >> 48
    c4_seeds = [(hi16 << 32) | lo for lo in range(4)]
    layouts = [231564844655014, 156186219368766, 270840896143627]
    eng.deep_sweep(layouts, s48=c4_seeds[:1], rect=(-64, 64, -64, 64))
    (c4_matches, c4_starts), c4_s = median_wall(lambda: eng.deep_sweep(layouts, s48=c4_seeds, rect=wg.WORLD_REGIONS))
    world_regions = (wg.WORLD_REGIONS[1] - wg.WORLD_REGIONS[0]) * (wg.WORLD_REGIONS[3] - wg.WORLD_REGIONS[2])
    # the solver on the -58 plan line (layout 231564844655014, regime 22, class odd: data/hunt/58)
    plan = [(231564844655014, (2, 2), "odd")]
    eng.deep_solve(plan, 0, 2)
    (shits, sst), solve_s = median_wall(lambda: eng.deep_solve(plan, 4096, 64))
    # the mineshaft finisher over 1,024 start chunks of the walk under fixed upper seed bits
    rng = np.random.default_rng(9)
    fin = hits[:1024]
    fin_ws = [((int(u) << 48) | (int(s) & 0xFFFFFFFFFFFF)) for u, s in zip(rng.integers(0, 1 << 16, len(fin)), fin["s48"])]
    eng.finish_rows(fin_ws[:2], fin["chunk_x"][:2], fin["chunk_z"][:2])
    frows, fin_s = median_wall(lambda: eng.finish_rows(fin_ws, fin["chunk_x"], fin["chunk_z"]))
    finisher = {"rows": len(fin_ws), "rows_per_s": len(fin_ws) / fin_s, "ms": 1e3 * fin_s,
                "accepted_by_lysh": int(frows["verdict_ok"].sum()), "trees": int((frows["tree_status"] == 0).sum()),
                "pieces": int(frows["pieces"].sum()),
                "cpu_baseline": finisher_cpu_baseline(fin_ws[:16], fin["chunk_x"][:16], fin["chunk_z"][:16])}
    return {"solver": {"plan": "231564844655014 22 odd", "groups": sst["groups"], "regions": sst["regions"],
                       "tasks": sst["tasks"], "candidates": sst["candidates"], "hits": sst["hits"],
                       "tasks_per_s": sst["tasks"] / solve_s, "groups_per_s": sst["groups"] / solve_s,
                       "device_tasks_per_s": sst["tasks"] / (sst["gpu_ms"] / 1e3), "ms": 1e3 * solve_s,
                       "gpu_ms": sst["gpu_ms"]},
            "walk": {"structure_seeds": n_s48, "regions": regions, "starts": int(len(hits)),
                     "regions_per_s": regions / walk_s, "ms": 1e3 * walk_s},
            "terrain": {"spots": int(len(spots)), "world_seeds": int(len(spots)) << 16,
                        "world_seeds_per_s": (len(spots) << 16) / spot_s, "ms": 1e3 * spot_s,
                        "survivors": int(len(surv)), "max_height": -54},
            "c4": {"slice": "structure seeds (hi16 << 32) | lo32, hi16 = splitmix64(4) >> 48, lo32 = 0..3, each "
                            "over every hut region of the +-30M world (117,187^2), catalogue = the 3 layouts of "
                            "data/hunt/58 and /59",
                   "structure_seeds": len(c4_seeds), "regions": len(c4_seeds) * world_regions,
                   "starts": int(c4_starts.sum()), "matches": int(len(c4_matches)),
                   "structure_seeds_per_s": len(c4_seeds) / c4_s, "regions_per_s": len(c4_seeds) * world_regions / c4_s,
                   "world_seeds_per_s_equivalent": (len(c4_seeds) << 16) / c4_s, "ms": 1e3 * c4_s,
                   "note": ("world seeds/s = structure seeds/s x 65,536 (each structure seed stands for its 65,536 "
                            "upper-16-bit world seeds); the terrain stage that expands a match runs at the "
                            "`terrain` rate; the reference's own figure is about 94 M world seeds/s for that "
                            "stage (hunt.py:463-464)")},
            "finisher": finisher,
            "timing": "wall clock around wg_deep_solve / wg_deep_starts / wg_deep_spots / wg_finish_rows (host "
                      "buffers in and out; the median of three calls each); device time of the solver from its "
                      "CUDA events"}


def finisher_cpu_baseline(ws, cx, cz) -> dict | None:
    """hunt.py's finish_row as the reference runs it (one process per tool: lysh hut, mstree, biome_at
    x 2, msroom, skyscan) on the first survivors, with the reference's tools built from its sources
    into oracle/_ref; None when they are not there."""
    ref = os.path.join(ROOT, "oracle", "_ref")
    tools = ("lysh", "mstree", "biome_at", "msroom", "skyscan")
    if not all(os.path.exists(os.path.join(ref, t)) for t in tools):
        return None
    import subprocess
    import tempfile

    def run(args, stdin=None, env=None):
        return subprocess.run(args, input=stdin, capture_output=True, text=True, env=dict(os.environ, **(env or {})),
                              timeout=120).stdout

    t0 = time.perf_counter()
    for w, x, z in zip(ws, cx, cz):
        w = w - (1 << 64) if w >= 1 << 63 else w
        hx, hz = 16 * int(x), 16 * int(z)
        run([os.path.join(ref, "lysh"), "hut", "--seed", str(w), "--x", str(hx), "--z", str(hz), "--max-y", "100",
             "--phase2-max-y", "100", "--version", "1.19.x~26.1"])
        tree = run([os.path.join(ref, "mstree"), str(w), str(int(x)), str(int(z))])
        if not tree.strip():
            continue
        fl = tree.split()[2]
        for env in (None, {"BIOME_26": "1"}):
            run([os.path.join(ref, "biome_at"), "--seed", str(w), "--cx", str(int(x)), "--cz", str(int(z)), "--ms",
                 "--y", fl], env=env)
        run([os.path.join(ref, "msroom"), "--seed", str(w), "--x", str(hx), "--z", str(hz)], stdin=tree,
            env={"MC_SHAPE": "79", "MC_TRIALS": "0"})
        with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
            f.write("X,u,wx,wz,fw,fd,dx,dz,bound\n%d,%d,%d,%d,7,9,%d,%d,0\n"
                    % (w & 0xFFFFFFFFFFFF, (w >> 48) & 0xFFFF, hx, hz, int(x), int(z)))
        try:
            run([os.path.join(ref, "skyscan"), "--list", f.name])
        finally:
            os.remove(f.name)
    secs = time.perf_counter() - t0
    return {"value": len(ws) / secs, "unit": "rows/s", "cores": 1, "kind": "reference",
            "sample": f"the first {len(ws)} rows through the reference's finisher tools, one process per tool "
                      "as hunt.py's finish_row spawns them"}


def biome_measure(eng) -> dict:
    """The map tab's biome raster (wg_biome_map): 2,048 x 2,048 cells of one chunk each (ss 1) around
    the SCAN_REFERENCE hut, wall clock around the call (world build included), median of 3 after a
    warm-up."""
    seed = 1473884015873122059
    eng.biome_map(seed, -16384, -17408, 64, 64, 16)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        m = eng.biome_map(seed, -16384 - 16 * 1024, -17408 - 16 * 1024, 2048, 2048, 16)
        times.append(time.perf_counter() - t0)
    secs = statistics.median(times)
    return {"cells": int(m.size), "cells_per_s": m.size / secs, "ms": 1e3 * secs, "swamp_cells": int((m == 6).sum()),
            "timing": "wall clock around wg_biome_map (one world build, raster back to the host), median of 3"}


def jobs_measure(wg, eng, n_jobs: int = 65536) -> dict:
    """Uneven batched jobs: the 65,536 jobs of the splitmix64(3) job stream (1..4,096 seeds,
    radius 1..64, floors -50..-54) through one wg_seed_check_jobs call, host seed lists in and
    survivors out (wall clock; device time from the call's own CUDA events), after a warm-up on
    the first 64 jobs."""
    jobs = wg.uneven_jobs(n_jobs=n_jobs)
    t0 = time.perf_counter()
    tuning = eng.tune()
    tune_s = time.perf_counter() - t0
    eng.seed_check_jobs(jobs[:64])
    t0 = time.perf_counter()
    got, st = eng.seed_check_jobs(jobs)
    secs = time.perf_counter() - t0
    seeds = sum(len(j["seeds"]) for j in jobs)
    return {"jobs": n_jobs, "seeds": seeds, "checks": st["scanned"], "survivors": st["accepted"],
            "seeds_per_s": seeds / secs, "checks_per_s": st["scanned"] / secs, "ms": 1e3 * secs,
            "gpu_ms": st["gpu_ms"], "slices": st["batches"], "retries": st["retries"],
            "gpu_launches": sum(st["kernel_launches"]),
            "mode": "device work queue: all seeds resident, one graph launch per rule set whose device-side "
                    "while-loop takes slices of units off the queue",
            "tuning": tuning, "tuning_s": tune_s,
            "timing": "wall clock around wg_seed_check_jobs (host seed lists in, survivors out), after "
                      "wg_engine_tune on this GPU"}


def serving_measure(wg, n_req: int = 200) -> dict:
    """Serving: one wg_server; the request stream of serving_requests (1..10^6 seeds as splitmix64
    generators, radius 1..32, floors -50..-54).  Peak = all requests submitted at once (checks/s
    over the makespan); then the same requests with Poisson arrivals at 30 %, 70 % and 100 % of
    that peak, p50 / p99 of submit-to-done latency and the seeds/s delivered."""
    import threading
    base_reqs = wg.serving_requests(n_req, rate_per_s=1.0)
    work = [q["gen"][1] * (q["rect"][1] - q["rect"][0]) * (q["rect"][3] - q["rect"][2]) for q in base_reqs]
    out = {"requests": n_req, "seeds": int(sum(q["gen"][1] for q in base_reqs)), "checks": int(sum(work))}
    with wg.Server(0) as srv:
        for q in base_reqs[:8]:   # warm-up
            srv.wait(srv.submit(gen=q["gen"], rect=q["rect"], max_height=q["max_height"]))
        t0 = time.perf_counter()
        ids = [srv.submit(gen=q["gen"], rect=q["rect"], max_height=q["max_height"]) for q in base_reqs]
        for j in ids:
            srv.wait(j)
            srv.take(j)
        peak_s = time.perf_counter() - t0
        peak = sum(work) / peak_s
        out["peak"] = {"checks_per_s": peak, "seeds_per_s": out["seeds"] / peak_s, "ms": 1e3 * peak_s}
        loads = []
        for frac in (0.3, 0.7, 1.0):
            rate = frac * peak / (sum(work) / n_req)
            reqs = wg.serving_requests(n_req, rate_per_s=rate)
            ids = [None] * n_req

            def feed():
                t_start = time.perf_counter()
                for i, q in enumerate(reqs):
                    delay = q["t"] - (time.perf_counter() - t_start)
                    if delay > 0:
                        time.sleep(delay)
                    ids[i] = srv.submit(gen=q["gen"], rect=q["rect"], max_height=q["max_height"])

            t0 = time.perf_counter()
            th = threading.Thread(target=feed)
            th.start()
            th.join()
            lat = []
            for j in ids:
                st = srv.wait(j)
                srv.take(j)
                lat.append(st["latency_ms"])
            secs = time.perf_counter() - t0
            lat = np.array(lat)
            loads.append({"offered": frac, "rate_per_s": rate, "p50_ms": float(np.percentile(lat, 50)),
                          "p99_ms": float(np.percentile(lat, 99)), "max_ms": float(lat.max()),
                          "seeds_per_s": out["seeds"] / secs, "checks_per_s": sum(work) / secs})
        out["loads"] = loads
        st = srv.stats()
        out["gpu_launches"] = sum(st["kernel_launches"])
    out["timing"] = ("wall clock; latency = submit to done inside the library (steady clock); requests "
                     "are generator jobs (seed lists made on the host at submit)")
    return out


def sorted_hits(wg, out_dev, n: int) -> np.ndarray:
    """The first n device candidates (wg_candidate rows of out_dev), sorted by (seed_index, rz, rx)."""
    n = min(int(n), out_dev.shape[0])
    rows = np.frombuffer(out_dev[:n].cpu().numpy().tobytes(), dtype=wg.CANDIDATE_DTYPE)
    return np.sort(rows, order=["seed_index", "rz", "rx"])


def splitmix_seeds(first: int, n: int) -> np.ndarray:
    """Seeds first .. first + n - 1 of the config-2 stream, splitmix64(2 + i), as int64."""
    idx = np.arange(first, first + n, dtype=np.uint64) + np.uint64(GEN_BASE)
    with np.errstate(over="ignore"):   # splitmix64 over the whole array, mod 2^64
        z = idx + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z.view(np.int64)


def profile_case(wg, eng, opts, args, local: int) -> None:
    """--profile N: the headline step (seed list resident in HBM, wg_seed_check_device) on the first
    N seeds of the stream, --warmup + --steps times, and nothing else: the command ncu captures."""
    import torch
    n = int(args.profile)
    seeds = torch.from_numpy(splitmix_seeds(0, n)).to(f"cuda:{local}")
    cap = 1 << 16
    out = torch.zeros((cap, 4), dtype=torch.int64, device=f"cuda:{local}")
    stream = torch.cuda.current_stream()
    found, st = 0, {}
    for _ in range(args.warmup + args.steps):
        found, st = eng.seed_check_device(seeds.data_ptr(), 0, n, RECT, MAX_HEIGHT, opts, out.data_ptr(), cap,
                                          stream.cuda_stream)
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": {"seeds": n, "noise_core": args.noise_core, "found": found,
                                       "kernel_launches": st["kernel_launches"], "kernel_ms": st["kernel_ms"],
                                       "records": st["records"], "climate_survivors": st["climate_survivors"],
                                       "rechecks": st["rechecks"]}}), flush=True)


def noise_core_measure(wg, eng, args, step_device, stream, flush, headline: dict) -> dict:
    """The other noise cores on the same device-resident step: seeds/s of each, the FP32 / FP64
    ratio, whether the hit sets and funnels agree, how often the FP32 core re-took a gate in FP64,
    and the measured |FP32 - FP64| of each climate noise and each cave noise of the entrance gate
    (wg_noise_probe, wg_noise_probe_3d)."""
    import torch
    runs = {args.noise_core: headline}
    for other in [c for c in ("fp32", "fp64", "fp32_caves") if c != args.noise_core]:
        eng.set_noise_core(other)
        for _ in range(args.warmup):
            step_device()
        times = []
        found, st = 0, {}
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            found, st = step_device()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        ms_other = sum(times) / len(times)
        runs[other] = {"seeds_per_s": N_SEEDS / (ms_other / 1e3), "ms_per_step": ms_other, "found": found,
                       "reject_hist": st["reject_hist"], "tier_hist": st["tier_hist"], "rechecks": st["rechecks"],
                       "kernel_ms": st["kernel_ms"]}
    eng.set_noise_core(args.noise_core)
    same = all(runs[c]["found"] == runs["fp64"]["found"] and runs[c]["reject_hist"] == runs["fp64"]["reject_hist"]
               and runs[c]["tier_hist"] == runs["fp64"]["tier_hist"] for c in runs)
    rng = np.random.default_rng(7)
    xz = (4 * rng.integers(-1_870_000, 1_870_000, size=(4096, 2)) + 2).astype(np.float64)
    seeds = [wg.splitmix64(GEN_BASE + i) for i in range(256)]
    err = {}
    for noise in ("erosion", "temperature", "ridge", "continentalness"):
        v32, v64 = eng.noise_probe(seeds, noise, xz)
        err[noise] = float(np.abs(v32 - v64).max())
    xyz = np.stack([16 * rng.integers(-1_870_000, 1_870_000, 4096) + 3, rng.choice([50, 60], 4096),
                    16 * rng.integers(-1_870_000, 1_870_000, 4096) + 3], axis=1).astype(np.float64)
    for noise in ("cave_entrance", "spaghetti_rarity", "spaghetti_thickness", "spaghetti_3d_1", "spaghetti_3d_2",
                  "roughness_modulator", "roughness"):
        v32, v64 = eng.noise_probe_3d(seeds, noise, xyz)
        err[noise] = float(np.abs(v32 - v64).max())
    scanned = N_SEEDS * (RECT[1] - RECT[0]) * (RECT[3] - RECT[2])
    return {"fp32": runs["fp32"], "fp64": runs["fp64"], "fp32_caves": runs["fp32_caves"],
            "fp32_over_fp64": runs["fp64"]["ms_per_step"] / runs["fp32"]["ms_per_step"],
            "fp32_caves_over_fp64": runs["fp64"]["ms_per_step"] / runs["fp32_caves"]["ms_per_step"],
            "same_hits_and_funnel": bool(same),
            "recheck_fraction": runs["fp32"]["rechecks"] / scanned,
            "max_abs_err": err,
            "max_abs_err_note": ("|FP32 core - FP64| of each y = 0 climate noise over 256 seeds x 4,096 climate points, "
                                 "and of each 3-D cave noise of the entrance gate over 256 seeds x 4,096 hut blocks "
                                 "(x, z up to +-3e7, y 50 / 60); the ladder's noises (cheese, cave layer, "
                                 "continentalness at the hut, floodedness) and phase 2 run in FP64 only, so their "
                                 "error is 0 by construction"),
            "bound": "the step's kernels; both cores on the same seeds, CUDA events per step"}


def run_reference(args) -> None:
    """--impl reference: the reference's CPU scanner on the host cores, same metric."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n_sample = 1 << 18
    for _ in range(args.warmup):
        cpu_baseline(n_sample // 8)
    vals = [cpu_baseline(n_sample) for _ in range(args.steps)]
    v = statistics.median(x["value"] for x in vals)
    cb = dict(vals[0])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n_sample / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "config 2 sample: splitmix64(2 + i) seeds x 9x9 regions, floor -50, "
                                   f"{VERSION}; {n_sample} seeds per step", "seeds_per_step": n_sample},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-jobs", action="store_true", help="skip the batched-jobs and serving measurements")
    ap.add_argument("--whole-world-only", action="store_true",
                    help="only hunt.py's per-seed workload: one seed over the whole +-30M world")
    ap.add_argument("--phase2-only", action="store_true",
                    help="one phase-1 pass for its survivors, then only the phase-2 measurement (a short "
                         "command for profiling the phase-2 kernels)")
    ap.add_argument("--noise-core", choices=("fp32", "fp64", "fp32_caves"), default="fp32",
                    help="noise core of the headline (the other cores are measured beside it)")
    ap.add_argument("--profile", type=int, default=0, metavar="SEEDS",
                    help="profiling case only: the headline step on SEEDS device-resident seeds, --warmup "
                         "untimed steps then --steps steps, no other measurement (a short command for ncu)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    wg = load_package()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    eng = wg.Engine(local, noise_core=args.noise_core)
    opts = wg.make_opts(VERSION)
    if args.profile:
        profile_case(wg, eng, opts, args, local)
        eng.close()
        return
    first = rank * N_SEEDS                       # weak scaling: each rank owns 2^24 seeds of the stream
    seeds_host = torch.empty(N_SEEDS, dtype=torch.int64, pin_memory=True)
    seeds_np = seeds_host.numpy()
    seeds_np[:] = splitmix_seeds(first, N_SEEDS)
    if args.whole_world_only:
        if rank == 0:
            print(json.dumps({"whole_world": whole_world_measure(eng, opts)}), flush=True)
        eng.close()
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.phase2_only:
        res = eng.seed_check(seeds=seeds_np, rect=RECT, max_height=MAX_HEIGHT, opts=opts)
        line = {"phase2": phase2_measure(eng, res.candidates, opts, cpu=False)}
        if rank == 0:
            print(json.dumps(line), flush=True)
        eng.close()
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    seeds_dev = seeds_host.to(f"cuda:{local}")
    out_cap = 1 << 16
    out_dev = torch.zeros((out_cap, 4), dtype=torch.int64, device=f"cuda:{local}")
    flush = torch.empty(64 << 20, dtype=torch.float32, device=f"cuda:{local}")   # 256 MiB > 126 MB L2
    stream = torch.cuda.current_stream()

    def step_device():
        return eng.seed_check_device(seeds_dev.data_ptr(), 0, N_SEEDS, RECT, MAX_HEIGHT, opts, out_dev.data_ptr(),
                                     out_cap, stream.cuda_stream)

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    # ---- device-resident timed region ----
    times, kernel_ms, kernel_launches, found, stats = [], [0.0, 0.0, 0.0], [0, 0, 0], 0, None
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            found, stats = step_device()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            for k in range(3):
                kernel_ms[k] += stats["kernel_ms"][k]
                kernel_launches[k] += stats["kernel_launches"][k]
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    total_ms = sum(times)
    hits_headline = sorted_hits(wg, out_dev, found)

    # ---- end to end through the public host API ----
    e2e_ms = []
    for i in range(1 + args.steps):
        t0 = time.perf_counter()
        res = eng.seed_check(seeds=seeds_np, rect=RECT, max_height=MAX_HEIGHT, opts=opts)
        dt = (time.perf_counter() - t0) * 1e3
        if i:
            e2e_ms.append(dt)
    e2e_total = sum(e2e_ms)
    survivors_e2e = len(res.candidates)
    d2h = survivors_e2e * 32 + res.stats["batches"] * (32 + 18 * 8)

    if world > 1:
        t = torch.tensor([total_ms, e2e_total], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, e2e_total = float(t[0]), float(t[1])
        n_found = torch.tensor([found], dtype=torch.int64, device=f"cuda:{local}")
        dist.all_reduce(n_found)
        found_all = int(n_found.item())
    else:
        found_all = found

    if rank == 0:
        n_total = N_SEEDS * world
        value = n_total * args.steps / (total_ms / 1e3)
        e2e_value = n_total * args.steps / (e2e_total / 1e3)
        n_regions = (RECT[1] - RECT[0]) * (RECT[3] - RECT[2])
        peaks = measured_peaks()
        sm_count = torch.cuda.get_device_properties(local).multi_processor_count
        max_mhz = float(peaks.get("sm_max_mhz", 1965.0))
        peak_ops = sm_count * 128 * max_mhz * 1e6
        fp32 = args.noise_core in ("fp32", "fp32_caves")
        ops, nbytes = climate_work(stats, N_SEEDS, n_regions, fp32)
        launch_ms = kernel_ms[0] / max(1, kernel_launches[0])
        ops_per_launch = ops / max(1, stats["kernel_launches"][0])
        bytes_per_launch = nbytes / max(1, stats["kernel_launches"][0])
        achieved = ops_per_launch / (launch_ms / 1e3)
        ent_ms = kernel_ms[1] / max(1, kernel_launches[1])
        caves32 = args.noise_core == "fp32_caves"   # the cave samples are FP32 only in that core
        ent_ops = entrance_work(stats, caves32) / max(1, stats["kernel_launches"][1])
        hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
        cs = clocks.summary()
        headline = {"seeds_per_s": value, "ms_per_step": total_ms / args.steps, "found": found,
                    "reject_hist": stats["reject_hist"], "tier_hist": stats["tier_hist"],
                    "rechecks": stats["rechecks"], "kernel_ms": [k / args.steps for k in kernel_ms]}
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if fp32 else "f64", "data": "synthetic",
            "config": {"workload": "config 2: Seed Check phase 1, 2^24 splitmix64(2 + i) world seeds per GPU x 9x9 "
                                   "swamp-hut regions (1.36e9 (seed, region) checks), floor -50, rules "
                                   f"{VERSION}, " + ("FP32 noise core with FP64 recheck (verdicts equal the FP64 "
                                                     "path's)" if fp32 else "bit-exact FP64"),
                       "noise_core": args.noise_core, "seeds_per_gpu": N_SEEDS,
                       "regions_per_seed": n_regions, "max_height": MAX_HEIGHT, "parallelism": f"seed-shard x{world}",
                       "l2": "256 MiB buffer written between timed steps (outside the events); seed input 134 MB",
                       "inputs": "seed list resident in HBM (value); pinned host seeds via wg_seed_check (e2e)"},
            "survivors_per_step": found_all,
            "funnel": stats["reject_hist"],
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": N_SEEDS * 8,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_total / args.steps},
            "gpu_launches": sum(kernel_launches),
            "kernel_ms_per_step": [k / args.steps for k in kernel_ms],
            "roofline": {
                "bound": "issue", "kernel": "climate_kernel", "unit": "Tlane-op/s",
                "achieved": achieved / 1e12, "peak": peak_ops / 1e12, "frac": achieved / peak_ops,
                "peak_source": f"nominal INT32/FP32 issue rate: {sm_count} SMs x 128 lanes x {max_mhz:.0f} MHz "
                               "(sm_max_mhz of MEASURED_PEAKS.json); the kernel is not HBM- or tensor-bound",
                "ops_per_launch": ops_per_launch, "launch_ms": launch_ms,
                "ops_model": ("18 Perlin tables per seed x 7,160 lane-ops, per y=0 sample "
                              f"{OPS_Y0_SAMPLE_F32 if fp32 else OPS_Y0_SAMPLE} lane-ops x the samples the funnel "
                              "implies, 40 per (seed, region) placement"),
                "traffic": TRAFFIC["climate_kernel"], "traffic_unit": "bytes per launch",
                "traffic_source": TRAFFIC["source"],
                "ncu_pipes": dict(PIPES["climate_kernel"], unit=PIPES["unit"]),
                "algorithmic_bytes": bytes_per_launch,
                "hbm": {"achieved_gbs": bytes_per_launch / (launch_ms / 1e3) / 1e9, "peak_gbs": hbm_peak,
                        "frac": bytes_per_launch / (launch_ms / 1e3) / 1e9 / hbm_peak,
                        "peak_source": "hbm_gbs of MEASURED_PEAKS.json"},
                "entrance_kernel": {
                    "bound": "issue", "unit": "Tlane-op/s", "achieved": ent_ops / (ent_ms / 1e3) / 1e12,
                    "peak": peak_ops / 1e12, "frac": ent_ops / (ent_ms / 1e3) / peak_ops, "ops_per_launch": ent_ops,
                    "launch_ms": ent_ms, "traffic": TRAFFIC["entrance_kernel"], "traffic_unit": "bytes per launch",
                    "ncu_pipes": dict(PIPES["entrance_kernel"], unit=PIPES["unit"]),
                    "ops_model": ("18 Perlin tables per record x 7,160 lane-ops, per climate survivor 36 3-D samples "
                                  f"x {OPS_3D_SAMPLE_F32 if caves32 else OPS_3D_SAMPLE} lane-ops + 600 for the octave "
                                  "sums and the decision")},
            },
            "clocks": cs,
        }
        if world == 1:
            nc = noise_core_measure(wg, eng, args, step_device, stream, flush, headline)
            # the output buffer holds the last core measured
            other = [c for c in ("fp32", "fp64", "fp32_caves") if c != args.noise_core][-1]
            hits_other = sorted_hits(wg, out_dev, nc[other]["found"])
            nc["same_hits_and_funnel"] = bool(nc["same_hits_and_funnel"] and np.array_equal(hits_other, hits_headline))
            line["noise_core"] = nc
        line["phase2"] = phase2_measure(eng, res.candidates, opts, cpu=(world == 1 and not args.no_cpu_baseline))
        line["whole_world"] = whole_world_measure(eng, opts)
        line["deep_dive"] = deep_measure(eng, opts)
        line["biome_map"] = biome_measure(eng)
        if world == 1 and not args.no_jobs:
            line["jobs"] = jobs_measure(wg, eng)
            line["serving"] = serving_measure(wg)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(1 << 19)
        print(json.dumps(line), flush=True)

    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
