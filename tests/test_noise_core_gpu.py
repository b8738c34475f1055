"""The FP32 noise core with its FP64 recheck, against the plain FP64 path and the reference.

The climate gates (erosion tiers, temperature, ridge) take their samples in FP32 and decide from
the FP32 sums wherever a sum lies outside its derived error band; inside the band the region is
recomputed in FP64 in the reference's order.  So the verdict of every (seed, region) must equal
the FP64 path's, and through it lysh's (engine/tools/lysh/src/phase1.c:130-200): the tests below
require identical survivor lists, reject histograms, erosion tier histograms and per-region codes.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RECT9 = (-4, 5, -4, 5)
VARIANTS = [("1.19.x~26.1", "NORMAL", -50), ("26.2", "NORMAL", -40), ("1.18.2", "NORMAL", -50),
            ("1.19.x~26.1", "LARGE_BIOMES", -50), ("1.19.x~26.1", "SINGLE_BIOME", -50),
            ("1.19.x~26.1", "NORMAL", 100), ("1.19.x~26.1", "NORMAL", -45)]

# |FP32 value - FP64 value| of one DoublePerlin at y = 0, from the per-sample bound (44 * 2^-24) summed
# over at most 18 octaves of weight <= 2 and the amplitude (< 1.2): far below 1e-4.
VALUE_BOUND = 1e-4


@pytest.fixture(scope="module")
def eng64(wg, engine):
    e = wg.Engine(0, noise_core="fp64")
    yield e
    e.close()


@pytest.fixture(scope="module")
def eng_all(wg, engine):
    e = wg.Engine(0, noise_core="fp32_recheck_all")
    yield e
    e.close()


def test_default_core_is_fp32(engine):
    assert engine.noise_core == "fp32"


def test_full_config2_same_hits_as_fp64(engine, eng64, golden):
    """All 2^24 seeds splitmix64(2 + i) over 9 x 9 regions: the FP32 core's survivors, funnel and tier histogram equal the
    FP64 path's and the reference's; the recheck fires, and rarely."""
    g = golden("c2_full_survivors.npz")
    n = 1 << 24
    a = engine.seed_check(gen=(2, n), rect=RECT9, max_height=-50)
    b = eng64.seed_check(gen=(2, n), rect=RECT9, max_height=-50)
    assert np.array_equal(a.candidates, b.candidates)
    assert np.array_equal(a.candidates, g["survivors"])
    assert a.stats["reject_hist"] == b.stats["reject_hist"]
    assert a.stats["tier_hist"] == b.stats["tier_hist"]
    assert a.stats["climate_survivors"] == b.stats["climate_survivors"]
    assert b.stats["rechecks"] == 0
    assert 0 < a.stats["rechecks"] < 1e-3 * a.stats["scanned"]


@pytest.mark.parametrize("k", range(len(VARIANTS)))
def test_rule_variants_codes(engine, eng64, golden, k):
    g = golden("variants.npz")
    version, preset, mh = VARIANTS[k]
    c32, t32 = engine.phase1_codes(seeds=g["seeds"], rect=RECT9, max_height=mh, version=version, preset=preset)
    c64, t64 = eng64.phase1_codes(seeds=g["seeds"], rect=RECT9, max_height=mh, version=version, preset=preset)
    assert np.array_equal(c32, c64) and np.array_equal(t32, t64)
    assert np.array_equal(c32, g[f"codes_{k}"]) and np.array_equal(t32, g[f"tiers_{k}"])


def test_c1_codes_with_every_gate_rechecked(eng_all, golden):
    """The check mode re-takes every FP32 decision in FP64: the recheck path alone must give the
    reference's per-region codes and tiers."""
    g = golden("c1_phase1.npz")
    codes, tiers = eng_all.phase1_codes(seeds=g["seeds"], rect=RECT9, max_height=-50)
    assert np.array_equal(codes, g["codes"]) and np.array_equal(tiers, g["tiers"])


@pytest.mark.parametrize("k", [0, 1, 2, 3, 5])
def test_variants_with_every_gate_rechecked(eng_all, golden, k):
    g = golden("variants.npz")
    version, preset, mh = VARIANTS[k]
    codes, tiers = eng_all.phase1_codes(seeds=g["seeds"], rect=RECT9, max_height=mh, version=version, preset=preset)
    assert np.array_equal(codes, g[f"codes_{k}"]) and np.array_equal(tiers, g[f"tiers_{k}"])


def test_recheck_all_counts_every_decision(eng_all, engine):
    a = eng_all.seed_check(gen=(2, 1 << 16), rect=RECT9, max_height=-50)
    b = engine.seed_check(gen=(2, 1 << 16), rect=RECT9, max_height=-50)
    assert np.array_equal(a.candidates, b.candidates) and a.stats["reject_hist"] == b.stats["reject_hist"]
    # at least one decision per region (its tier-0 check)
    assert a.stats["rechecks"] >= a.stats["scanned"] > b.stats["rechecks"]


def test_relaxed_floors_same_as_fp64(engine, eng64):
    """More regions reach the later tiers, temperature and ridge at max_height 100 over a larger
    rect: identical survivors and funnels."""
    for mh in (0, 100):
        a = engine.seed_check(gen=(123, 1 << 17), rect=(-12, 12, -12, 12), max_height=mh, version="26.2")
        b = eng64.seed_check(gen=(123, 1 << 17), rect=(-12, 12, -12, 12), max_height=mh, version="26.2")
        assert np.array_equal(a.candidates, b.candidates), mh
        assert a.stats["reject_hist"] == b.stats["reject_hist"] and a.stats["tier_hist"] == b.stats["tier_hist"]


def test_large_biomes_and_118_same_as_fp64(engine, eng64):
    for version, preset in (("1.19.x~26.1", "LARGE_BIOMES"), ("1.18.2", "NORMAL")):
        a = engine.seed_check(gen=(31, 1 << 17), rect=RECT9, max_height=100, version=version, preset=preset)
        b = eng64.seed_check(gen=(31, 1 << 17), rect=RECT9, max_height=100, version=version, preset=preset)
        assert np.array_equal(a.candidates, b.candidates), (version, preset)
        assert a.stats["reject_hist"] == b.stats["reject_hist"] and a.stats["tier_hist"] == b.stats["tier_hist"]


@pytest.mark.parametrize("noise", ["erosion", "temperature", "ridge", "continentalness", "erosion_large",
                                   "temperature_large", "continentalness_large"])
def test_noise_probe_error_is_small(engine, wg, noise):
    """The measured |FP32 - FP64| of each climate noise over 64 seeds x 4,096 points spread over the
    world (climate coordinates x = 4 * chunk + 2 of chunks up to +-1.87e6) stays inside the bound
    and is non-zero (the FP32 core is really in use)."""
    rng = np.random.default_rng(7)
    chunks = rng.integers(-1_870_000, 1_870_000, size=(4096, 2))
    xz = (4 * chunks + 2).astype(np.float64)
    seeds = [wg.splitmix64(2 + i) for i in range(64)]
    v32, v64 = engine.noise_probe(seeds, noise, xz)
    err = np.abs(v32 - v64)
    assert np.all(np.isfinite(v64)) and np.abs(v64).max() < 2.0
    assert 0 < err.max() < VALUE_BOUND, err.max()


# |FP32 core - FP64| bound of an entrance-gate DoublePerlin value: 2 |amplitude| sum_p |amp_p per_p|
# times the 3-D sample bound (60 * 2^-24) stays below 3e-5 for every cave noise of the gate
VALUE_BOUND_3D = 3e-5


@pytest.mark.parametrize("noise", ["cave_entrance", "spaghetti_rarity", "spaghetti_thickness", "spaghetti_3d_1",
                                   "spaghetti_3d_2", "roughness_modulator", "roughness"])
def test_noise_probe_3d_error_is_small(engine, wg, noise):
    """The entrance gate's cave noises in the FP32 core: measured |FP32 - FP64| over 32 seeds x
    4,096 points spread over the world (block x, z up to +-3e7, y in the build range) stays inside
    the bound and is non-zero (the FP32 samples are really in use)."""
    rng = np.random.default_rng(11)
    xyz = np.stack([rng.integers(-30_000_000, 30_000_000, 4096), rng.integers(-64, 320, 4096),
                    rng.integers(-30_000_000, 30_000_000, 4096)], axis=1).astype(np.float64)
    seeds = [wg.splitmix64(2 + i) for i in range(32)]
    v32, v64 = engine.noise_probe_3d(seeds, noise, xyz)
    err = np.abs(v32 - v64)
    assert np.all(np.isfinite(v64)) and np.abs(v64).max() < 4.0
    assert 0 < err.max() < VALUE_BOUND_3D, err.max()


@pytest.fixture(scope="module")
def eng_caves(wg, engine):
    e = wg.Engine(0, noise_core="fp32_caves")
    yield e
    e.close()


def test_fp32_caves_full_config2_same_hits_as_fp64(eng_caves, eng64, golden):
    """The entrance gate's cave samples in the FP32 core too: all 2^24 seeds splitmix64(2 + i) over 9 x 9 regions give the FP64
    path's survivors, funnel and tier histogram, and the reference's survivors."""
    g = golden("c2_full_survivors.npz")
    n = 1 << 24
    a = eng_caves.seed_check(gen=(2, n), rect=RECT9, max_height=-50)
    b = eng64.seed_check(gen=(2, n), rect=RECT9, max_height=-50)
    assert np.array_equal(a.candidates, b.candidates)
    assert np.array_equal(a.candidates, g["survivors"])
    assert a.stats["reject_hist"] == b.stats["reject_hist"] and a.stats["tier_hist"] == b.stats["tier_hist"]
    assert a.stats["deep_candidates"] == b.stats["deep_candidates"]


@pytest.mark.parametrize("k", range(len(VARIANTS)))
def test_fp32_caves_rule_variants_codes(eng_caves, golden, k):
    g = golden("variants.npz")
    version, preset, mh = VARIANTS[k]
    c, t = eng_caves.phase1_codes(seeds=g["seeds"], rect=RECT9, max_height=mh, version=version, preset=preset)
    assert np.array_equal(c, g[f"codes_{k}"]) and np.array_equal(t, g[f"tiers_{k}"])


def test_fp32_caves_relaxed_floor_same_as_fp64(eng_caves, eng64):
    """A relaxed floor sends more climate survivors past the entrance gate to the ladder."""
    a = eng_caves.seed_check(gen=(123, 1 << 17), rect=(-12, 12, -12, 12), max_height=100, version="26.2")
    b = eng64.seed_check(gen=(123, 1 << 17), rect=(-12, 12, -12, 12), max_height=100, version="26.2")
    assert np.array_equal(a.candidates, b.candidates)
    assert a.stats["reject_hist"] == b.stats["reject_hist"] and a.stats["deep_candidates"] == b.stats["deep_candidates"]
