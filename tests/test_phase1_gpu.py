"""GPU parity of the Seed Check phase 1, called through the C ABI (libwitchgpu.so).

Bar: bit-exact.  Per-region reject codes and erosion tiers must equal lysh's
(lysh_phase1_check_ex, engine/tools/lysh/src/phase1.c:130-200) for every (seed, region), and
survivor lists must be identical, chunk for chunk.  Golden fixtures come from the reference's
own lysh (tests/golden/make_golden.py); larger cases use the C restatement in oracle/, which
tests/test_oracle.py pins to those fixtures.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RECT9 = (-4, 5, -4, 5)
VARIANTS = [("1.19.x~26.1", "NORMAL", -50), ("26.2", "NORMAL", -40), ("1.18.2", "NORMAL", -50),
            ("1.19.x~26.1", "LARGE_BIOMES", -50), ("1.19.x~26.1", "SINGLE_BIOME", -50),
            ("1.19.x~26.1", "NORMAL", 100), ("1.19.x~26.1", "NORMAL", -45)]


def test_c1_codes_all_4096(engine, golden):
    g = golden("c1_phase1.npz")
    codes, tiers = engine.phase1_codes(seeds=g["seeds"], rect=RECT9, max_height=-50)
    assert np.array_equal(codes, g["codes"])
    assert np.array_equal(tiers, g["tiers"])


def test_c1_generator_equals_list(engine, golden):
    g = golden("c1_phase1.npz")
    codes, tiers = engine.phase1_codes(gen=(1, 4096), rect=RECT9, max_height=-50)
    assert np.array_equal(codes, g["codes"]) and np.array_equal(tiers, g["tiers"])
    res = engine.seed_check(gen=(1, 4096), rect=RECT9, max_height=-50)
    assert len(res.candidates) == 0
    assert res.stats["reject_hist"] == np.bincount(g["codes"].ravel(), minlength=11).tolist()
    assert res.stats["tier_hist"] == [int((g["tiers"] == t).sum()) for t in range(7)]
    assert res.stats["scanned"] == 4096 * 81


@pytest.mark.parametrize("k", range(len(VARIANTS)))
def test_rule_variants(engine, golden, k):
    g = golden("variants.npz")
    version, preset, mh = VARIANTS[k]
    codes, tiers = engine.phase1_codes(seeds=g["seeds"], rect=RECT9, max_height=mh, version=version, preset=preset)
    assert np.array_equal(codes, g[f"codes_{k}"])
    assert np.array_equal(tiers, g[f"tiers_{k}"])


def test_known_answers(engine, golden):
    k = golden("known_answers.json")
    for label in ("scan_reference_40000", "scan_reference_5000", "verified_54"):
        want = k[label]
        res = engine.seed_check(seeds=[want["seed"]], rect=tuple(want["rect"]), max_height=-50)
        assert res.stats["reject_hist"] == want["hist"], label
        assert [[int(c["chunk_x"]), int(c["chunk_z"])] for c in res.candidates] == want["survivors"], label
    # hunt.py SCAN_REFERENCE: /tp -15792 -54 -17168 lies in the 40,000-block area only
    res = engine.seed_check(seeds=[1473884015873122059], rect=(-79, 79, -79, 79))
    assert [(c["chunk_x"] * 16, c["chunk_z"] * 16) for c in res.candidates] == [(-15792, -17168)]


def test_c2_sample_funnel(engine, golden):
    g = golden("c2_sample.npz")
    res = engine.seed_check(gen=(2, 65536), rect=RECT9, max_height=-50)
    assert res.stats["reject_hist"] == g["hist"].tolist()
    assert len(res.candidates) == 0


def test_c2_first_4m_seeds_survivors(engine, golden):
    g = golden("c2_4m_survivors.npz")
    res = engine.seed_check(gen=(2, int(g["n_seeds"])), rect=RECT9, max_height=-50)
    assert np.array_equal(res.candidates, g["survivors"])
    assert res.stats["accepted"] == len(g["survivors"]) == 52
    assert sum(res.stats["reject_hist"]) == res.stats["scanned"] == int(g["n_seeds"]) * 81


def test_full_config2(engine, port, bind_mod, golden):
    """All 2^24 seeds of config 2: the survivor list equals the reference's exactly, the funnel adds
    up, and every survivor is re-verified by the oracle region by region."""
    g = golden("c2_full_survivors.npz")
    n = 1 << 24
    res = engine.seed_check(gen=(2, n), rect=RECT9, max_height=-50)
    st = res.stats
    assert np.array_equal(res.candidates, g["survivors"])
    assert sum(st["reject_hist"]) == st["scanned"] == n * 81
    assert st["reject_hist"][10] == st["accepted"] == len(res.candidates) == len(g["survivors"])
    assert sum(st["tier_hist"]) == st["reject_hist"][0]
    r = bind_mod.rules("1.19.x~26.1")
    for c in res.candidates:
        assert int(c["seed"]) == wg_signed(port.splitmix64(2 + int(c["seed_index"])))
        codes, _, cx, cz = port.phase1_rect(int(c["seed"]), r, -50, RECT9)
        k = (int(c["rz"]) + 4) * 9 + (int(c["rx"]) + 4)
        assert codes[k] == 10 and (cx[k], cz[k]) == (c["chunk_x"], c["chunk_z"])
    keys = {(int(c["seed_index"]), int(c["rx"]), int(c["rz"])) for c in res.candidates}
    assert len(keys) == len(res.candidates)


def wg_signed(v: int) -> int:
    v &= 0xFFFFFFFFFFFFFFFF
    return v - (1 << 64) if v >= (1 << 63) else v


@pytest.mark.parametrize("rect", [(-200, 200, -200, 200), (-58594, -58560, 58560, 58594), (0, 1, 0, 1),
                                  (-3, -2, 7, 9), (1000, 1090, -5, 60)])
def test_rects_and_windows_vs_oracle(engine, port, bind_mod, rect):
    """Single regions, world-border regions and rects larger than one 4,096-region window."""
    r = bind_mod.rules("1.19.x~26.1")
    for seed in (1473884015873122059, 0, -1, -(1 << 63), (1 << 63) - 1):
        codes, tiers = engine.phase1_codes(seeds=[seed], rect=rect, max_height=-50)
        c, t, _, _ = port.phase1_rect(seed, r, -50, rect)
        assert np.array_equal(codes[0], c) and np.array_equal(tiers[0], t), (seed, rect)


def test_many_seeds_large_rect_vs_oracle(engine, port, bind_mod):
    r = bind_mod.rules("1.19.x~26.1")
    rect = (-40, 40, -40, 40)          # 6,400 regions: two windows per seed
    res = engine.seed_check(gen=(77, 512), rect=rect, max_height=-50)
    want, hist = port.scan_seeds(r, -50, rect, gen=(77, 512))
    assert np.array_equal(res.candidates, want)
    assert res.stats["reject_hist"] == hist.tolist()


def test_relaxed_floor_survivors_vs_oracle(engine, port, bind_mod):
    """max_height 0 and 100 let more regions through the ladder: survivor lists must match."""
    for mh in (0, 100):
        r = bind_mod.rules("26.2")
        res = engine.seed_check(gen=(5, 20000), rect=(-8, 8, -8, 8), max_height=mh, version="26.2")
        want, hist = port.scan_seeds(r, mh, (-8, 8, -8, 8), gen=(5, 20000))
        assert np.array_equal(res.candidates, want), mh
        assert res.stats["reject_hist"] == hist.tolist(), mh


def test_single_biome_overflow_retry(engine, port, bind_mod):
    """SINGLE_BIOME passes every region through the climate stage; the survivor lists fill and the
    engine re-runs smaller batches without losing or duplicating anything."""
    r = bind_mod.rules("1.19.x~26.1", "SINGLE_BIOME")
    res = engine.seed_check(gen=(9, 1000), rect=(-20, 20, -20, 20), max_height=-50, preset="SINGLE_BIOME")
    want, hist = port.scan_seeds(r, -50, (-20, 20, -20, 20), gen=(9, 1000))
    assert res.stats["retries"] > 0
    assert np.array_equal(res.candidates, want)
    assert res.stats["reject_hist"] == hist.tolist()


def test_seed_list_edge_values(engine, port, bind_mod):
    seeds = [0, 1, -1, (1 << 63) - 1, -(1 << 63), 1473884015873122059, 1473884015873122059, 42]
    r = bind_mod.rules("1.19.x~26.1")
    codes, tiers = engine.phase1_codes(seeds=seeds, rect=(-6, 6, -6, 6), max_height=-50)
    for i, s in enumerate(seeds):
        c, t, _, _ = port.phase1_rect(s, r, -50, (-6, 6, -6, 6))
        assert np.array_equal(codes[i], c) and np.array_equal(tiers[i], t)
    assert np.array_equal(codes[5], codes[6])


def test_generator_wraps_at_2_64(engine, port, bind_mod):
    base = (1 << 64) - 100
    res = engine.seed_check(gen=(base, 200), rect=RECT9, max_height=100)
    want, hist = port.scan_seeds(bind_mod.rules("1.19.x~26.1"), 100, RECT9, gen=(base, 200))
    assert np.array_equal(res.candidates, want) and res.stats["reject_hist"] == hist.tolist()


def test_empty_request_is_an_error(engine, wg):
    with pytest.raises(wg.EngineError, match="status 1"):
        engine.seed_check(seeds=[1], rect=(3, 3, 0, 5))
    with pytest.raises(wg.EngineError, match="status 1"):
        engine.seed_check(gen=(1, 0), rect=RECT9)


def test_device_entry_point_equals_host(engine, wg):
    import torch
    n = 1 << 16
    seeds = torch.tensor([wg_signed(wg.splitmix64(2 + i)) for i in range(n)], dtype=torch.int64, device="cuda")
    out = torch.zeros((1024, 4), dtype=torch.int64, device="cuda")   # 1024 x 32-byte records
    o = wg.make_opts()
    stream = torch.cuda.current_stream()
    found, st = engine.seed_check_device(seeds.data_ptr(), 0, n, RECT9, -50, o, out.data_ptr(), 1024,
                                         stream.cuda_stream)
    host = engine.seed_check(gen=(2, n), rect=RECT9, max_height=-50)
    assert found == len(host.candidates)
    assert st["reject_hist"] == host.stats["reject_hist"]
    got = np.frombuffer(out[:found].cpu().numpy().tobytes(), dtype=wg.CANDIDATE_DTYPE)
    got = np.sort(got, order=["seed_index", "rz", "rx"])
    assert np.array_equal(got, host.candidates)


def test_repeat_is_deterministic(engine):
    a = engine.seed_check(gen=(11, 1 << 18), rect=RECT9, max_height=0)
    b = engine.seed_check(gen=(11, 1 << 18), rect=RECT9, max_height=0)
    assert np.array_equal(a.candidates, b.candidates) and a.stats["reject_hist"] == b.stats["reject_hist"]


@pytest.mark.parametrize("rect,mh,version,preset,salt", [((3, 4, -2, -1), -50, "1.19.x~26.1", "NORMAL", 0),
                                                         ((-40000, -39999, 17, 18), 100, "26.2", "NORMAL", 0),
                                                         ((0, 1, 0, 1), 0, "1.18.2", "NORMAL", 0),
                                                         ((5, 6, 5, 6), 0, "1.19.x~26.1", "LARGE_BIOMES", 0),
                                                         ((-7, -6, 2, 3), 100, "1.19.x~26.1", "NORMAL", 10387312)])
def test_one_region_requests_vs_oracle(engine, port, bind_mod, rect, mh, version, preset, salt):
    """One-region units take the breadth-first climate stage (tables built per erosion step):
    survivors and the whole reject histogram must equal the oracle's."""
    r = bind_mod.rules(version, preset)
    res = engine.seed_check(gen=(17, 300000), rect=rect, max_height=mh, version=version, preset=preset, salt=salt)
    want, hist = port.scan_seeds(r, mh, rect, gen=(17, 300000), salt=salt)
    assert np.array_equal(res.candidates, want)
    assert res.stats["reject_hist"] == hist.tolist()
