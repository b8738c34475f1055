"""GPU: phase 2 (lysh_eval_hut) against the reference's own values.

The fixtures in tests/golden/ (made by tests/golden/make_golden_p2.py from the compiled
reference lysh) hold, for the same seeds and points:
  * the phase-2 probes (blended noise, raw / interpolated density, column tops, terrain info,
    computeFluid, block states, heights before and after carvers): compared bit for bit;
  * lysh_eval_hut on 1,806 forced hut positions (the 81 region huts of config-1 seeds, other
    versions and presets, the 185 config-2 phase-1 survivors, the SCAN_REFERENCE hut):
    every field of the result must be equal;
  * lysh_grade_scan of the SCAN_REFERENCE seed over its 40,000-block rect.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# fixture column -> HUT_DTYPE field
HUT_FIELDS = {"dir": "dir", "size_x": "size_x", "size_z": "size_z", "avg_y": "avg_y", "sum_h": "sum_h",
              "wet_columns": "wet_columns", "flooded": "flooded", "ok": "ok", "reject": "reject",
              "biome_ok": "biome_ok", "biome_winner": "biome_winner", "biome_qx": "biome_qx",
              "biome_qy": "biome_qy", "biome_qz": "biome_qz", "biome_occ_y": "biome_occ_y", "rx": "rx",
              "rz": "rz", "all_dry": "all_dry"}


def _opts(wg, o):
    return wg.Opts(mc_1_18_2=int(o[0]), single_biome=int(o[1]), pre_26_2=int(o[2]), large_biomes=int(o[3]),
                   biome_tree=int(o[4]))


def _mismatch(name, got, want, pts=None):
    bad = np.nonzero(~((got == want) | (np.isnan(got) & np.isnan(want))))[0] if got.dtype.kind == "f" else \
        np.nonzero(got != want)[0]
    if len(bad) == 0:
        return None
    i = bad[0]
    where = f" at {pts[i].tolist()}" if pts is not None else ""
    return f"{name}: {len(bad)} of {len(want)} differ; first{where}: gpu {got[i]!r} ref {want[i]!r}"


def test_probes_match_reference(wg, engine):
    d = np.load(os.path.join(GOLDEN, "p2_probes.npz"))
    o = _opts(wg, d["opts"])
    errors = []
    for si, seed in enumerate(d["seeds"]):
        for kind in range(14):
            pts = d[f"s{si}_k{kind}_pts"]
            want = d[f"s{si}_k{kind}_vals"]
            got = engine.p2_probe(int(seed), kind, pts, opts=o)
            msg = _mismatch(f"seed {si} kind {kind}", got, want, pts)
            if msg:
                errors.append(msg)
    assert not errors, "\n".join(errors)


def test_eval_huts_match_reference(wg, engine):
    h = np.load(os.path.join(GOLDEN, "p2_huts.npz"))
    optcols = np.stack([h["mc_1_18_2"], h["single_biome"], h["pre_26_2"], h["large_biomes"], h["biome_tree"]], 1)
    errors = []
    for key in sorted({tuple(r) for r in optcols.tolist()}):
        sel = np.nonzero((optcols == np.array(key)).all(axis=1))[0]
        res = engine.eval_huts(h["seed"][sel], h["hut_x"][sel], h["hut_z"][sel], max_y=-50, opts=_opts(wg, key))
        for col, field in HUT_FIELDS.items():
            msg = _mismatch(f"opts {key} {col}", res[field].astype(np.int64), h[col][sel])
            if msg:
                errors.append(msg)
        t = np.stack([h[f"t{k}"][sel] for k in range(6)], 1)
        if not np.array_equal(res["biome_t"], t):
            errors.append(f"opts {key} biome_t differs")
        if not (np.array_equal(res["hut_x"], h["hut_x"][sel]) and np.array_equal(res["hut_z"], h["hut_z"][sel])):
            errors.append(f"opts {key} hut position echo differs")
    assert not errors, "\n".join(errors)


def test_eval_huts_scan_reference_hut(engine):
    # the reference project's known answer: /tp -15792 -54 -17168 (hunt.py SCAN_REFERENCE)
    res = engine.eval_huts([1473884015873122059], [-15792], [-17168], max_y=-50)
    r = res[0]
    assert (r["ok"], r["avg_y"], r["biome_ok"], r["flooded"]) == (1, -54, 1, 0)


def test_grade_scan_matches_reference(wg, engine):
    g = json.load(open(os.path.join(GOLDEN, "p2_grade.json")))
    hits, counts = engine.grade_scan(g["seed"], tuple(g["rect"]), max_height=g["max_height"], max_y=g["max_y"],
                                     opts=_opts(wg, g["opts"]))
    assert hits.tolist() == g["hits"]
    st = g["stats"]
    assert [counts["scanned"], counts["evaluated"], counts["accepted"], counts["rejected_y"],
            counts["rejected_flood"], counts["rejected_biome"], counts["hits_written"]] == st


def test_eval_huts_empty_and_bad_args(wg, engine):
    assert len(engine.eval_huts([], [], [])) == 0
    with pytest.raises(ValueError):
        engine.eval_huts([1, 2], [0], [0])
    with pytest.raises(wg.EngineError):
        engine.p2_probe(1, 99, [(0, 0, 0)])
