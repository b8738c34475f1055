"""CPU: the phase-2 golden fixtures still equal the compiled reference (oracle/_ref).

tests/golden/make_golden_p2.py wrote them from lysh; this re-evaluates a sample of every
kind on the reference itself, so a changed fixture or a changed reference build shows up
here.  Skipped when the reference library has not been built (it is built from the
reference sources, which only the development machine has).
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rules(o):
    return {"mc_1_18_2": int(o[0]), "single_biome": int(o[1]), "pre_26_2": int(o[2]), "large_biomes": int(o[3])}


def test_probe_fixtures_pinned(ref, bind_mod):
    d = np.load(os.path.join(GOLDEN, "p2_probes.npz"))
    o = d["opts"]
    for si, seed in enumerate(d["seeds"]):
        with ref.ctx(int(seed), _rules(o), -50, int(o[4])) as ctx:
            for kind in range(14):
                pts = d[f"s{si}_k{kind}_pts"][:16]
                assert np.array_equal(ctx.probe(kind, pts), d[f"s{si}_k{kind}_vals"][:16]), (si, kind)


def test_hut_fixtures_pinned(ref, bind_mod):
    h = np.load(os.path.join(GOLDEN, "p2_huts.npz"))
    rng = np.random.default_rng(0)
    for i in sorted(rng.choice(len(h["seed"]), 24, replace=False).tolist()) + [len(h["seed"]) - 1]:
        o = [h[c][i] for c in ("mc_1_18_2", "single_biome", "pre_26_2", "large_biomes", "biome_tree")]
        with ref.ctx(int(h["seed"][i]), _rules(o), -50, int(o[4])) as ctx:
            e = ctx.eval_hut(int(h["hut_x"][i]), int(h["hut_z"][i]), -50)
        for f in bind_mod.EVAL_FIELDS:
            assert e[f] == int(h[f][i]), (i, f)


def test_hut_fixture_accept_side():
    """The accept path (biome-OK, not flooded, floor under the ceiling) is covered by real finds:
    the 50 located data/finds.tsv huts (set 4) are all accepted by lysh at -50, 62 forced huts in
    all are biome-OK and dry."""
    h = np.load(os.path.join(GOLDEN, "p2_huts.npz"))
    s4 = h["set"] == 4
    assert s4.sum() == 50 and (h["ok"][s4] == 1).all() and (h["biome_ok"][s4] == 1).all()
    assert (h["flooded"][s4] == 0).all() and (h["avg_y"][s4] <= -50).all()
    assert ((h["biome_ok"] == 1) & (h["flooded"] == 0)).sum() >= 62


def test_grade_fixture_pinned(ref):
    g = json.load(open(os.path.join(GOLDEN, "p2_grade.json")))
    hits, st = ref.grade_scan(g["seed"], _rules(g["opts"]), g["max_height"], tuple(g["rect"]), g["max_y"],
                              tree=g["opts"][4])
    assert hits.tolist() == g["hits"] and [int(v) for v in st] == g["stats"]
