"""GPU: the mineshaft finisher (wg_mineshaft_tree, wg_finish_rows) against the reference's own
finisher tools (tests/golden/finish_rows.npz from oracle/_ref's lysh, mstree, biome_at, msroom and
skyscan, as hunt.py's finish_row runs them): trees piece for piece, then every value finish_row
reads, on hunt.py's REFERENCE, the TERRAIN_REFERENCE spots, the 50 located data/finds.tsv huts,
random-seed starts and non-start chunks."""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
LETTER = {0: ord("R"), 1: ord("C"), 2: ord("X"), 3: ord("Y"), 4: ord("S")}


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(GOLDEN, "finish_rows.npz"))


def test_trees_equal_mstree(engine, wg, fx):
    off = np.concatenate([[0], np.cumsum(fx["n_pieces"])])
    for i in range(len(fx["ws"])):
        ws, cx, cz = int(fx["ws"][i]), int(fx["cx"][i]), int(fx["cz"][i])
        if not fx["start"][i]:
            with pytest.raises(wg.EngineError):
                engine.mineshaft_tree(ws, cx, cz)
            continue
        pieces, floor = engine.mineshaft_tree(ws, cx, cz)
        want = fx["pieces"][off[i]:off[i + 1]]
        got = np.stack([pieces[f] for f in ("kind", "x0", "y0", "z0", "x1", "y1", "z1", "facing", "parent",
                                            "rails")], 1)
        want = want.copy()
        want[:, 0] = [LETTER[int(k)] for k in want[:, 0]]
        assert np.array_equal(got, want), i
        assert floor == int(fx["floor"][i]) == int(want[0, 2])


def test_finish_rows_equal_the_reference_tools(engine, fx):
    rows = engine.finish_rows(fx["ws"], fx["cx"], fx["cz"])
    start = fx["start"] == 1
    assert rows["verdict_ok"].tolist() == fx["verdict_ok"].tolist()
    assert rows["tree_status"].tolist() == [0 if s else 1 for s in start]
    assert rows["pieces"][start].tolist() == fx["n_pieces"][start].tolist()
    assert rows["room_floor"][start].tolist() == fx["floor"][start].tolist()
    assert rows["biome"][start, 0].tolist() == fx["biome0"][start].tolist()
    assert rows["biome"][start, 1].tolist() == fx["biome1"][start].tolist()
    assert rows["nat"][start].tolist() == fx["nat"][start].tolist()
    for k in range(2):
        assert rows["sum_top"][start, k].tolist() == fx[f"top{k}_sum"][start].tolist(), k
        assert rows["top"][start, k].tolist() == fx[f"top{k}"][start].tolist(), k
        assert rows["refused"][start, k].tolist() == fx["refused"][start, k].tolist(), k
        assert rows["sum_no_guard"][start, k].tolist() == fx[f"ng{k}_sum"][start].tolist(), k
        assert rows["no_guard"][start, k].tolist() == fx[f"ng{k}"][start].tolist(), k
    # skyscan --list (its mean printed with two decimals)
    assert [f"{s / 63:.2f}" for s in rows["scan_sum"][start]] == [f"{m:.2f}" for m in fx["scan_mean"][start]]
    for name in ("scan_min", "scan_max", "le54", "lava", "solid", "nw", "ne", "sw", "se", "above53"):
        assert rows[name][start].tolist() == fx[name][start].tolist(), name


def test_finish_reference_line(engine):
    """hunt.py's REFERENCE (hunt.py:83): accepted, a start, the mineshaft floor at -58."""
    r = engine.finish_rows([3159335117276934358], [-1852878], [-1380275])[0]
    assert (r["verdict_ok"], r["tree_status"], r["room_floor"], r["nat"], r["top"][1]) == (1, 0, -62, -53, -58)
