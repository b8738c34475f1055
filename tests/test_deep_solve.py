"""CPU: the Deep Dive solver's restatement in oracle/ (wo_solve_task, wo_group_regions,
wo_perm_group) against the reference's own solver output (tests/golden/deep_solve.npz, written by
tests/golden/make_golden_solve.py from hut_lookup_v4 --solve5) and against planted solutions."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

M48 = (1 << 48) - 1


def planted(port, rng, want_class=None, tries=400):
    """(S, rx, rz, ox, oz, X): a random structure seed's hut in a random region and its carver state."""
    for _ in range(tries):
        S = int(rng.integers(0, 1 << 48))
        rx, rz = (int(v) for v in rng.integers(-58593, 58594, 2))
        cx, cz = C.c_int(), C.c_int()
        port.lib.wo_hut_in_region(S, rx, rz, 14357620, C.byref(cx), C.byref(cz))
        ox, oz = cx.value - 32 * rx, cz.value - 32 * rz
        if ox == 0 and oz == 0:
            continue
        vx = (ox & -ox).bit_length() - 1 if ox else 99
        vz = (oz & -oz).bit_length() - 1 if oz else 99
        cls = 3 if vx == vz else (1 if min(vx, vz) == 0 else 2)
        if want_class and cls != want_class:
            continue
        _, X = port.mineshaft_start(S, cx.value, cz.value)
        return S, rx, rz, ox, oz, X
    raise AssertionError("no planted task of that class")


@pytest.mark.parametrize("cls", [1, 2, 3])
def test_oracle_finds_planted_seeds(port, cls):
    rng = np.random.default_rng(100 + cls)
    for _ in range(4):
        S, rx, rz, ox, oz, X = planted(port, rng, cls)
        assert S in port.solve_task(X, rx, rz, ox, oz)


def test_perm_group_is_a_bijection(port):
    seen = {port.perm_group(g) for g in range(0, 1 << 20, 97)}
    assert len(seen) == len(range(0, 1 << 20, 97))


def test_reference_hits_pin_the_oracle(port, golden):
    """Every sampled reference hit is found by the oracle for its task, with nothing more, and its
    region belongs to one of the case's groups."""
    d = golden("deep_solve.npz")
    rng = np.random.default_rng(0)
    for k, (lay, rgx, rgz, tier, first, count) in enumerate(d["cases"]):
        hits = d[f"hits{k}"]
        assert len(hits) > 0
        residues = {port.perm_group(int(g)) for g in range(first, first + count)}
        by_chunk = {}
        for S, cx, cz, X in hits:
            assert int(X) == int(lay)
            by_chunk.setdefault((int(cx), int(cz)), set()).add(int(S) & M48)
        for cx, cz in list(by_chunk)[:400]:
            assert port.region_const(cx >> 5, cz >> 5) & 0xFFFFF in residues
        for i in rng.choice(len(by_chunk), min(6, len(by_chunk)), replace=False):
            cx, cz = list(by_chunk)[i]
            rx, rz = cx >> 5, cz >> 5
            assert set(port.solve_task(int(lay), rx, rz, cx - 32 * rx, cz - 32 * rz)) == by_chunk[(cx, cz)]
