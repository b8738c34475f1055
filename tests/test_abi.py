"""CPU: the C-ABI library loads, exports every symbol include/witchgpu.h declares, and its
host-only entry points behave like the reference's option parsing; without a GPU the engine
fails loudly instead of falling back to anything."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import pytest


def declared_symbols(header: str) -> set[str]:
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(wg_[a-z0-9_]+)\s*\(", text))


def test_header_and_exports(wg):
    decl = declared_symbols(wg.HEADER_PATH)
    assert decl == set(wg.EXPORTS)
    lib = wg.library()
    for name in decl:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", wg.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (wg_[a-z0-9_]+)$", out, flags=re.M))
    assert decl <= exported


def test_struct_layouts(wg):
    assert C.sizeof(wg.Opts) == 20
    assert wg.CANDIDATE_DTYPE.itemsize == 32
    assert C.sizeof(wg.Stats) == 8 * (4 + 11 + 7 + 2 + 3) + 8 * 3 + 16 + 16


def test_job_struct_layouts_match_the_header(wg, tmp_path):
    """wg_job / wg_job_status as the C compiler lays them out = the ctypes mirrors."""
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stddef.h>\n#include <stdio.h>\n#include "witchgpu.h"\n'
        'int main(void) { printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(wg_job), offsetof(wg_job, n_seeds),'
        ' offsetof(wg_job, max_height), offsetof(wg_job, opts), sizeof(wg_job_status),'
        ' offsetof(wg_job_status, queue_ms), offsetof(wg_job_status, batch_jobs)); return 0; }\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.dirname(wg.HEADER_PATH), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(wg.Job), wg.Job.n_seeds.offset, wg.Job.max_height.offset, wg.Job.opts.offset,
            C.sizeof(wg.JobStatus), wg.JobStatus.queue_ms.offset, wg.JobStatus.batch_jobs.offset]
    assert got == want


def test_server_without_gpu_fails_loudly(wg):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(wg.EngineError, match="status 5"):
        wg.Server(0)


@pytest.mark.parametrize("name,mc,pre,tree", [("1.19.x~26.1", 0, 1, 0), ("26.2", 0, 0, 7), ("26.2~26.3", 0, 0, 0),
                                              ("1.18.2", 1, 1, 1), ("1.18.x", 1, 1, 0), ("1.21", 0, 1, 4),
                                              ("1.21.5", 0, 1, 6), ("26.3", 0, 0, 8), ("1.20.1", 0, 1, 4)])
def test_version_names(wg, name, mc, pre, tree):
    o = wg.make_opts(name)
    assert (o.mc_1_18_2, o.pre_26_2, o.biome_tree) == (mc, pre, tree)


def test_version_names_match_reference(wg, ref):
    for name in ("1.19.x~26.1", "26.2", "26.2~26.3", "1.18.2", "1.18.x", "1.21", "1.21.4", "1.21.5", "26.1",
                 "26.3", "1.20.1", "1.19.2", "1.21.x~26.1", "1.19.x"):
        o = wg.make_opts(name)
        assert (o.mc_1_18_2, o.pre_26_2, o.biome_tree) == ref.version(name), name


def test_bad_names(wg):
    with pytest.raises(ValueError):
        wg.make_opts("1.17")
    with pytest.raises(ValueError):
        wg.make_opts(preset="AMPLIFIED")
    o = wg.make_opts(preset="LARGE_BIOMES")
    assert o.large_biomes == 1 and o.single_biome == 0


def test_no_gpu_fails_loudly(wg):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(wg.EngineError, match="status 5"):
        wg.Engine(0)


def test_shard_partition(wg):
    for n in (0, 1, 7, 1 << 24, 1000003):
        for world in (1, 2, 3, 8):
            spans = [wg.shard(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1


def test_solver_struct_layouts_match_the_header(wg, tmp_path):
    src = tmp_path / "solve_layout.c"
    src.write_text(
        '#include <stddef.h>\n#include <stdio.h>\n#include "witchgpu.h"\n'
        'int main(void) { printf("%zu %zu %zu %zu %zu\\n", sizeof(wg_solve_bundle), offsetof(wg_solve_bundle, tier),'
        ' sizeof(wg_solve_hit), offsetof(wg_solve_hit, layout), sizeof(wg_solve_stats)); return 0; }\n')
    exe = tmp_path / "solve_layout"
    subprocess.run(["gcc", "-I", os.path.dirname(wg.HEADER_PATH), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [C.sizeof(wg.SolveBundle), wg.SolveBundle.tier.offset, wg.SOLVE_HIT_DTYPE.itemsize,
                   wg.SOLVE_HIT_DTYPE.fields["layout"][1], C.sizeof(wg.SolveStats)]


def test_finisher_struct_layouts_match_the_header(wg, tmp_path):
    fields = ["verdict_ok", "room_floor", "biome", "nat", "top", "refused", "no_guard", "sum_nat", "sum_top",
              "sum_no_guard", "scan_sum", "scan_min", "above53"]
    src = tmp_path / "finish_layout.c"
    src.write_text(
        '#include <stddef.h>\n#include <stdio.h>\n#include "witchgpu.h"\n'
        'int main(void) { printf("%zu %zu %zu", sizeof(wg_ms_piece), offsetof(wg_ms_piece, rails), sizeof(wg_finish_row));'
        + "".join(f' printf(" %zu", offsetof(wg_finish_row, {f}));' for f in fields) + ' return 0; }\n')
    exe = tmp_path / "finish_layout"
    subprocess.run(["gcc", "-I", os.path.dirname(wg.HEADER_PATH), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [wg.MS_PIECE_DTYPE.itemsize, wg.MS_PIECE_DTYPE.fields["rails"][1], wg.FINISH_DTYPE.itemsize]
    want += [wg.FINISH_DTYPE.fields[f][1] for f in fields]
    assert got == want
