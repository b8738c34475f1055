"""CPU: the phase1_scan worker's command-line contract (engine/gpu/low54/phase1_scan.cu:561-601):
usage, argument errors and a loud failure when no GPU is present."""
from __future__ import annotations

import subprocess

import pytest


def run(wg, *args, stdin=None, timeout=60):
    return subprocess.run([wg.WORKER_PATH, *args], input=stdin, capture_output=True, text=True, timeout=timeout)


def test_usage(wg):
    r = run(wg, "--help")
    assert r.returncode == 0 and "--worker" in r.stdout and "--seed-gen" in r.stdout
    assert run(wg).returncode == 2


@pytest.mark.parametrize("args", [["--seed"], ["--seed", "1", "--bogus"], ["--seed-gen", "1", "0"],
                                  ["--seed", "1", "--seed-gen", "1", "5"], ["--seed", "1", "--min-region-x", "5",
                                                                            "--max-region-x", "5"],
                                  ["--seed", "1", "--version", "9.9"], ["--seed", "1", "--quad-bases", "f"],
                                  ["--seed-list", "/nonexistent/file"]])
def test_bad_arguments(wg, args):
    r = run(wg, *args)
    assert r.returncode == 2
    assert r.stderr.strip()


def test_no_gpu_worker_fails_loudly(wg):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    r = run(wg, "--worker", stdin="--seed 1 --out x.csv\n")
    assert r.returncode == 1 and "cannot open the GPU engine" in r.stderr
    assert "WORKER_READY" not in r.stdout


def test_hut_lookup_usage_errors(wg, tmp_path):
    """The Deep Dive worker refuses bad command lines with exit 2 before touching a GPU, and without
    a GPU fails loudly (exit 1)."""
    r = subprocess.run([wg.HUT_LOOKUP_PATH, "--bogus"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 2 and "unknown arg" in r.stderr
    r = subprocess.run([wg.HUT_LOOKUP_PATH, "--regime", "33"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 2
    r = subprocess.run([wg.HUT_LOOKUP_PATH, "--solve5"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 2 and "usage" in r.stderr
    (tmp_path / "cat.txt").write_text("231564844655014 331 331\n")
    try:
        import torch
        if torch.cuda.is_available():
            return
    except ImportError:
        pass
    r = subprocess.run([wg.HUT_LOOKUP_PATH, "--catalog", "cat.txt", "--solve5", "--regime", "22"],
                       capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and "no GPU" in r.stderr


def test_quad_option_errors(wg, tmp_path):
    """--quad-bases follows the reference's checks (phase1_scan.cu:705-724): an unreadable or
    empty base list, an offset outside it, or a second seed source is refused with exit 2."""
    (tmp_path / "empty.txt").write_text("\n")
    (tmp_path / "two.txt").write_text("20015998343868 5\n")
    rect = ["--min-region-x", "0", "--max-region-x", "1", "--min-region-z", "0", "--max-region-z", "1"]
    cases = [(["--quad-bases", str(tmp_path / "missing.txt")], "cannot open"),
             (["--quad-bases", str(tmp_path / "empty.txt")], "no seeds"),
             (["--quad-bases", str(tmp_path / "two.txt"), "--quad-base-offset", "2"], "out of range"),
             (["--quad-bases", str(tmp_path / "two.txt"), "--quad-base-offset", "-1"], "out of range"),
             (["--quad-bases", str(tmp_path / "two.txt"), "--seed-gen", "1", "5"], "cannot be combined"),
             (["--quad-bases", str(tmp_path / "two.txt"), "--seed", "3"], "cannot be combined"),
             (["--max-hut-dist"], "missing value")]
    for args, msg in cases:
        r = run(wg, *rect, *args)
        assert r.returncode == 2, args
        assert msg in r.stderr, (args, r.stderr)
