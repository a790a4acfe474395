"""The rebuilt optixNSearch CLI: flags and the reference's CSV format (CPU), and a full
run checked against the oracle (GPU)."""
import os
import subprocess

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "rtnn_b200", "bin", "optixNSearch")


def _write_csv(path, pts):
    with open(path, "w") as f:
        for x, y, z in pts:
            f.write(f"{x!r},{y!r},{z!r}\n")


def test_help_lists_reference_flags():
    r = subprocess.run([CLI, "-h"], capture_output=True, text=True)
    assert r.returncode == 0
    for flag in ("-f", "-q", "-sm", "-r", "-k", "-d", "-c", "-p"):
        assert f"| {flag} " in r.stderr or f"| {flag}  " in r.stderr, flag


def test_csv_parsed_as_double_then_float(tmp_path):
    rng = np.random.default_rng(0)
    pts = rng.uniform(-1e3, 1e3, (257, 3))
    f = tmp_path / "p.txt"
    _write_csv(f, pts.tolist())
    r = subprocess.run([CLI, "-f", str(f), "--parse-only"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    n, s = r.stdout.split()[1], float(r.stdout.split()[3])
    assert int(n) == 257
    assert s == pytest.approx(float(pts.astype(np.float32).astype(np.float64).sum()), rel=1e-9)


def test_bad_mode_prints_usage(tmp_path):
    r = subprocess.run([CLI, "-f", "x", "-sm", "nearest"], capture_output=True, text=True)
    assert "Usage" in r.stderr


def test_ignored_reference_flags_warn(tmp_path):
    f = tmp_path / "p.txt"
    _write_csv(f, [[0.0, 0.0, 0.0]])
    r = subprocess.run([CLI, "-f", str(f), "-ps", "1", "-a", "2", "--parse-only"],
                       capture_output=True, text=True)
    assert r.returncode == 0 and "has no effect" in r.stderr


def test_empty_input_exits_cleanly(tmp_path):
    f = tmp_path / "empty.txt"
    f.write_text("")
    r = subprocess.run([CLI, "-f", str(f)], capture_output=True, text=True)
    assert r.returncode == 0 and "empty query and/or points" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("mode,r,k", [("radius", 3.0, 50), ("knn", 3.0, 5)])
def test_cli_run_matches_oracle(tmp_path, mode, r, k):
    rng = np.random.default_rng(1)
    pts = rng.uniform(0, 40, (20000, 3)).astype(np.float64)
    f = tmp_path / "p.txt"
    _write_csv(f, pts.tolist())
    out = tmp_path / "rows.bin"
    cmd = [CLI, "-f", str(f), "-sm", mode, "-r", str(r), "-c", "1", "-o", str(out)]
    if mode == "radius":
        cmd += ["-k", str(k)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "Sanity check done." in res.stderr
    rows = np.fromfile(out, dtype=np.int32).reshape(-1, k)
    exp = oracle.grid_search(pts.astype(np.float32), None, mode, r, k)
    big = np.iinfo(np.int32).max
    srt = lambda a: np.sort(np.where(a < 0, big, a), axis=1)
    assert np.array_equal(srt(rows), srt(exp))
