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


def _convert(src, dst, threads=0):
    r = subprocess.run([CLI, "-f", str(src), "--threads", str(threads), "--convert", str(dst)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return np.fromfile(dst, dtype=np.float32).reshape(-1, 3)


# lines the reference's sscanf("%lf,%lf,%lf") reads in unusual ways: blanks, signs, hex,
# inf / nan, overflow and underflow, exponents without digits, missing or extra fields
_ODD_LINES = [
    "1 ,2,3", "", "inf,nan,-0", "infinity,1,2", "-inf,+inf,+nan", "0x1p3,-0x1.8p1,+0x10",
    "1e400,-1e400,1e-400", "+-1,2,3", "1,,3", "1,2", "  ,1,2", "1.,.5,5.e2", "1e,2e+,3e-1x",
    "1.5\r", "1,2,3\r", "3.4028235e38,3.4028236e38,1.4e-45",
    "7.0064923216240854e-46,7.006492321624086e-46,-7.0064923216240862e-46", "1,2,3,4", "abc",
    "1;2;3", "1e5e,2,3", "0x1p,2,3", "0x1p4p,5,6", "1E,2E-,3", "infe,1,2", "nan(12)e,1,2",
    "-e,1,2", ".e,1,2", "0x,1,2", "\t 1.25e-3,\t-7 , 8", "00012.5000,-000.0,+.5"]


def _odd_csv(path, n=20000, seed=2):
    rng = np.random.default_rng(seed)
    forms = ["%r", "%.3f", "%e", "%+.9g", " %g", "%.20g", "%.17E", "  \t%.1f"]
    vals = rng.uniform(-1e4, 1e4, (n, 3)) * 10.0 ** rng.integers(-8, 9, (n, 3))
    fmt = rng.integers(0, len(forms), (n, 3))
    lines = [",".join(forms[f] % v for f, v in zip(fr, vr))
             for fr, vr in zip(fmt.tolist(), vals.tolist())]
    for i, e in enumerate(_ODD_LINES):
        lines.insert(int(rng.integers(0, len(lines))), e)
    path.write_text("\n".join(lines) + "\n")


@pytest.mark.parametrize("threads", [1, 3, 0])
def test_text_reader_matches_reference_reader(tmp_path, threads):
    """The multithreaded reader gives the reference reader's floats bit for bit."""
    f = tmp_path / "odd.txt"
    _odd_csv(f)
    got = _convert(f, tmp_path / "odd.f32", threads)
    exp = oracle.read_pc(str(f))
    assert got.shape == exp.shape
    assert np.array_equal(got.view(np.uint32), exp.view(np.uint32))


@pytest.mark.parametrize("ending", ["crlf", "no_final_newline", "blank_lines"])
def test_text_reader_line_endings(tmp_path, ending):
    rng = np.random.default_rng(3)
    lines = [f"{x!r},{y!r},{z!r}" for x, y, z in rng.uniform(-5, 5, (3000, 3)).tolist()]
    if ending == "crlf":
        text = "\r\n".join(lines) + "\r\n"
    elif ending == "no_final_newline":
        text = "\n".join(lines)
    else:
        text = "\n".join(lines[:1000] + ["", ""] + lines[1000:]) + "\n"
    f = tmp_path / "p.txt"
    f.write_text(text)
    for t in (1, 4):
        got = _convert(f, tmp_path / f"p{t}.f32", t)
        exp = oracle.read_pc(str(f))
        assert got.shape == exp.shape == (3002 if ending == "blank_lines" else 3000, 3)
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32))


def test_binary_points_round_trip(tmp_path):
    rng = np.random.default_rng(4)
    pts = rng.uniform(-1e3, 1e3, (4097, 3)).astype(np.float32)
    b = tmp_path / "p.f32"
    pts.tofile(b)
    t = tmp_path / "p.txt"
    _write_csv(t, pts.astype(np.float64).tolist())
    runs = [subprocess.run([CLI, "-f", str(x), "--parse-only"], capture_output=True, text=True)
            for x in (b, t)]
    assert all(r.returncode == 0 for r in runs)
    assert runs[0].stdout == runs[1].stdout
    assert np.array_equal(_convert(b, tmp_path / "q.bin"), pts)


def test_ragged_binary_file_is_an_error(tmp_path):
    b = tmp_path / "p.bin"
    b.write_bytes(b"\0" * 20)
    r = subprocess.run([CLI, "-f", str(b), "--parse-only"], capture_output=True, text=True)
    assert r.returncode == 1 and "whole number" in r.stderr


def test_missing_file_is_an_error(tmp_path):
    r = subprocess.run([CLI, "-f", str(tmp_path / "none.txt"), "--parse-only"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "Could not read" in r.stderr


@pytest.mark.gpu
def test_cli_binary_input_gives_the_text_input_rows(tmp_path):
    rng = np.random.default_rng(5)
    pts = rng.uniform(0, 30, (15000, 3)).astype(np.float32)
    t, b = tmp_path / "p.txt", tmp_path / "p.f32"
    _write_csv(t, pts.astype(np.float64).tolist())
    pts.tofile(b)
    rows = []
    for src in (t, b):
        out = tmp_path / (src.name + ".rows")
        r = subprocess.run([CLI, "-f", str(src), "-sm", "knn", "-r", "2", "-o", str(out)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        rows.append(np.fromfile(out, dtype=np.int32).reshape(-1, 5))
    # rows are neighbor sets (slot order follows the search's arrival order)
    assert np.array_equal(np.sort(rows[0], axis=1), np.sort(rows[1], axis=1))


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
