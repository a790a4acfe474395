"""C-ABI library: loads, exports every declared symbol, rejects bad calls (CPU only)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import rtnn_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w \*]*?\b(rtnn_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(rtnn_b200.library_path())
    names = _declared()
    assert "rtnn_search" in names and "rtnn_search_batched" in names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol():
    lib = rtnn_b200.load_library()
    for n in _declared():
        assert n in rtnn_b200._SIGS, f"{n} has no Python binding"
        assert getattr(lib, n).argtypes is not None


def test_version_and_k_range():
    lib = rtnn_b200.load_library()
    assert b"sm_100a" in lib.rtnn_version()
    assert lib.rtnn_k_supported(1) == 1 and lib.rtnn_k_supported(rtnn_b200.MAX_K) == 1
    assert lib.rtnn_k_supported(0) == 0 and lib.rtnn_k_supported(rtnn_b200.MAX_K + 1) == 0
    # the K values with kernels compiled in (the benchmark configurations' K among them)
    assert [k for k in range(0, 130) if lib.rtnn_k_compiled(k)] == [5, 8, 16, 32, 50, 64]


def test_model_size_matches_layout():
    lib = rtnn_b200.load_library()
    F, H = rtnn_b200.MODEL_FEATURES, rtnn_b200.MODEL_HIDDEN
    assert lib.rtnn_model_size() == 2 * F + 2 + H * F + H + H * H + H + H + 1


def test_python_model_constants_match_header():
    hdr = open(os.path.join(ROOT, "include", "rtnn_learn.h")).read()
    feats = int(re.search(r"#define RTNN_MODEL_FEATURES (\d+)", hdr).group(1))
    norm = int(re.search(r"#define RTNN_MODEL_NORM_PARAMS (\d+)", hdr).group(1))
    hidden = int(re.search(r"#define RTNN_MODEL_HIDDEN (\d+)", hdr).group(1))
    assert (feats, norm) == (rtnn_b200.MODEL_FEATURES, rtnn_b200.MODEL_NORM_PARAMS)
    assert hidden == rtnn_b200.MODEL_HIDDEN
    from oracle import mlp
    assert (mlp.F, mlp.H, mlp.NORM) == (feats, hidden, norm)
    assert norm == 2 * feats + 2


def test_python_flags_match_header():
    hdr = open(os.path.join(ROOT, "include", "rtnn.h")).read()
    flags = dict(re.findall(r"#define RTNN_FLAG_(\w+)\s+(0x[0-9a-fA-F]+)u", hdr))
    assert {"DEVICE_POINTERS", "ANY_K", "KEEP_ORDER"} <= set(flags)
    for name, value in flags.items():
        assert getattr(rtnn_b200, "FLAG_" + name) == int(value, 16), name
    assert len(set(flags.values())) == len(flags)


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_have_gpu(), reason="checks the no-device error path")
def test_create_without_device_reports_no_device():
    with pytest.raises(rtnn_b200.RtnnError) as e:
        rtnn_b200.Context(0)
    assert e.value.code == "RTNN_ERR_NO_DEVICE"


def test_null_context_is_rejected():
    lib = rtnn_b200.load_library()
    out = np.zeros(4, dtype=np.int32)
    st = lib.rtnn_search(None, None, 0, None, 0, 0, 1.0, 1, 0, out.ctypes.data_as(ctypes.c_void_p), None)
    assert st == 1  # RTNN_ERR_INVALID_ARGUMENT
    assert lib.rtnn_destroy(None) == 0
    assert lib.rtnn_plan_destroy(None) == 0


def test_mode_names():
    assert rtnn_b200._mode("radius") == rtnn_b200.RADIUS
    assert rtnn_b200._mode("knn") == rtnn_b200.KNN
    with pytest.raises(ValueError):
        rtnn_b200._mode("nearest")


def test_headers_are_c99_and_link_from_c(tmp_path):
    """The public headers compile as strict C99 and a C program links against the library
    (what a cgo or plain-C caller does); without a GPU, rtnn_create reports an error
    status instead of crashing."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("gcc not found")
    src = tmp_path / "caller.c"
    src.write_text('#include "rtnn.h"\n#include "rtnn_learn.h"\n'
                   "int main(void) {\n"
                   "  rtnn_ctx* c = 0; rtnn_stats s; rtnn_tuning t; (void)s; (void)t;\n"
                   "  rtnn_status st = rtnn_create(&c, 0);\n"
                   "  if (st == RTNN_OK) { rtnn_destroy(c); return 0; }\n"
                   "  return 1;\n}\n")
    lib_dir = os.path.dirname(rtnn_b200.library_path())
    exe = tmp_path / "caller"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                    "-I" + os.path.join(ROOT, "include"), str(src), "-L" + lib_dir,
                    "-lrtnn_b200", "-Wl,-rpath," + lib_dir, "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, timeout=120)
    assert r.returncode in (0, 1)


def test_python_structs_match_the_c_layout(tmp_path):
    """The ctypes mirrors of rtnn_tuning and rtnn_stats have the C structs' sizes and field
    offsets (a field added to the header without the Python mirror would shift every
    later field)."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("gcc not found")
    checks = []
    for cname, py in (("rtnn_tuning", rtnn_b200.Tuning), ("rtnn_stats", rtnn_b200.Stats)):
        checks.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            checks.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "rtnn.h"\n'
                   "int main(void) {\n  " + "\n  ".join(checks) + "\n  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I" + os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out.splitlines()}
    for cname, py in (("rtnn_tuning", rtnn_b200.Tuning), ("rtnn_stats", rtnn_b200.Stats)):
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
