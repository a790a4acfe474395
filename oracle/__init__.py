"""CPU oracle for the neighbor-search path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, and
only to check results or as the timed CPU reference; the library (rtnn_b200) never imports it.

- liboracle.so (oracle.c): FP32 restatement of the reference's distance and predicates,
  brute force and grid-accelerated, plus an FP64 brute force and the FP32/FP64 boundary
  pairs.
  Also the reference's point-cloud text reader (util.cpp:100-135), for the CLI's.
- _ref/refcheck: the reference's own check.cpp (sanityCheckRadius / sanityCheckKNN),
  compiled from the reference sources by oracle/Makefile.
- _ref/libref.so: the reference's calcSearchSize / MortonCode3 (grid.cu,
  helper_mortonCode.h), compiled from the reference sources.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_lib = None
_ref = None

_P = ctypes.c_void_p
_U64 = ctypes.c_uint64


def build():
    """Compiles liboracle.so (and oracle/_ref when the reference sources exist)."""
    r = subprocess.run(["make", "-s", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        for name in ("oracle_bruteforce", "oracle_grid_search", "oracle_bruteforce_fp64"):
            f = getattr(L, name)
            f.restype = ctypes.c_int
            f.argtypes = [_P, _U64, _P, _U64, ctypes.c_int, ctypes.c_float, ctypes.c_uint32, _P,
                          ctypes.c_int]
        L.oracle_grid_search_batched.restype = ctypes.c_int
        L.oracle_grid_search_batched.argtypes = [_P, _P, ctypes.c_uint32, _P, _P, ctypes.c_int,
                                                 ctypes.c_float, ctypes.c_uint32, ctypes.c_int,
                                                 _P, ctypes.c_int]
        L.oracle_boundary_pairs.restype = ctypes.c_int64
        L.oracle_boundary_pairs.argtypes = [_P, _U64, _P, _U64, ctypes.c_int, ctypes.c_float, _P,
                                            ctypes.c_int64]
        L.oracle_ref_shell_mask.restype = ctypes.c_int
        L.oracle_ref_shell_mask.argtypes = [_P] + [ctypes.c_int] * 6 + [ctypes.c_float,
                                                                         ctypes.c_float,
                                                                         ctypes.c_uint32]
        L.oracle_read_pc.restype = ctypes.c_int64
        L.oracle_read_pc.argtypes = [ctypes.c_char_p, _P, _U64]
        L.oracle_box_counts.restype = None
        L.oracle_box_counts.argtypes = [_P] + [ctypes.c_int] * 7 + [_P]
        _lib = L
    return _lib


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1, 3))


def _mode(mode):
    return 1 if mode in ("knn", 1) else 0


def _run(fn, points, queries, mode, r, k, threads):
    p = _f32(points)
    q = p if queries is None else _f32(queries)
    out = np.empty((q.shape[0], k), dtype=np.int32)
    e = fn(p.ctypes.data_as(_P), p.shape[0], q.ctypes.data_as(_P), q.shape[0], _mode(mode),
           float(r), int(k), out.ctypes.data_as(_P), int(threads))
    if e:
        raise MemoryError("oracle ran out of memory")
    return out


def bruteforce(points, queries=None, mode="radius", r=2.0, k=50, threads=0):
    """Rows sorted by (FP32 distance, index), -1 padded. O(N*Q)."""
    return _run(lib().oracle_bruteforce, points, queries, mode, r, k, threads)


def grid_search(points, queries=None, mode="radius", r=2.0, k=50, threads=0):
    """Same rows as bruteforce(), uniform-grid accelerated (OpenMP)."""
    return _run(lib().oracle_grid_search, points, queries, mode, r, k, threads)


def bruteforce_fp64(points, queries=None, mode="radius", r=2.0, k=50, threads=0):
    """Rows of the same selection rule with distances in FP64."""
    return _run(lib().oracle_bruteforce_fp64, points, queries, mode, r, k, threads)


def grid_search_batched(points, point_offsets, queries=None, query_offsets=None, mode="knn",
                        r=0.2, k=32, local=False, threads=0):
    p = _f32(points)
    po = np.ascontiguousarray(np.asarray(point_offsets, dtype=np.uint64))
    q = None if queries is None else _f32(queries)
    qo = None if query_offsets is None else np.ascontiguousarray(np.asarray(query_offsets, dtype=np.uint64))
    nq = int(po[-1]) if q is None else int(qo[-1])
    out = np.empty((nq, k), dtype=np.int32)
    e = lib().oracle_grid_search_batched(
        p.ctypes.data_as(_P), po.ctypes.data_as(_P), po.shape[0] - 1,
        None if q is None else q.ctypes.data_as(_P), None if qo is None else qo.ctypes.data_as(_P),
        _mode(mode), float(r), int(k), 1 if local else 0, out.ctypes.data_as(_P), int(threads))
    if e:
        raise MemoryError("oracle ran out of memory")
    return out


def boundary_pairs(points, queries=None, mode="radius", r=2.0, max_pairs=100000):
    """[n, 2] (query, point) pairs whose FP32 and FP64 classifications differ."""
    p = _f32(points)
    q = p if queries is None else _f32(queries)
    buf = np.empty((max_pairs, 2), dtype=np.int64)
    n = lib().oracle_boundary_pairs(p.ctypes.data_as(_P), p.shape[0], q.ctypes.data_as(_P),
                                    q.shape[0], _mode(mode), float(r), buf.ctypes.data_as(_P),
                                    max_pairs)
    return buf[:min(n, max_pairs)].copy()


def read_pc(path):
    """Points of a text file as the reference's reader gives them: [n, 3] float32."""
    L = lib()
    n = L.oracle_read_pc(os.fsencode(path), None, 0)
    if n < 0:
        raise FileNotFoundError(path)
    out = np.zeros((n, 3), dtype=np.float32)
    L.oracle_read_pc(os.fsencode(path), out.ctypes.data_as(_P), n)
    return out


def box_counts(counts, cx, cy, cz, shells=3):
    """N_s of a raster count grid counts[z, y, x] around cell (cx, cy, cz)."""
    c = np.ascontiguousarray(np.asarray(counts, dtype=np.uint32))
    dz, dy, dx = c.shape
    N = np.zeros(shells, dtype=np.uint32)
    lib().oracle_box_counts(c.ctypes.data_as(_P), dx, dy, dz, cx, cy, cz, shells,
                            N.ctypes.data_as(_P))
    return N


def ref_shell_mask(counts, cx, cy, cz, cell, max_width, knn):
    """Restated reference calcSearchSize mask on counts[z, y, x]."""
    c = np.ascontiguousarray(np.asarray(counts, dtype=np.uint32))
    dz, dy, dx = c.shape
    return int(lib().oracle_ref_shell_mask(c.ctypes.data_as(_P), dx, dy, dz, cx, cy, cz,
                                           float(cell), float(max_width), int(knn)))


def analytic_width(N, need, cell, radius, alpha=1.24):
    """Width rule of the partition: alpha * (s* + 1) * cell, s* = first s with N_s >= need."""
    for s, n in enumerate(N):
        if n >= need:
            w = np.float32(alpha) * np.float32(s + 1) * np.float32(cell)
            return float(min(w, np.float32(radius)))
    return float(radius)


# ---- the reference's own code (compiled from its sources) -------------------------------

def ref_available():
    return os.path.exists(os.path.join(REF_DIR, "refcheck")) and \
        os.path.exists(os.path.join(REF_DIR, "libref.so"))


def refcheck(points, queries, rows, mode, r, k, q_begin=None, q_end=None, procs=1):
    """Runs the reference's sanityCheckRadius / sanityCheckKNN on rows. Returns
    (passed, output). procs > 1 (KNN): the query range is split over that many
    processes, each running the reference's check on its part."""
    exe = os.path.join(REF_DIR, "refcheck")
    with tempfile.TemporaryDirectory() as d:
        pf, qf, rf = (os.path.join(d, n) for n in ("p.bin", "q.bin", "r.bin"))
        _f32(points).tofile(pf)
        if queries is None:
            qarg = "-"
        else:
            _f32(queries).tofile(qf)
            qarg = qf
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        rows.tofile(rf)
        cmd = [exe, pf, qarg, rf, "knn" if _mode(mode) else "radius", repr(float(r)), str(int(k))]
        if _mode(mode) and procs > 1:
            lo = 0 if q_begin is None else int(q_begin)
            hi = rows.shape[0] if q_end is None else int(q_end)
            cuts = np.linspace(lo, hi, procs + 1).astype(int)
            ps = [subprocess.Popen(cmd + [str(cuts[i]), str(cuts[i + 1])], stdout=subprocess.PIPE,
                                   stderr=subprocess.STDOUT, text=True)
                  for i in range(procs) if cuts[i + 1] > cuts[i]]
            outs = [pp.communicate()[0] for pp in ps]
            ok = all(pp.returncode == 0 for pp in ps) and all("REFCHECK OK" in o for o in outs)
            return ok, "".join(outs)
        if q_begin is not None:
            cmd += [str(q_begin), str(q_end)]
        res = subprocess.run(cmd, capture_output=True, text=True)
    return res.returncode == 0 and "REFCHECK OK" in res.stdout, res.stdout + res.stderr


def _reflib():
    global _ref
    if _ref is None:
        L = ctypes.CDLL(os.path.join(REF_DIR, "libref.so"))
        L.ref_calc_search_size.restype = ctypes.c_int
        L.ref_calc_search_size.argtypes = [ctypes.c_int] * 3 + [ctypes.c_uint] * 3 + \
            [_P, ctypes.c_float, ctypes.c_float, ctypes.c_uint]
        L.ref_morton3.restype = ctypes.c_uint
        L.ref_morton3.argtypes = [ctypes.c_uint] * 3
        L.ref_width_from_iter.restype = ctypes.c_float
        L.ref_width_from_iter.argtypes = [ctypes.c_int, ctypes.c_float]
        _ref = L
    return _ref


def ref_calc_search_size(counts_zyx, cx, cy, cz, cell_size, max_width, knn):
    """Reference calcSearchSize on counts[z, y, x]; returns its mask (shell iteration)."""
    c = np.asarray(counts_zyx, dtype=np.uint32)
    ref_layout = np.ascontiguousarray(c.transpose(2, 1, 0))  # (x, y, z): z fastest
    dz, dy, dx = c.shape
    return _reflib().ref_calc_search_size(cx, cy, cz, dx, dy, dz, ref_layout.ctypes.data_as(_P),
                                          float(cell_size), float(max_width), int(knn))


def ref_morton3(x, y, z):
    return int(_reflib().ref_morton3(x, y, z))


def ref_width_from_iter(it, cell):
    return float(_reflib().ref_width_from_iter(it, cell))
