"""rtnn_b200 -- B200-native fixed-radius and KNN neighbor search (host-side mirror).

Python mirror of the reference's search interface: the `optixNSearch` flags
-f/-q/-sm/-r/-k/-d (src/optixNSearch/util.cpp:137-383) become the arguments of
`search()`, and its per-query K-slot index buffer with the UINT_MAX fill
(search.cpp:18) is the returned [Q, K] int32 array with -1 in unused slots.
Everything runs in librtnn_b200.so (CUDA, sm_100a) through its C ABI (include/rtnn.h);
this module only marshals arguments. There is no CPU fallback: importing the package
fails loudly when the library is missing, and every call needs a CUDA device.
"""
import ctypes
import os

import numpy as np

__all__ = ["RtnnError", "Stats", "Tuning", "Context", "Plan", "search", "search_batched",
           "RADIUS", "KNN", "FLAG_DEVICE_POINTERS", "FLAG_PARTITION", "FLAG_LEARNED",
           "FLAG_SORTED_ROWS", "FLAG_LOCAL_INDICES", "FLAG_ANY_K", "FLAG_KEEP_ORDER",
           "FLAG_REF_LAYOUT", "MAX_K", "from_ref_layout",
           "library_path", "load_library"]

RADIUS = 0
KNN = 1
FLAG_DEVICE_POINTERS = 0x1
FLAG_PARTITION = 0x2
FLAG_LEARNED = 0x4
FLAG_SORTED_ROWS = 0x8
FLAG_LOCAL_INDICES = 0x10
FLAG_ANY_K = 0x20
FLAG_KEEP_ORDER = 0x40
FLAG_REF_LAYOUT = 0x80
MAX_K = 128
MODEL_FEATURES = 6   # RTNN_MODEL_FEATURES
MODEL_HIDDEN = 16    # RTNN_MODEL_HIDDEN
MODEL_NORM_PARAMS = 2 * MODEL_FEATURES + 2   # RTNN_MODEL_NORM_PARAMS

_STATUS = {
    0: "RTNN_OK", 1: "RTNN_ERR_INVALID_ARGUMENT", 2: "RTNN_ERR_CUDA",
    3: "RTNN_ERR_OUT_OF_MEMORY", 4: "RTNN_ERR_UNSUPPORTED_K", 5: "RTNN_ERR_DEVICE_TIMEOUT",
    6: "RTNN_ERR_NO_DEVICE", 7: "RTNN_ERR_NO_MODEL", 8: "RTNN_ERR_INTERNAL",
}

_HERE = os.path.dirname(os.path.abspath(__file__))


def library_path():
    return os.path.join(_HERE, "lib", "librtnn_b200.so")


class RtnnError(RuntimeError):
    def __init__(self, status, message):
        self.status = status
        self.code = _STATUS.get(status, str(status))
        super().__init__(f"{self.code}: {message}")


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_points", ctypes.c_uint64), ("n_queries", ctypes.c_uint64),
        ("n_clouds", ctypes.c_uint32), ("n_buckets", ctypes.c_uint32),
        ("n_fallback", ctypes.c_uint64), ("n_tiles", ctypes.c_uint64),
        ("n_cells", ctypes.c_uint64), ("cell_size", ctypes.c_float),
        ("grid_dims", ctypes.c_uint32 * 3),
        ("ms_build", ctypes.c_float), ("ms_partition", ctypes.c_float),
        ("ms_search", ctypes.c_float), ("ms_total", ctypes.c_float),
        ("n_launches", ctypes.c_uint32), ("ms_fallback", ctypes.c_float),
        ("n_loaded", ctypes.c_uint64), ("n_tested", ctypes.c_uint64),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["grid_dims"] = list(self.grid_dims)
        return d


class Tuning(ctypes.Structure):
    _fields_ = [("cell_ratio", ctypes.c_float), ("min_cell_ratio", ctypes.c_float),
                ("points_per_cell", ctypes.c_float), ("cell_budget", ctypes.c_float),
                ("warps_per_block", ctypes.c_uint32), ("blocks_per_sm", ctypes.c_uint32),
                ("width_margin", ctypes.c_float), ("fallback_passes", ctypes.c_uint32),
                ("lane_walk_ratio", ctypes.c_float), ("gap_ratio", ctypes.c_float),
                ("pending_slots", ctypes.c_uint32), ("query_warps", ctypes.c_uint32),
                ("buckets_per_halving", ctypes.c_float), ("width_model", ctypes.c_uint32),
                ("width_clip", ctypes.c_uint32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None

_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_F = ctypes.c_float
_I = ctypes.c_int
_SIGS = {
    "rtnn_version": (ctypes.c_char_p, []),
    "rtnn_k_supported": (_I, [_U32]),
    "rtnn_k_compiled": (_I, [_U32]),
    "rtnn_create": (_I, [ctypes.POINTER(_P), _I]),
    "rtnn_destroy": (_I, [_P]),
    "rtnn_last_error": (ctypes.c_char_p, [_P]),
    "rtnn_set_stream": (_I, [_P, _P]),
    "rtnn_get_tuning": (_I, [_P, ctypes.POINTER(Tuning)]),
    "rtnn_set_tuning": (_I, [_P, ctypes.POINTER(Tuning)]),
    "rtnn_search": (_I, [_P, _P, _U64, _P, _U64, _I, _F, _U32, _U32, _P, ctypes.POINTER(Stats)]),
    "rtnn_search_batched": (_I, [_P, _P, _P, _U32, _P, _P, _I, _F, _U32, _U32, _P,
                                 ctypes.POINTER(Stats)]),
    "rtnn_plan_create": (_I, [_P, ctypes.POINTER(_P), _P, _U32, _P, _I, _F, _U32, _U32, _I]),
    "rtnn_plan_execute": (_I, [_P, _P, _P, _P, ctypes.POINTER(Stats)]),
    "rtnn_plan_destroy": (_I, [_P]),
    "rtnn_plan_resort": (_I, [_P]),
    "rtnn_model_size": (_U32, []),
    "rtnn_model_set": (_I, [_P, _P, _U32]),
    "rtnn_model_get": (_I, [_P, _P, _U32]),
    "rtnn_collect_training": (_I, [_P, _P, _U64, _P, _U64, _I, _F, _U32, _P, _P,
                                   ctypes.POINTER(_U64)]),
    "rtnn_model_train": (_I, [_P, _P, _P, _U64, _U32, _U32, _F, _U64, _P]),
    "rtnn_query_widths": (_I, [_P, _P, _U64, _P, _U64, _I, _F, _U32, _U32, _P]),
    "rtnn_mlp_loss_grad": (_I, [_P, _P, _P, _P, _U32, _P, _P]),
    "rtnn_mlp_forward": (_I, [_P, _P, _P, _U32, _P]),
    "rtnn_mlp_adam_step": (_I, [_P, _P, _P, _P, _P, _F, _U32, _F]),
    "rtnn_search_noalloc": (_I, [_P, _U32, _P, _U32, _I, _F, _U32, _P, _P, ctypes.c_char_p,
                                 ctypes.c_size_t]),
    "rtnn_selftest_wait_timeout": (_I, [_P]),
    "rtnn_sort_pairs": (_I, [_P, _P, _U32, _P, _U64, _U32]),
    "rtnn_layout": (_I, [_P, _P, _U64, _P, _U64, _U32]),
}


def load_library():
    """Loads librtnn_b200.so (built by rtnn_b200/build.py); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise ImportError(f"rtnn_b200: CUDA library not built ({path}); run "
                          f"`python -m rtnn_b200.build` or __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _host_f32(a, name):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if a.ndim != 2 or a.shape[1] != 3:
        raise ValueError(f"{name} must have shape [n, 3]")
    return a


class Context:
    """One device context (rtnn_create). Not thread-safe; one per host thread."""

    def __init__(self, device=0):
        lib = load_library()
        h = _P()
        st = lib.rtnn_create(ctypes.byref(h), int(device))
        if st != 0:
            raise RtnnError(st, f"rtnn_create(device={device}) failed")
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            load_library().rtnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st):
        if st != 0:
            msg = load_library().rtnn_last_error(self._h)
            raise RtnnError(st, msg.decode() if msg else "")

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr):
        self._check(load_library().rtnn_set_stream(self._h, _P(stream_ptr)))

    def tuning(self):
        t = Tuning()
        self._check(load_library().rtnn_get_tuning(self._h, ctypes.byref(t)))
        return t

    def set_tuning(self, **kw):
        t = self.tuning()
        for k_, v in kw.items():
            setattr(t, k_, v)
        self._check(load_library().rtnn_set_tuning(self._h, ctypes.byref(t)))

    # -- single cloud -------------------------------------------------------------------
    def search(self, points, queries=None, mode="radius", radius=2.0, k=50, partition=False,
               learned=False, sorted_rows=False, any_k=False, ref_layout=False, out=None,
               stats=None):
        """Neighbors of every query: [Q, k] int32, -1 in unused slots.

        points / queries: numpy [n, 3] float32 (host; copies happen inside the call) or
        CUDA torch tensors [n, 3] float32 (device; `out` may be a preallocated CUDA
        int32 tensor [Q, k]). mode: "radius" (self included) or "knn" (0 < d < r^2).
        any_k: any K qualifying points (the reference's radius semantics) instead of the
        K nearest. ref_layout: rows in the engine's sorted query order holding positions in
        its sorted point copy (the reference's layout); layout() maps them back.
        """
        lib = load_library()
        m = _mode(mode)
        flags = ((FLAG_PARTITION if partition else 0) | (FLAG_LEARNED if learned else 0) |
                 (FLAG_SORTED_ROWS if sorted_rows else 0) | (FLAG_ANY_K if any_k else 0) |
                 (FLAG_REF_LAYOUT if ref_layout else 0))
        st = stats if stats is not None else Stats()
        if _is_torch(points):
            import torch
            assert points.is_cuda and points.dtype == torch.float32 and points.is_contiguous()
            nq = points.shape[0] if queries is None else queries.shape[0]
            if queries is not None:
                assert queries.is_cuda and queries.dtype == torch.float32 and queries.is_contiguous()
            if out is None:
                out = torch.empty((nq, k), dtype=torch.int32, device=points.device)
            self._check(lib.rtnn_search(self._h, _P(points.data_ptr()), points.shape[0],
                                        _P(queries.data_ptr()) if queries is not None else None,
                                        nq, m, float(radius), int(k),
                                        flags | FLAG_DEVICE_POINTERS, _P(out.data_ptr()),
                                        ctypes.byref(st)))
            return out
        p = _host_f32(points, "points")
        q = None if queries is None else _host_f32(queries, "queries")
        nq = p.shape[0] if q is None else q.shape[0]
        if out is None:
            out = np.empty((nq, k), dtype=np.int32)
        self._check(lib.rtnn_search(self._h, p.ctypes.data_as(_P), p.shape[0],
                                    None if q is None else q.ctypes.data_as(_P), nq, m,
                                    float(radius), int(k), flags, out.ctypes.data_as(_P),
                                    ctypes.byref(st)))
        return out

    # -- many clouds --------------------------------------------------------------------
    def search_batched(self, points, point_offsets, queries=None, query_offsets=None,
                       mode="knn", radius=0.2, k=32, partition=False, learned=False,
                       sorted_rows=False, local_indices=False, any_k=False, ref_layout=False,
                       out=None, stats=None):
        """Many independent clouds in one launch; offsets have n_clouds + 1 entries."""
        lib = load_library()
        po = np.ascontiguousarray(np.asarray(point_offsets, dtype=np.uint64))
        qo = (None if query_offsets is None
              else np.ascontiguousarray(np.asarray(query_offsets, dtype=np.uint64)))
        n_clouds = po.shape[0] - 1
        flags = ((FLAG_PARTITION if partition else 0) | (FLAG_LEARNED if learned else 0) |
                 (FLAG_SORTED_ROWS if sorted_rows else 0) | (FLAG_LOCAL_INDICES if local_indices else 0) |
                 (FLAG_ANY_K if any_k else 0) | (FLAG_REF_LAYOUT if ref_layout else 0))
        st = stats if stats is not None else Stats()
        nq = int(po[-1]) if queries is None else int(qo[-1])
        if _is_torch(points):
            import torch
            if out is None:
                out = torch.empty((nq, k), dtype=torch.int32, device=points.device)
            self._check(lib.rtnn_search_batched(
                self._h, _P(points.data_ptr()), po.ctypes.data_as(_P), n_clouds,
                _P(queries.data_ptr()) if queries is not None else None,
                qo.ctypes.data_as(_P) if qo is not None else None, _mode(mode), float(radius),
                int(k), flags | FLAG_DEVICE_POINTERS, _P(out.data_ptr()), ctypes.byref(st)))
            return out
        p = _host_f32(points, "points")
        q = None if queries is None else _host_f32(queries, "queries")
        if out is None:
            out = np.empty((nq, k), dtype=np.int32)
        self._check(lib.rtnn_search_batched(
            self._h, p.ctypes.data_as(_P), po.ctypes.data_as(_P), n_clouds,
            None if q is None else q.ctypes.data_as(_P),
            None if qo is None else qo.ctypes.data_as(_P), _mode(mode), float(radius), int(k),
            flags, out.ctypes.data_as(_P), ctypes.byref(st)))
        return out

    def plan(self, point_offsets, query_offsets=None, mode="knn", radius=0.2, k=32,
             partition=False, learned=False, sorted_rows=False, local_indices=False,
             use_graph=True, any_k=False, keep_order=False):
        """keep_order (RTNN_FLAG_KEEP_ORDER): the first execute sorts the queries and later
        executes reuse that order, skipping the query keys and sort (time stepping);
        Plan.resort() makes the next execute sort again."""
        return Plan(self, point_offsets, query_offsets, mode, radius, k, partition, learned,
                    sorted_rows, local_indices, use_graph, any_k, keep_order)

    # -- learned widths -------------------------------------------------------------------
    def model_size(self):
        return int(load_library().rtnn_model_size())

    def set_model(self, params):
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float32))
        self._check(load_library().rtnn_model_set(self._h, p.ctypes.data_as(_P), p.size))

    def get_model(self):
        p = np.empty(self.model_size(), dtype=np.float32)
        self._check(load_library().rtnn_model_get(self._h, p.ctypes.data_as(_P), p.size))
        return p

    def collect_training(self, points, queries=None, mode="knn", radius=2.0, k=16):
        """(features [S, 6], targets [S]) as CUDA tensors from one plain search
        (rtnn_collect_training): one sample per query, or one per 32-query tile when the
        context's tuning has width_model = 1."""
        import torch
        nq = points.shape[0] if queries is None else queries.shape[0]
        cap = max(1, nq if self.tuning().width_model == 0 else (nq + 31) // 32)
        feats = torch.empty((cap, MODEL_FEATURES), dtype=torch.float32, device=points.device)
        tgt = torch.empty((cap,), dtype=torch.float32, device=points.device)
        n = _U64(0)
        self._check(load_library().rtnn_collect_training(
            self._h, _P(points.data_ptr()), points.shape[0],
            _P(queries.data_ptr()) if queries is not None else None, nq, _mode(mode),
            float(radius), int(k), _P(feats.data_ptr()), _P(tgt.data_ptr()), ctypes.byref(n)))
        return feats[:n.value], tgt[:n.value]

    def train_model(self, feats, target, epochs=20, batch=8192, lr=3e-3, seed=0):
        """Trains the width model on the GPU; returns the per-epoch mean loss."""
        losses = np.zeros(epochs, dtype=np.float32)
        self._check(load_library().rtnn_model_train(
            self._h, _P(feats.data_ptr()), _P(target.data_ptr()), feats.shape[0], int(epochs),
            int(batch), float(lr), int(seed), losses.ctypes.data_as(_P)))
        return losses

    def query_widths(self, points, queries=None, mode="knn", radius=2.0, k=16, learned=False):
        """Per-query partition widths (CUDA tensor, query order)."""
        import torch
        nq = points.shape[0] if queries is None else queries.shape[0]
        w = torch.empty((nq,), dtype=torch.float32, device=points.device)
        self._check(load_library().rtnn_query_widths(
            self._h, _P(points.data_ptr()), points.shape[0],
            _P(queries.data_ptr()) if queries is not None else None, nq, _mode(mode),
            float(radius), int(k), FLAG_LEARNED if learned else 0, _P(w.data_ptr())))
        return w

    def mlp_loss_grad(self, params, feats, target):
        import torch
        n_train = self.model_size() - MODEL_NORM_PARAMS
        grad = torch.zeros(n_train, dtype=torch.float32, device=feats.device)
        loss = torch.zeros(1, dtype=torch.float32, device=feats.device)
        self._check(load_library().rtnn_mlp_loss_grad(
            self._h, _P(params.data_ptr()), _P(feats.data_ptr()), _P(target.data_ptr()),
            feats.shape[0], _P(grad.data_ptr()), _P(loss.data_ptr())))
        return grad, loss

    def mlp_forward(self, params, feats):
        import torch
        y = torch.empty(feats.shape[0], dtype=torch.float32, device=feats.device)
        self._check(load_library().rtnn_mlp_forward(
            self._h, _P(params.data_ptr()), _P(feats.data_ptr()), feats.shape[0], _P(y.data_ptr())))
        return y

    def layout(self, n_points, n_queries, device=False):
        """(point_order, query_order) of the last search (rtnn_layout): numpy uint32 arrays,
        or CUDA int32 tensors with device=True."""
        lib = load_library()
        if device:
            import torch
            po = torch.empty(n_points, dtype=torch.int32, device=f"cuda:{self.device}")
            qo = torch.empty(n_queries, dtype=torch.int32, device=f"cuda:{self.device}")
            self._check(lib.rtnn_layout(self._h, _P(po.data_ptr()), n_points, _P(qo.data_ptr()),
                                        n_queries, FLAG_DEVICE_POINTERS))
            return po, qo
        po = np.empty(n_points, dtype=np.uint32)
        qo = np.empty(n_queries, dtype=np.uint32)
        self._check(lib.rtnn_layout(self._h, po.ctypes.data_as(_P), n_points,
                                    qo.ctypes.data_as(_P), n_queries, 0))
        return po, qo

    def sort_pairs(self, keys, values, key_bits=None):
        """Sorts CUDA tensors keys (int32/uint32 or int64/uint64) and values (int32, the same
        length) in place by the low key_bits bits of the keys, stably (rtnn_sort_pairs)."""
        kb = keys.element_size()
        bits = 8 * kb if key_bits is None else int(key_bits)
        self._check(load_library().rtnn_sort_pairs(self._h, _P(keys.data_ptr()), kb,
                                                   _P(values.data_ptr()), keys.numel(), bits))
        return keys, values

    def mlp_adam_step(self, params, grad, m, v, lr, step, grad_scale):
        self._check(load_library().rtnn_mlp_adam_step(
            self._h, _P(params.data_ptr()), _P(grad.data_ptr()), _P(m.data_ptr()),
            _P(v.data_ptr()), float(lr), int(step), float(grad_scale)))


class Plan:
    """Fixed-shape batched search replayed from a CUDA graph (rtnn_plan_*)."""

    def __init__(self, ctx, point_offsets, query_offsets, mode, radius, k, partition, learned,
                 sorted_rows, local_indices, use_graph, any_k=False, keep_order=False):
        self.ctx = ctx
        lib = load_library()
        po = np.ascontiguousarray(np.asarray(point_offsets, dtype=np.uint64))
        qo = (None if query_offsets is None
              else np.ascontiguousarray(np.asarray(query_offsets, dtype=np.uint64)))
        flags = ((FLAG_PARTITION if partition else 0) | (FLAG_LEARNED if learned else 0) |
                 (FLAG_SORTED_ROWS if sorted_rows else 0) | (FLAG_LOCAL_INDICES if local_indices else 0) |
                 (FLAG_ANY_K if any_k else 0) | (FLAG_KEEP_ORDER if keep_order else 0))
        self.k = k
        self.n_queries = int((qo if qo is not None else po)[-1])
        h = _P()
        ctx._check(lib.rtnn_plan_create(ctx._h, ctypes.byref(h), po.ctypes.data_as(_P),
                                        po.shape[0] - 1,
                                        None if qo is None else qo.ctypes.data_as(_P),
                                        _mode(mode), float(radius), int(k), flags,
                                        1 if use_graph else 0))
        self._h = h

    def execute(self, points, queries=None, out=None, stats=None):
        import torch
        if out is None:
            out = torch.empty((self.n_queries, self.k), dtype=torch.int32, device=points.device)
        st = stats if stats is not None else Stats()
        self.ctx._check(load_library().rtnn_plan_execute(
            self._h, _P(points.data_ptr()), _P(queries.data_ptr()) if queries is not None else None,
            _P(out.data_ptr()), ctypes.byref(st)))
        return out

    def resort(self):
        """The next execute sorts the queries again (keep_order plans)."""
        self.ctx._check(load_library().rtnn_plan_resort(self._h))

    def close(self):
        if getattr(self, "_h", None):
            load_library().rtnn_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def from_ref_layout(rows, point_order, query_order):
    """Rows of a reference-layout search (RTNN_FLAG_REF_LAYOUT) in the caller's layout:
    row query_order[j] = point_order[rows[j]], -1 kept (host numpy)."""
    rows = np.asarray(rows)
    po = np.asarray(point_order).astype(np.int64)
    qo = np.asarray(query_order).astype(np.int64)
    out = np.full_like(rows, -1)
    valid = rows >= 0
    out[qo] = np.where(valid, po[np.where(valid, rows, 0)], -1).astype(rows.dtype)
    return out


def _mode(mode):
    if mode in ("radius", RADIUS):
        return RADIUS
    if mode in ("knn", KNN):
        return KNN
    raise ValueError("mode must be 'radius' or 'knn'")


_default = {}


def _ctx(device):
    if device not in _default:
        _default[device] = Context(device)
    return _default[device]


def search(points, queries=None, mode="radius", radius=2.0, k=50, device=0, **kw):
    """Module-level convenience around Context(device).search()."""
    return _ctx(device).search(points, queries, mode=mode, radius=radius, k=k, **kw)


def search_batched(points, point_offsets, queries=None, query_offsets=None, device=0, **kw):
    return _ctx(device).search_batched(points, point_offsets, queries, query_offsets, **kw)
