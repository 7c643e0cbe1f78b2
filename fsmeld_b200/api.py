"""Python binding of the C ABI in include/fsmeld_cuda.h (ctypes).

Mirrors the reference's entry points (include/funcs.h:64-72) by name and
argument meaning:

    FSMELD(target_path, query_path, m, cutoff, tag, w, arg, exclude_start=-1, exclude_end=-1)
    FSMELD_find_threshold(target_path, query_path, m, threshold, tag, w, arg, top_k, ...)
    FSMELD_exact(target_path, query_path, m, cutoff, tag, w, arg, top_k=0, ...)

which print the reference's output, and an in-memory `Engine` for callers
that hold the target and query as arrays.  Errors raise `FsmeldError` with
the library's message, as the reference raises std::runtime_error /
std::invalid_argument.  There is no CPU fallback: importing without the
built library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libfsmeld_cuda.so")
CLI_PATH = os.path.join(_PKG, "bin", "fsmeld")

METRICS = {"dtw": 1, "edr": 2, "erp": 3, "lcss": 4, "msm": 5}
OK, E_ARG, E_CUDA, E_NOMEM, E_SHORT, E_FEWER_K, E_UNSUPPORTED, E_IO = 0, -1, -2, -3, -4, -5, -6, -7


class FsmeldError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class Counters(C.Structure):
    _fields_ = [("valid", C.c_int64), ("invalid", C.c_int64), ("after_lb", C.c_int64),
                ("after_glb", C.c_int64), ("exact_evals", C.c_int64), ("matches", C.c_int64),
                ("threshold", C.c_double), ("m_k", C.c_int32), ("reserved", C.c_int32),
                ("segments", C.c_int64), ("tail", C.c_int64), ("device_ms", C.c_double),
                ("dp_cells", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class Query(C.Structure):
    _fields_ = [("query", C.POINTER(C.c_double)), ("m", C.c_int32), ("metric", C.c_int32),
                ("w", C.c_int32), ("k", C.c_int32), ("arg", C.c_double), ("cutoff", C.c_double),
                ("exclude_begin", C.c_int64), ("exclude_end", C.c_int64)]


class Result(C.Structure):
    _fields_ = [("idx", C.POINTER(C.c_int64)), ("dist", C.POINTER(C.c_double)),
                ("capacity", C.c_int64), ("count", C.c_int64), ("status", C.c_int32),
                ("reserved", C.c_int32), ("counters", Counters),
                ("seg_counts", C.POINTER(C.c_int64))]


_lib = None


def lib():
    """Load the CUDA library (built in-tree by fsmeld_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FsmeldError(E_CUDA, f"CUDA library not built: {LIB_PATH} (run python -m fsmeld_b200.build)")
        L = C.CDLL(LIB_PATH)
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int64)
        ctxp = C.c_void_p
        sig = {
            "fsmeld_open": (C.c_int, [C.c_int, dp, C.c_int64, C.POINTER(ctxp)]),
            "fsmeld_open_file": (C.c_int, [C.c_int, C.c_char_p, C.POINTER(ctxp)]),
            "fsmeld_load": (C.c_int, [ctxp, dp, C.c_int64]),
            "fsmeld_open_device": (C.c_int, [C.c_int, C.c_void_p, C.c_int64, C.POINTER(ctxp)]),
            "fsmeld_close": (C.c_int, [ctxp]),
            "fsmeld_target_length": (C.c_int64, [ctxp]),
            "fsmeld_last_error": (C.c_char_p, [ctxp]),
            "fsmeld_strerror": (C.c_char_p, [C.c_int]),
            "fsmeld_set_workspace_limit": (C.c_int, [ctxp, C.c_int64]),
            "fsmeld_workspace_bytes": (C.c_int64, [ctxp]),
            "fsmeld_target_device": (C.c_void_p, [ctxp]),
            "fsmeld_release_workspace": (C.c_int, [ctxp]),
            "fsmeld_set_concurrency": (C.c_int, [ctxp, C.c_int]),
            "fsmeld_set_normalization": (C.c_int, [ctxp, C.c_int]),
            "fsmeld_set_lb_form": (C.c_int, [ctxp, C.c_int]),
            "fsmeld_set_tuning": (C.c_int, [ctxp, C.c_char_p]),
            "fsmeld_normalization": (C.c_int, [ctxp]),
            "fsmeld_kernel_launches": (C.c_int64, [ctxp]),
            "fsmeld_set_profiling": (C.c_int, [ctxp, C.c_int]),
            "fsmeld_stage_times": (C.c_int, [ctxp, dp, ip, C.c_int]),
            "fsmeld_stage_name": (C.c_char_p, [C.c_int]),
            "fsmeld_last_call_ms": (C.c_double, [ctxp]),
            "fsmeld_search": (C.c_int, [ctxp, dp, C.c_int, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int64,
                                        C.c_int64, ip, C.c_int64, ip, C.POINTER(Counters), ip]),
            "fsmeld_cutoff": (C.c_int, [ctxp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int64,
                                        C.c_int64, ip, dp, C.POINTER(Counters)]),
            "fsmeld_exact": (C.c_int, [ctxp, dp, C.c_int, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int64,
                                       C.c_int64, ip, dp, C.c_int64, ip, C.POINTER(Counters)]),
            "fsmeld_batch": (C.c_int, [ctxp, C.c_int, C.POINTER(Query), C.c_int, C.POINTER(Result)]),
            "fsmeld_inspect": (C.c_int64, [ctxp, dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, dp,
                                           C.c_int64]),
            "fsmeld_exact_noalloc": (C.c_int, [C.c_int, C.c_void_p, C.c_int64, dp, C.c_int, C.c_int, C.c_int,
                                               C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_int64, ip,
                                               C.c_void_p]),
            "fsmeld_search_file": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_double, C.c_char_p, C.c_int,
                                             C.c_double, C.c_int64, C.c_int64]),
            "fsmeld_cutoff_file": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_char_p, C.c_int,
                                             C.c_double, C.c_int64, C.c_int64]),
            "fsmeld_exact_file": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_double, C.c_char_p, C.c_int,
                                            C.c_double, C.c_int64, C.c_int64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols(header=None):
    """Names of the C ABI entry points declared in include/fsmeld_cuda.h."""
    import re
    header = header or os.path.join(os.path.dirname(_PKG), "include", "fsmeld_cuda.h")
    text = re.sub(r"/\*.*?\*/", "", open(header).read(), flags=re.S)
    return sorted(set(re.findall(r"\b(fsmeld_[a-z_0-9]+)\s*\(", text)))


def _check(status, ctx=None):
    if status != OK:
        msg = lib().fsmeld_last_error(ctx).decode(errors="replace") or lib().fsmeld_strerror(status).decode()
        raise FsmeldError(status, msg)


def _metric(tag):
    if isinstance(tag, int):
        return tag
    if tag not in METRICS:
        raise FsmeldError(E_ARG, f"Unsupported metric: {tag}")
    return METRICS[tag]


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


TUNE_TABLE = os.path.join(_PKG, "tune_table.txt")


class Engine:
    """A target series resident on one GPU, queried through the C ABI.

    tuning: the tuning table's text (see fsmeld_set_tuning); by default the
    measured table fsmeld_b200/tune_table.txt when present; "" for none."""

    def __init__(self, target=None, *, path=None, device=0, device_ptr=None, n=None, tuning=None):
        self._ctx = C.c_void_p()
        L = lib()
        if path is not None:
            _check(L.fsmeld_open_file(device, os.fsencode(path), C.byref(self._ctx)))
        elif device_ptr is not None:
            _check(L.fsmeld_open_device(device, C.c_void_p(device_ptr), int(n), C.byref(self._ctx)))
        else:
            t = np.ascontiguousarray(target, dtype=np.float64)
            _check(L.fsmeld_open(device, _dptr(t), len(t), C.byref(self._ctx)))
        self.n = L.fsmeld_target_length(self._ctx)
        if tuning is None and os.path.exists(TUNE_TABLE):
            with open(TUNE_TABLE) as f:
                tuning = f.read()
        if tuning:
            self.set_tuning(tuning)

    def set_tuning(self, table_text):
        """Rules for the automatic kernel choices (fsmeld_set_tuning)."""
        _check(lib().fsmeld_set_tuning(self._ctx, table_text.encode()), self._ctx)

    def load(self, target):
        """Replace the target (host array, e.g. pinned memory) keeping the workspace."""
        t = np.ascontiguousarray(target, dtype=np.float64)
        _check(lib().fsmeld_load(self._ctx, _dptr(t), len(t)), self._ctx)
        self.n = len(t)

    def close(self):
        if self._ctx:
            lib().fsmeld_close(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self):
        return lib().fsmeld_kernel_launches(self._ctx)

    @property
    def last_call_ms(self):
        """Device time (CUDA events on the engine's stream) of the last query call."""
        return lib().fsmeld_last_call_ms(self._ctx)

    def set_profiling(self, on=True):
        _check(lib().fsmeld_set_profiling(self._ctx, int(on)), self._ctx)

    def stage_times(self):
        ms = np.zeros(16)
        n = np.zeros(16, dtype=np.int64)
        k = lib().fsmeld_stage_times(self._ctx, _dptr(ms), _iptr(n), 16)
        return {lib().fsmeld_stage_name(i).decode(): (float(ms[i]), int(n[i])) for i in range(k)}

    def set_workspace_limit(self, nbytes):
        _check(lib().fsmeld_set_workspace_limit(self._ctx, int(nbytes)), self._ctx)

    def target_device_ptr(self):
        """Device address of the resident target (for engines that borrow it)."""
        return int(lib().fsmeld_target_device(self._ctx))

    def workspace_bytes(self):
        """Device workspace bytes this engine holds now (its batch workers included)."""
        return int(lib().fsmeld_workspace_bytes(self._ctx))

    def release_workspace(self):
        """Free the engine's workspace; the target stays resident."""
        _check(lib().fsmeld_release_workspace(self._ctx), self._ctx)

    def set_concurrency(self, queries):
        """Queries of one (m, w) group of a batch run concurrently on this many streams."""
        _check(lib().fsmeld_set_concurrency(self._ctx, int(queries)), self._ctx)

    def set_normalization(self, mode):
        """'zscore' (default, the reference command line's mode) or 'raw'
        (the reference's NormalizationMode::Raw, include/funcs.h:20-28)."""
        if mode not in ("zscore", "raw"):
            raise FsmeldError(E_ARG, f"unknown normalization mode: {mode}")
        _check(lib().fsmeld_set_normalization(self._ctx, 1 if mode == "raw" else 0), self._ctx)

    def set_lb_form(self, form):
        """LB_IP form of batched searches of equal (m, w) and metric: 'auto',
        'fft' (per query, the reference's) or 'gemm' (tensor-core product)."""
        ids = {"auto": 0, "fft": 1, "gemm": 2}
        if form not in ids:
            raise FsmeldError(E_ARG, f"unknown LB_IP form: {form}")
        _check(lib().fsmeld_set_lb_form(self._ctx, ids[form]), self._ctx)

    @property
    def normalization(self):
        return "raw" if lib().fsmeld_normalization(self._ctx) == 1 else "zscore"

    def search(self, query, m, cutoff, metric, w, arg=0.0, exclude=(-1, -1), seg_counts=False):
        q = np.ascontiguousarray(query[:m], dtype=np.float64)
        cap = 1 << 16
        cnt = Counters()
        nseg = max(1, (self.n - m + 1) // _kml(m, self.n))
        segs = np.zeros(3 * nseg, dtype=np.int64) if seg_counts else None
        while True:
            idx = np.zeros(cap, dtype=np.int64)
            count = C.c_int64(0)
            st = lib().fsmeld_search(self._ctx, _dptr(q), m, float(cutoff), _metric(metric), w, float(arg),
                                     exclude[0], exclude[1], _iptr(idx), cap, C.byref(count), C.byref(cnt),
                                     _iptr(segs) if segs is not None else None)
            _check(st, self._ctx)
            if count.value <= cap:
                res = (idx[:count.value].copy(), cnt.as_dict())
                return res + ((segs.reshape(-1, 3),) if seg_counts else ())
            cap = count.value

    def cutoff(self, query, m, k, metric, w, arg=0.0, exclude=(-1, -1)):
        q = np.ascontiguousarray(query[:m], dtype=np.float64)
        idx = np.zeros(k, dtype=np.int64)
        dist = np.zeros(k)
        cnt = Counters()
        _check(lib().fsmeld_cutoff(self._ctx, _dptr(q), m, k, _metric(metric), w, float(arg), exclude[0],
                                   exclude[1], _iptr(idx), _dptr(dist), C.byref(cnt)), self._ctx)
        return idx, dist, cnt.as_dict()

    def exact(self, query, m, cutoff, metric, w, arg=0.0, exclude=(-1, -1)):
        q = np.ascontiguousarray(query[:m], dtype=np.float64)
        cap = 1 << 16
        cnt = Counters()
        while True:
            idx = np.zeros(cap, dtype=np.int64)
            dist = np.zeros(cap)
            count = C.c_int64(0)
            _check(lib().fsmeld_exact(self._ctx, _dptr(q), m, float(cutoff), _metric(metric), w, float(arg),
                                      exclude[0], exclude[1], _iptr(idx), _dptr(dist), cap, C.byref(count),
                                      C.byref(cnt)), self._ctx)
            if count.value <= cap:
                return idx[:count.value].copy(), dist[:count.value].copy(), cnt.as_dict()
            cap = count.value

    def batch(self, mode, queries, capacity=1 << 14):
        """queries: list of dicts with query, m, metric, w, arg, cutoff or k, exclude."""
        mode_id = {"search": 0, "cutoff": 1, "exact": 2}[mode]
        n = len(queries)
        qs = (Query * n)()
        rs = (Result * n)()
        keep = []
        for i, d in enumerate(queries):
            q = np.ascontiguousarray(d["query"][:d["m"]], dtype=np.float64)
            cap = d.get("k", capacity) if mode == "cutoff" else capacity
            idx = np.zeros(cap, dtype=np.int64)
            dist = np.zeros(cap)
            keep += [q, idx, dist]
            ex = d.get("exclude", (-1, -1))
            qs[i] = Query(_dptr(q), d["m"], _metric(d["metric"]), d["w"], d.get("k", 0), float(d.get("arg", 0.0)),
                          float(d.get("cutoff", 0.0)), ex[0], ex[1])
            rs[i].idx = _iptr(idx)
            rs[i].dist = _dptr(dist)
            rs[i].capacity = cap
        st = lib().fsmeld_batch(self._ctx, mode_id, qs, n, rs)
        out = []
        for i in range(n):
            r = rs[i]
            idx, dist = keep[3 * i + 1], keep[3 * i + 2]
            c = min(r.count, r.capacity)
            out.append({"status": r.status, "idx": idx[:c].copy(), "dist": dist[:c].copy(), "count": r.count,
                        "counters": r.counters.as_dict()})
        if st not in (OK,) and all(o["status"] == OK for o in out):
            _check(st, self._ctx)
        return out

    def inspect(self, query, m, metric, w, arg, what):
        q = np.ascontiguousarray(query[:m], dtype=np.float64)
        n = lib().fsmeld_inspect(self._ctx, _dptr(q), m, _metric(metric), w, float(arg), what, None, 0)
        if n < 0:
            _check(int(n), self._ctx)
        out = np.zeros(n)
        lib().fsmeld_inspect(self._ctx, _dptr(q), m, _metric(metric), w, float(arg), what, _dptr(out), n)
        return out


def _kml(m, n):
    sel = 1
    while sel < 8 * m:
        sel *= 2
    sel = min(sel, n)
    return sel - m + 1


def exact_noalloc(device_target_ptr, n, query, m, cutoff, metric, w, arg, out_idx_ptr, out_dist_ptr, capacity,
                  device=0, stream=None):
    """fsmeld_exact_noalloc: device pointers in and out, no device allocation."""
    q = np.ascontiguousarray(query[:m], dtype=np.float64)
    count = C.c_int64(0)
    st = lib().fsmeld_exact_noalloc(device, C.c_void_p(device_target_ptr), int(n), _dptr(q), m, _metric(metric), w,
                                    float(arg), float(cutoff), C.c_void_p(out_idx_ptr), C.c_void_p(out_dist_ptr),
                                    int(capacity), C.byref(count), C.c_void_p(stream) if stream else None)
    _check(st)
    return count.value


# ---- reference-named entry points (print the reference's output) -------------

def FSMELD(bi_t, bi_q, m, threshold, tag, w, arg, exclude_start=-1, exclude_end=-1):
    _check(lib().fsmeld_search_file(os.fsencode(bi_t), os.fsencode(bi_q), m, float(threshold), tag.encode(), w,
                                    float(arg), exclude_start, exclude_end))


def FSMELD_find_threshold(bi_t, bi_q, m, threshold, tag, w, arg, top_k, exclude_start=-1, exclude_end=-1):
    del threshold  # the reference passes DBL_MAX here (src/main.cpp:95)
    _check(lib().fsmeld_cutoff_file(os.fsencode(bi_t), os.fsencode(bi_q), m, int(top_k), tag.encode(), w,
                                    float(arg), exclude_start, exclude_end))


def FSMELD_exact(bi_t, bi_q, m, threshold, tag, w, arg, top_k=0, exclude_start=-1, exclude_end=-1):
    if top_k:
        raise FsmeldError(E_UNSUPPORTED, "exact top-k derivation is not exposed by the command line")
    _check(lib().fsmeld_exact_file(os.fsencode(bi_t), os.fsencode(bi_q), m, float(threshold), tag.encode(), w,
                                   float(arg), exclude_start, exclude_end))
