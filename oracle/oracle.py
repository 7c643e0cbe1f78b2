"""ctypes access to the C restatement (liboracle.so) and to the reference's own
functions (oracle/_ref/libfsmeld_ref.so, built from the reference sources with
the project's FFTW-API shim).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libfsmeld_ref.so")
BIN_REF = os.path.join(HERE, "_ref", "fsmeld_ref")
# The reference source tree: $FSMELD_REFERENCE_TREE, else the folder
# `reference` beside the repository.  Only build() reads it.
REFERENCE_TREE = os.environ.get("FSMELD_REFERENCE_TREE") or os.path.normpath(
    os.path.join(HERE, "..", "..", "reference"))

METRICS = {"dtw": 1, "edr": 2, "erp": 3, "lcss": 4, "msm": 5}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_longlong)
_u8 = C.POINTER(C.c_uint8)


class Counters(C.Structure):
    _fields_ = [
        ("valid", C.c_longlong), ("invalid", C.c_longlong), ("after_lb", C.c_longlong),
        ("after_glb", C.c_longlong), ("exact_evals", C.c_longlong), ("matches", C.c_longlong),
        ("threshold", C.c_double), ("m_k", C.c_int), ("segments", C.c_longlong),
        ("tail", C.c_longlong),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def build(reference: bool = True) -> None:
    """Compile liboracle.so (and, when the reference tree exists, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)
    if reference and os.path.isdir(os.path.join(REFERENCE_TREE, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "reference", f"REF={REFERENCE_TREE}"], check=True)


def have_reference() -> bool:
    return os.path.exists(LIB_REF) and os.path.exists(BIN_REF)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return a.ctypes.data_as(_dp)


class _Lib:
    def __init__(self, path, prefix):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        self.p = prefix

    def fn(self, name, restype, *argtypes):
        f = getattr(self.lib, self.p + name)
        f.restype = restype
        f.argtypes = list(argtypes)
        return f


class Oracle:
    """Thin numpy front end shared by the restatement and the reference wrappers."""

    def __init__(self, which: str = "oracle"):
        if which == "oracle":
            if not os.path.exists(LIB_ORACLE):
                build(reference=False)
            self.L = _Lib(LIB_ORACLE, "orc_")
        else:
            self.L = _Lib(LIB_REF, "ref_")
        self.which = which
        L = self.L
        self._mvmean = L.fn("mvmean", None, _dp, C.c_int, C.c_int, _dp, _dp)
        self._mask = L.fn("invalid_mask", None, _dp, _dp, C.c_int, C.c_int, _u8)
        self._mmw = L.fn("min_max_window", None, _dp, C.c_int, C.c_int, _dp, _dp)
        self._lemire = L.fn("lemire", None, _dp, C.c_int, C.c_int, _dp, _dp)
        self._norm = L.fn("normalized", None, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp)
        self._q2h = L.fn("q_to_h", None, C.c_int, C.c_int, _dp, C.c_int, C.c_double, C.c_double, _dp)
        self._s2g = L.fn("s_to_g", None, C.c_int, _dp, C.c_int, C.c_double, _dp)
        self._lbx = L.fn("lbip_exceeds", C.c_int, C.c_double, C.c_double, C.c_int)
        self._glb = L.fn("glb", C.c_double, C.c_int, _dp, _dp, C.c_int, C.c_double, _dp, _dp,
                         C.c_int, C.c_double)
        self._dist = L.fn("distance", C.c_double, C.c_int, _dp, _dp, C.c_int, C.c_int, C.c_double)
        if which == "oracle":
            self._findt = L.fn("find_t", C.c_double, C.c_int, C.c_int, _dp, C.c_int, _dp, _dp,
                               C.c_int, C.c_double)
            self._sip = L.fn("sip", None, C.c_int, C.c_int, _dp, _dp, _dp)
            self._search = L.fn("search", C.c_longlong, _dp, C.c_longlong, _dp, C.c_int, C.c_double,
                                C.c_int, C.c_int, C.c_double, C.c_longlong, C.c_longlong, _ip,
                                C.c_longlong, C.POINTER(Counters), _ip)
            self._exact = L.fn("exact", C.c_longlong, _dp, C.c_longlong, _dp, C.c_int, C.c_double,
                               C.c_int, C.c_int, C.c_double, C.c_longlong, C.c_longlong, _ip, _dp,
                               C.c_longlong, C.POINTER(Counters))
            self._cutoff = L.fn("cutoff", C.c_longlong, _dp, C.c_longlong, _dp, C.c_int, C.c_int,
                                C.c_int, C.c_int, C.c_double, C.c_longlong, C.c_longlong, _ip, _dp,
                                C.POINTER(Counters))
            self._macro = L.fn("macro_length", C.c_int, C.c_int, C.c_longlong)
            self._normq = L.fn("normalize_query", None, _dp, C.c_int, _dp)
            self._setnorm = L.fn("set_normalization", None, C.c_int)
        else:
            self._findt = L.fn("find_t", C.c_double, C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int,
                               C.c_double)
            self._sip = L.fn("sip", None, C.c_int, C.c_int, _dp, _dp, _dp)

    # -- per-function ---------------------------------------------------
    def mvmean(self, a, m):
        a = _d(a)
        k = len(a) - m + 1
        mu, si = np.empty(k), np.empty(k)
        self._mvmean(_ptr(a), len(a), m, _ptr(mu), _ptr(si))
        return mu, si

    def invalid_mask(self, t, si, m):
        t, si = _d(t), _d(si)
        out = np.zeros(len(t) - m + 1, dtype=np.uint8)
        self._mask(_ptr(t), _ptr(si), len(t), m, out.ctypes.data_as(_u8))
        return out

    def min_max_window(self, a, n, m):
        a = _d(a)
        mn, mx = np.empty(n), np.empty(n)
        self._mmw(_ptr(a), n, m, _ptr(mn), _ptr(mx))
        return mn, mx

    def lemire(self, a, r):
        a = _d(a)
        lo, up = np.empty(len(a)), np.empty(len(a))
        self._lemire(_ptr(a), len(a), r, _ptr(lo), _ptr(up))
        return lo, up

    def normalized(self, U, L, mumax, mumin, simax, simin):
        U, L = _d(U), _d(L)
        Un, Ln = np.empty(len(U)), np.empty(len(U))
        self._norm(_ptr(U), _ptr(L), _ptr(Un), _ptr(Ln), len(U), _ptr(_d(mumax)), _ptr(_d(mumin)),
                   _ptr(_d(simax)), _ptr(_d(simin)))
        return Un, Ln

    def find_t(self, upper, metric, env, q, m, arg):
        env, q = _d(env), _d(q)
        mid = METRICS[metric] if isinstance(metric, str) else metric
        if self.which == "oracle":
            return self._findt(int(upper), mid, _ptr(env), len(env), _ptr(q), None, m, arg)
        return self._findt(int(upper), mid, _ptr(env), len(env), _ptr(q), m, arg)

    def q_to_h(self, upper, metric, q, t, arg):
        q = _d(q)
        h = np.zeros(len(q))
        mid = METRICS[metric] if isinstance(metric, str) else metric
        self._q2h(int(upper), mid, _ptr(q), len(q), t, arg, _ptr(h))
        return h

    def s_to_g(self, upper, env, t):
        env = _d(env)
        g = np.zeros(len(env))
        self._s2g(int(upper), _ptr(env), len(env), t, _ptr(g))
        return g

    def sip(self, n, m, h, g):
        z = np.zeros(n)
        self._sip(n, m, _ptr(_d(h)), _ptr(_d(g)), _ptr(z))
        return z

    def lbip_exceeds(self, bound, cutoff, metric):
        mid = METRICS[metric] if isinstance(metric, str) else metric
        return bool(self._lbx(bound, cutoff, mid))

    def glb(self, metric, Q, T, arg, LQ, UQ, w, bsf):
        mid = METRICS[metric] if isinstance(metric, str) else metric
        Q, T = _d(Q), _d(T)
        return self._glb(mid, _ptr(Q), _ptr(T), len(Q), arg, _ptr(_d(LQ)), _ptr(_d(UQ)), w, bsf)

    def distance(self, metric, q, t, w, arg):
        mid = METRICS[metric] if isinstance(metric, str) else metric
        q, t = _d(q), _d(t)
        return self._dist(mid, _ptr(q), _ptr(t), len(q), w, arg)

    # -- drivers (restatement only) ------------------------------------
    def macro_length(self, m, n):
        return self._macro(m, n)

    def normalize_query(self, q):
        q = _d(q)
        out = np.empty(len(q))
        self._normq(_ptr(q), len(q), _ptr(out))
        return out

    def set_normalization(self, mode: str) -> None:
        """'zscore' (default) or 'raw' for the restatement's drivers."""
        if mode not in ("zscore", "raw"):
            raise ValueError(mode)
        self._setnorm(1 if mode == "raw" else 0)

    def search(self, target, query, m, cutoff, metric, w, arg, excl=(-1, -1), seg_counts=False):
        target, query = _d(target), _d(query)
        cnt = Counters()
        cap = 1 << 16
        while True:
            idx = np.zeros(cap, dtype=np.int64)
            segs = None
            if seg_counts:
                mk = self.macro_length(m, len(target))
                nseg = (len(target) - m + 1) // (mk - m + 1)
                segs = np.zeros(3 * max(nseg, 1), dtype=np.int64)
            r = self._search(_ptr(target), len(target), _ptr(query), m, cutoff, METRICS[metric], w,
                             arg, excl[0], excl[1], idx.ctypes.data_as(_ip), cap, C.byref(cnt),
                             segs.ctypes.data_as(_ip) if segs is not None else None)
            if r < 0:
                raise ValueError(f"orc_search failed ({r})")
            if r <= cap:
                out = (idx[:r].copy(), cnt.as_dict())
                return out + ((segs.reshape(-1, 3),) if seg_counts else ())
            cap = int(r)

    def exact(self, target, query, m, cutoff, metric, w, arg, excl=(-1, -1)):
        target, query = _d(target), _d(query)
        cnt = Counters()
        cap = 1 << 16
        while True:
            idx = np.zeros(cap, dtype=np.int64)
            dist = np.zeros(cap)
            r = self._exact(_ptr(target), len(target), _ptr(query), m, cutoff, METRICS[metric], w,
                            arg, excl[0], excl[1], idx.ctypes.data_as(_ip), _ptr(dist), cap,
                            C.byref(cnt))
            if r < 0:
                raise ValueError(f"orc_exact failed ({r})")
            if r <= cap:
                return idx[:r].copy(), dist[:r].copy(), cnt.as_dict()
            cap = int(r)

    def cutoff(self, target, query, m, k, metric, w, arg, excl=(-1, -1)):
        target, query = _d(target), _d(query)
        cnt = Counters()
        idx = np.zeros(k, dtype=np.int64)
        dist = np.zeros(k)
        r = self._cutoff(_ptr(target), len(target), _ptr(query), m, k, METRICS[metric], w, arg,
                         excl[0], excl[1], idx.ctypes.data_as(_ip), _ptr(dist), C.byref(cnt))
        if r == -2:
            raise ValueError("Fewer valid, non-excluded candidates than requested k.")
        if r < 0:
            raise ValueError(f"orc_cutoff failed ({r})")
        return idx, dist, cnt.as_dict()


def run_reference_cli(args, cwd=None, env=None, timeout=None):
    """Run the reference CLI built from its own sources; returns (rc, stdout, stderr)."""
    p = subprocess.run([BIN_REF] + [str(a) for a in args], cwd=cwd, env=env, capture_output=True,
                       text=True, timeout=timeout)
    return p.returncode, p.stdout, p.stderr
