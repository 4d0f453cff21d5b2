"""Python mirror of the C ABI in include/bpmax_gpu.h (ctypes over bpmax_b200/libbpmax_gpu.so).

There is no CPU fallback: if the library or a B200 is missing, every call raises.
Sequences are int arrays of bases 0..3 = A,C,G,U (4 = other), strand 2 in 5'->3' order exactly
as the reference's bpmax() receives it (it reverses strand 2 internally).
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbpmax_gpu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "bpmax_gpu.h")

STATUS = {0: "ok", 1: "invalid argument", 2: "out of memory", 3: "CUDA error", 4: "no usable CUDA device",
          5: "device wait timed out"}

_lib = None


class BpmaxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def header_functions() -> list[str]:
    """Names of the functions include/bpmax_gpu.h declares."""
    with open(HEADER) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(bpmax_gpu_\w+)\s*\(", text, flags=re.M)


def load_library():
    """Loads libbpmax_gpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `python -m bpmax_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    c_long, c_int, c_float = ctypes.c_long, ctypes.c_int, ctypes.c_float
    vp = ctypes.c_void_p
    L.bpmax_gpu_create.argtypes = [c_int, P(vp)]
    L.bpmax_gpu_destroy.argtypes = [vp]
    L.bpmax_gpu_destroy.restype = None
    L.bpmax_gpu_last_error.argtypes = [vp]
    L.bpmax_gpu_last_error.restype = ctypes.c_char_p
    L.bpmax_gpu_status_string.argtypes = [c_int]
    L.bpmax_gpu_status_string.restype = ctypes.c_char_p
    L.bpmax_gpu_set_weights.argtypes = [vp, vp]
    L.bpmax_gpu_fill.argtypes = [vp, vp, c_long, vp, c_long, c_long, vp, vp]
    L.bpmax_gpu_fill_compact.argtypes = [vp, vp, c_long, vp, c_long, vp, vp]
    L.bpmax_gpu_r0_only.argtypes = [vp, vp, c_long, vp, c_long, vp, vp]
    L.bpmax_gpu_score.argtypes = [vp, vp, c_long, vp, c_long, vp]
    for name in ("bpmax_gpu_score_batch", "bpmax_gpu_score_each"):
        getattr(L, name).argtypes = [vp, c_int, vp, vp, vp, vp, vp]
    L.bpmax_gpu_grad_batch.argtypes = [vp, c_int, vp, vp, vp, vp, vp, vp]
    L.bpmax_gpu_last_timing.argtypes = [vp, P(c_float), P(c_long)]
    L.bpmax_gpu_profile_kernels.argtypes = [vp, vp, vp, vp]
    L.bpmax_gpu_maxplus_peak.argtypes = [vp, P(ctypes.c_double)]
    L.bpmax_gpu_score_noalloc.argtypes = [vp, c_long, vp, c_long, vp, vp, vp]
    L.bpmax_gpu_read_cells.argtypes = [vp, c_int, c_long, c_long, c_long, c_long, vp]
    L.bpmax_gpu_shim_set_weights.argtypes = [vp]
    L.bpmax_gpu_set_tuning.argtypes = [vp, c_int, c_long]
    L.bpmax_gpu_get_tuning.argtypes = [vp, c_int, P(c_long)]
    L.bpmax_gpu_autotune.argtypes = [vp, c_int, vp, vp, vp, vp, c_int, vp, P(c_float)]
    for name in header_functions():
        if name not in ("bpmax_gpu_destroy", "bpmax_gpu_last_error", "bpmax_gpu_status_string"):
            getattr(L, name).restype = c_int
    _lib = L
    return L


def _seq(s) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(s, dtype=np.int32))
    if a.ndim != 1:
        raise ValueError("a sequence must be a 1-D array of base codes")
    return a


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def score_noalloc(seq1, seq2, w12, stream: int | None = None) -> float:
    """bpmax_gpu_score_noalloc: one pair's score with no memory allocated by the library (its
    scratch is a fixed 64 MiB device array, enough for N <= 64 and M <= 114 at N = 64).
    Raises BpmaxError on a non-zero status."""
    L = load_library()
    a, b = _seq(seq1), _seq(seq2)
    w = np.ascontiguousarray(np.asarray(w12, dtype=np.float32))
    out = np.zeros(1, dtype=np.float32)
    st = L.bpmax_gpu_score_noalloc(_ptr(a), len(a), _ptr(b), len(b), _ptr(w), _ptr(out),
                                   ctypes.c_void_p(stream) if stream else None)
    if st != 0:
        raise BpmaxError(st, "bpmax_gpu_score_noalloc failed")
    return float(out[0])


class Engine:
    """One CUDA device context (stream, device buffers, cached CUDA graphs)."""

    def __init__(self, device: int = 0):
        self._L = load_library()
        self._ctx = ctypes.c_void_p()
        st = self._L.bpmax_gpu_create(int(device), ctypes.byref(self._ctx))
        if st != 0:
            raise BpmaxError(st, f"bpmax_gpu_create(device={device}) failed")

    def close(self) -> None:
        if self._ctx:
            self._L.bpmax_gpu_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != 0:
            raise BpmaxError(st, self._L.bpmax_gpu_last_error(self._ctx).decode())

    def set_weights(self, w12) -> None:
        w = np.ascontiguousarray(np.asarray(w12, dtype=np.float32))
        if w.shape != (12,):
            raise ValueError("weights must have 12 entries")
        self._check(self._L.bpmax_gpu_set_weights(self._ctx, _ptr(w)))

    def score(self, seq1, seq2) -> float:
        a, b = _seq(seq1), _seq(seq2)
        out = np.zeros(1, dtype=np.float32)
        self._check(self._L.bpmax_gpu_score(self._ctx, _ptr(a), len(a), _ptr(b), len(b), _ptr(out)))
        return float(out[0])

    def fill_compact(self, seq1, seq2):
        """Returns (F[T(M), N, N] float32, score); i2 > j2 cells hold -FLT_MAX."""
        a, b = _seq(seq1), _seq(seq2)
        M, N = len(a), len(b)
        F = np.empty((M * (M + 1) // 2, N, N), dtype=np.float32)
        sc = np.zeros(1, dtype=np.float32)
        self._check(self._L.bpmax_gpu_fill_compact(self._ctx, _ptr(a), M, _ptr(b), N, _ptr(F), _ptr(sc)))
        return F, float(sc[0])

    def r0_only(self, seq1, seq2, want_table: bool = True):
        """bpmax_gpu_r0_only: the R0-only double max-plus microbenchmark of the reference's IPDPSW
        program (non-negative integer sequences). Returns (F[T(M), N, N] float32 or None, score)."""
        a = np.ascontiguousarray(seq1, dtype=np.int32)
        b = np.ascontiguousarray(seq2, dtype=np.int32)
        M, N = len(a), len(b)
        F = np.empty((M * (M + 1) // 2, N, N), dtype=np.float32) if want_table else None
        sc = np.zeros(1, dtype=np.float32)
        self._check(self._L.bpmax_gpu_r0_only(self._ctx, _ptr(a), M, _ptr(b), N, _ptr(F) if want_table else None,
                                              _ptr(sc)))
        return F, float(sc[0])

    @staticmethod
    def reference_size(M: int, N: int, n_tile: int) -> int:
        ns = (N + n_tile - 1) // n_tile
        return M * M * ns * ns * (n_tile + 1) * n_tile

    def fill(self, seq1, seq2, n_tile: int, out: np.ndarray | None = None):
        """Reference-layout fill; returns (F_lin, score). ``out`` (float32, reference size) may
        be a pinned buffer; cells the reference never writes are left as they are for i1>j1."""
        a, b = _seq(seq1), _seq(seq2)
        M, N = len(a), len(b)
        n = self.reference_size(M, N, n_tile)
        if out is None:
            out = np.full(n, np.nan, dtype=np.float32)
        if out.dtype != np.float32 or out.size != n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float32 buffer of the reference size")
        sc = np.zeros(1, dtype=np.float32)
        self._check(self._L.bpmax_gpu_fill(self._ctx, _ptr(a), M, _ptr(b), N, int(n_tile), _ptr(out), _ptr(sc)))
        return out, float(sc[0])

    def _batch_args(self, pairs):
        s1 = [_seq(p[0]) for p in pairs]
        s2 = [_seq(p[1]) for p in pairs]
        n = len(pairs)
        p1 = (ctypes.c_void_p * n)(*[x.ctypes.data for x in s1])
        p2 = (ctypes.c_void_p * n)(*[x.ctypes.data for x in s2])
        Ms = np.array([len(x) for x in s1], dtype=np.int64)
        Ns = np.array([len(x) for x in s2], dtype=np.int64)
        return n, p1, p2, Ms, Ns, (s1, s2)

    def score_batch(self, pairs) -> np.ndarray:
        n, p1, p2, Ms, Ns, keep = self._batch_args(pairs)
        out = np.zeros(n, dtype=np.float32)
        self._check(self._L.bpmax_gpu_score_batch(self._ctx, n, p1, _ptr(Ms), p2, _ptr(Ns), _ptr(out)))
        return out

    def score_each(self, pairs) -> np.ndarray:
        n, p1, p2, Ms, Ns, keep = self._batch_args(pairs)
        out = np.zeros(n, dtype=np.float32)
        self._check(self._L.bpmax_gpu_score_each(self._ctx, n, p1, _ptr(Ms), p2, _ptr(Ns), _ptr(out)))
        return out

    def grad_batch(self, pairs):
        n, p1, p2, Ms, Ns, keep = self._batch_args(pairs)
        scores = np.zeros(n, dtype=np.float32)
        grads = np.zeros((n, 12), dtype=np.float32)
        self._check(self._L.bpmax_gpu_grad_batch(self._ctx, n, p1, _ptr(Ms), p2, _ptr(Ns), _ptr(scores), _ptr(grads)))
        return scores, grads

    def read_cells(self, pair: int, i1_lo: int, i1_hi: int, j1_lo: int, j1_hi: int, N: int) -> np.ndarray:
        """bpmax_gpu_read_cells: inner tables of outer cells [i1_lo, i1_hi) x [j1_lo, j1_hi) of pair
        ``pair`` of the last fill, as float32 [i1, j1, N, N] (-FLT_MAX where i2 > j2, NaN where
        i1 > j1). N is that pair's strand-2 length."""
        out = np.empty((i1_hi - i1_lo, j1_hi - j1_lo, N, N), dtype=np.float32)
        self._check(self._L.bpmax_gpu_read_cells(self._ctx, int(pair), int(i1_lo), int(i1_hi), int(j1_lo), int(j1_hi),
                                                 _ptr(out)))
        return out

    TUNING_KEYS = {"r0_pairs_per_job": 0, "r0_merge_items": 1, "class_streams": 2, "wait_limit_us": 3,
                   "inject_wait_timeout": 4, "wide_stages": 5, "r0_variant": 6, "class_share": 7,
                   "persistent": 8}
    #: the tunables bpmax_gpu_autotune chooses, in the order it reports them
    AUTOTUNED = ("r0_pairs_per_job", "r0_merge_items", "class_streams", "r0_variant", "wide_stages", "class_share",
                 "persistent")

    def set_tuning(self, key: str, value: int) -> None:
        self._check(self._L.bpmax_gpu_set_tuning(self._ctx, self.TUNING_KEYS[key], int(value)))

    def get_tuning(self, key: str) -> int:
        v = ctypes.c_long()
        self._check(self._L.bpmax_gpu_get_tuning(self._ctx, self.TUNING_KEYS[key], ctypes.byref(v)))
        return int(v.value)

    def autotune(self, pairs, trials: int = 1):
        """bpmax_gpu_autotune: times the candidate schedules on these pairs and keeps the fastest
        for their shapes. Returns ({tunable: value}, fill ms)."""
        n, p1, p2, Ms, Ns, keep = self._batch_args(pairs)
        best = np.zeros(len(self.AUTOTUNED), dtype=np.int64)
        ms = ctypes.c_float()
        self._check(self._L.bpmax_gpu_autotune(self._ctx, n, p1, _ptr(Ms), p2, _ptr(Ns), int(trials), _ptr(best),
                                               ctypes.byref(ms)))
        return {k: int(best[i]) for i, k in enumerate(self.AUTOTUNED)}, float(ms.value)

    def profile_kernels(self):
        """Per kernel kind (strand, r0, finalize): (ms, launches, terms) of an eager re-run of
        the last fill with CUDA events around every launch."""
        ms = np.zeros(3, dtype=np.float32)
        n = np.zeros(3, dtype=np.int64)
        t = np.zeros(3, dtype=np.float64)
        self._check(self._L.bpmax_gpu_profile_kernels(self._ctx, _ptr(ms), _ptr(n), _ptr(t)))
        return {k: (float(ms[i]), int(n[i]), float(t[i])) for i, k in enumerate(("strand", "r0", "finalize"))}

    def maxplus_peak(self) -> float:
        v = ctypes.c_double()
        self._check(self._L.bpmax_gpu_maxplus_peak(self._ctx, ctypes.byref(v)))
        return float(v.value)

    def last_timing(self):
        ms = ctypes.c_float()
        n = ctypes.c_long()
        self._check(self._L.bpmax_gpu_last_timing(self._ctx, ctypes.byref(ms), ctypes.byref(n)))
        return float(ms.value), int(n.value)
