"""ctypes bindings for the checkers (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module.
It wraps

* ``liboracle.so``: the CPU restatement of the reference recurrence
  (TPDS/source/release/MPT_RT_V3/bpmax_complete_otf_ftable/src/bpmax_verify.c:533-721), and
* ``_ref/libbpmax_ref.so``: the reference's own optimised fill ``bpmax()``
  (V3/bpmax.c:129) and memoised ``bpmax_verify()`` (V3/bpmax_verify.c:156), compiled from
  the reference sources by ``oracle/Makefile``.

The compact table layout used here is: T(M)=M(M+1)/2 outer cells in row-major upper-triangle
order, each an N x N float32 inner table indexed [i2, j2] over the reversed strand 2.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libbpmax_ref.so")
_REF_R0_CHECK = os.path.join(HERE, "_ref", "ospsqmax_check")  # the reference's R0-only program, printing F
_REF_R0_TIME = os.path.join(HERE, "_ref", "ospsqmax_time")    # the same, random sequences, timing only

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_L = ctypes.c_long

_lib = None
_ref = None


_REF_CLI = os.path.join(HERE, "_ref", "bpmax_gpu_cli")              # the reference's CLI wrapper on the GPU library
_REF_CLI_CHECK = os.path.join(HERE, "_ref", "bpmax_gpu_cli_check")  # the same, -DCHECKING -DNO_PROMPT


def reference_root() -> str | None:
    """The reference project's root: $REFERENCE_ROOT, else its mount in the build container."""
    root = os.environ.get("REFERENCE_ROOT") or "/root/reference"
    return root if os.path.isdir(root) else None


def build(targets=()) -> None:
    """Compile the checkers (make -C oracle). The parts built from the reference's sources only
    build where those sources exist."""
    cmd = ["make", "-s", "-C", HERE]
    root = reference_root()
    if root:
        cmd.append(f"REFERENCE_ROOT={root}")
    subprocess.run(cmd + list(targets), check=True)


def cli_available() -> bool:
    return os.path.exists(_REF_CLI) and os.path.exists(_REF_CLI_CHECK)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_ORACLE):
            build()
        L = ctypes.CDLL(_ORACLE)
        L.oracle_fill.argtypes = [_L, _L, _i32p, _i32p, _f32p, _f32p, _f32p, _f32p]
        L.oracle_fill.restype = ctypes.c_int
        L.oracle_traceback.argtypes = [_L, _L, _i32p, _i32p, _f32p, _f32p, _f32p, _f32p, _f64p]
        L.oracle_traceback.restype = ctypes.c_long
        L.oracle_to_reference_layout.argtypes = [_L, _L, _L, _f32p, _f32p]
        L.oracle_to_reference_layout.restype = None
        L.oracle_reference_size.argtypes = [_L, _L, _L]
        L.oracle_reference_size.restype = ctypes.c_long
        L.oracle_single_strand.argtypes = [_L, _i32p, _f32p, _f32p]
        L.oracle_single_strand.restype = None
        L.oracle_r0only.argtypes = [_L, _L, _i32p, _i32p, _f32p]
        L.oracle_r0only.restype = ctypes.c_int
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(_REF):
            raise FileNotFoundError(f"{_REF} not built (the reference sources are needed to build it)")
        L = ctypes.CDLL(_REF)
        L.ref_bpmax_fill.argtypes = [_L, _L, _L, _L, _L, ctypes.c_int, _i32p, _i32p, _f32p, _f32p, ctypes.c_int]
        L.ref_bpmax_fill.restype = ctypes.c_int
        L.ref_bpmax_fill_timed.argtypes = [_L, _L, _L, _L, _L, ctypes.c_int, _i32p, _i32p, _f32p, _f32p, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_double)]
        L.ref_bpmax_fill_timed.restype = ctypes.c_int
        L.ref_bpmax_verify.argtypes = [_L, _L, _i32p, _i32p, _f32p, _f32p]
        L.ref_bpmax_verify.restype = ctypes.c_int
        _ref = L
    return _ref


def _as(seq) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(seq, dtype=np.int32))


def _w(w12) -> np.ndarray:
    w = np.ascontiguousarray(np.asarray(w12, dtype=np.float32))
    assert w.shape == (12,)
    return w


def fill(seq1, seq2, w12):
    """Oracle fill. Returns (F[T(M), N, N], S1[M, M], S2[N, N])."""
    s1, s2, w = _as(seq1), _as(seq2), _w(w12)
    M, N = len(s1), len(s2)
    F = np.empty((M * (M + 1) // 2, N, N), dtype=np.float32)
    S1 = np.zeros((M, M), dtype=np.float32)
    S2 = np.zeros((N, N), dtype=np.float32)
    rc = lib().oracle_fill(M, N, s1, s2, w, F, S1, S2)
    if rc != 0:
        raise ValueError("oracle_fill rejected its arguments")
    return F, S1, S2


def r0only(seq1, seq2):
    """R0-only double max-plus (oracle_r0only). seq1, seq2: non-negative integer sequences.
    Returns F[T(M), N, N] (compact layout, -FLT_MAX where i2 > j2)."""
    s1 = np.ascontiguousarray(seq1, dtype=np.int32)
    s2 = np.ascontiguousarray(seq2, dtype=np.int32)
    M, N = len(s1), len(s2)
    F = np.empty((M * (M + 1) // 2, N, N), dtype=np.float32)
    if lib().oracle_r0only(M, N, s1, s2, F) != 0:
        raise ValueError("oracle_r0only rejected its arguments")
    return F


def ref_r0only_available() -> bool:
    return os.path.exists(_REF_R0_CHECK)


def ref_r0only(seq1, seq2):
    """The reference's own R0-only program (oracle/_ref/ospsqmax_check, built from
    IPDPSW/source/R0/ospsq_coarse_diag_top_down/src by oracle/Makefile with -DCHECKING
    -DNO_PROMPT): sequences on stdin, every F(i1<=j1, i2<=j2) printed with %0.2f. Returns the
    compact F like r0only (exact: the printed values are integers)."""
    s1 = [int(x) for x in seq1]
    s2 = [int(x) for x in seq2]
    M, N = len(s1), len(s2)
    out = subprocess.run([_REF_R0_CHECK, str(M), str(N)], input=" ".join(map(str, s1 + s2)) + "\n",
                         capture_output=True, text=True, check=True, env=dict(os.environ, OMP_NUM_THREADS="1"))
    lines = out.stdout.splitlines()
    vals = [float(x) for x in lines[lines.index(next(l for l in lines if l.startswith("Execution time"))) + 1:]]
    F = np.full((M * (M + 1) // 2, N, N), -np.finfo(np.float32).max, dtype=np.float32)
    it = iter(vals)
    for i1 in range(M):
        for j1 in range(i1, M):
            c = cell(M, i1, j1)
            for i2 in range(N):
                for j2 in range(i2, N):
                    F[c, i2, j2] = next(it)
    return F


def cell(M: int, i1: int, j1: int) -> int:
    return i1 * M - i1 * (i1 - 1) // 2 + (j1 - i1)


def score(F, M: int, N: int) -> float:
    return float(F[cell(M, 0, M - 1), 0, N - 1])


def traceback(seq1, seq2, w12, F, S1, S2) -> np.ndarray:
    """Pair-type usage counts (= d score / d w) of the optimum, reference tie-break."""
    s1, s2, w = _as(seq1), _as(seq2), _w(w12)
    counts = np.zeros(12, dtype=np.float64)
    n = lib().oracle_traceback(len(s1), len(s2), s1, s2, w, np.ascontiguousarray(F), np.ascontiguousarray(S1),
                               np.ascontiguousarray(S2), counts)
    if n < 0:
        raise RuntimeError("oracle_traceback failed")
    return counts


def reference_size(M: int, N: int, T: int) -> int:
    return int(lib().oracle_reference_size(M, N, T))


def to_reference_layout(F, M: int, N: int, T: int, fill_value=np.nan) -> np.ndarray:
    out = np.full(reference_size(M, N, T), fill_value, dtype=np.float32)
    lib().oracle_to_reference_layout(M, N, T, np.ascontiguousarray(F), out)
    return out


def reference_written_mask(M: int, N: int, T: int) -> np.ndarray:
    """Boolean mask over the reference linear buffer of the cells the reference fill writes."""
    Ns = (N + T - 1) // T
    R = (T - N % T) % T
    i1 = np.arange(M)[:, None, None, None, None, None]
    j1 = np.arange(M)[None, :, None, None, None, None]
    I2 = np.arange(Ns)[None, None, :, None, None, None]
    J2 = np.arange(Ns)[None, None, None, :, None, None]
    r = np.arange(T + 1)[None, None, None, None, :, None]
    c = np.arange(T)[None, None, None, None, None, :]
    Ri = np.where(I2 == 0, R, 0)
    Rj = np.where((I2 == 0) & (J2 == 0), R, 0)
    m = (i1 <= j1) & (I2 <= J2) & (c >= Rj) & ((r == T) | (r >= Ri))
    return np.broadcast_to(m, (M, M, Ns, Ns, T + 1, T)).reshape(-1)


def logical_from_reference(F_ref, M: int, N: int, T: int) -> np.ndarray:
    """Gather the logical cells of a reference-layout buffer into the compact layout
    (cells with i2 > j2 set to -FLT_MAX). Follows the FTable macro, V3/bpmax-wrapper.c:44."""
    Ns = (N + T - 1) // T
    R = (T - N % T) % T
    V = np.asarray(F_ref).reshape(M, M, Ns, Ns, T + 1, T)
    ii = np.arange(N) + R
    out = np.full((M * (M + 1) // 2, N, N), -np.finfo(np.float32).max, dtype=np.float32)
    iu, ju = np.triu_indices(M)
    I, J = np.meshgrid(ii, ii, indexing="ij")
    tri = I <= J
    for c, (a, b) in enumerate(zip(iu, ju)):
        blk = V[a, b][I // T, J // T, I % T, J % T]
        out[c][tri] = blk[tri]
    return out


def ref_fill(seq1, seq2, w12, N_tile: int, MR: int = 3, NR: int = 8, threads: int | None = None,
             sentinel=np.nan, zero_scratch: bool = True, timed: bool = False):
    """Reference fill into its own linear layout; unwritten cells keep ``sentinel``. With
    ``timed`` returns (table, seconds of the bpmax() call alone)."""
    s1, s2, w = _as(seq1), _as(seq2), _w(w12)
    M, N = len(s1), len(s2)
    out = np.full(reference_size(M, N, N_tile), sentinel, dtype=np.float32)
    if threads is None:
        threads = min(os.cpu_count() or 1, 128)
    secs = ctypes.c_double(0.0)
    rc = ref().ref_bpmax_fill_timed(M, N, N_tile, MR, NR, threads, s1, s2, w, out, int(zero_scratch),
                                    ctypes.byref(secs))
    if rc != 0:
        raise ValueError("reference fill rejected its arguments")
    return (out, secs.value) if timed else out


def ref_verify(seq1, seq2, w12) -> np.ndarray:
    """The reference's memoised verify program; returns F4[M, M, N, N] (i1<=j1, i2<=j2 valid)."""
    s1, s2, w = _as(seq1), _as(seq2), _w(w12)
    M, N = len(s1), len(s2)
    out = np.full(M * M * N * N, np.nan, dtype=np.float32)
    rc = ref().ref_bpmax_verify(M, N, s1, s2, w, out)
    if rc != 0:
        raise ValueError("reference verify rejected its arguments")
    return out.reshape(M, M, N, N)


def compact_from_4d(F4, M: int, N: int) -> np.ndarray:
    out = np.full((M * (M + 1) // 2, N, N), -np.finfo(np.float32).max, dtype=np.float32)
    tri = np.triu(np.ones((N, N), dtype=bool))
    iu, ju = np.triu_indices(M)
    for c, (a, b) in enumerate(zip(iu, ju)):
        out[c][tri] = F4[a, b][tri]
    return out
