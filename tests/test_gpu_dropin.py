"""The drop-in boundary on a B200: callers written for the reference's fill call this library.

* ``shim_harness.cpp`` allocates F exactly like V3/bpmax-wrapper.c:175-197 and calls the C++
  ``bpmax()`` symbol (V3/bpmax.c:129); with weights it first calls bpmax_gpu_shim_set_weights.
* ``oracle/_ref/bpmax_gpu_cli`` is the reference's own, unmodified CLI wrapper and sequence-file
  reader (V3/bpmax-wrapper.c, V3/external_functions.c:315-467) linked against libbpmax_gpu.so
  (built by oracle/Makefile where the reference sources exist); the tests run it on sequence files
  and, in its -DCHECKING -DNO_PROMPT build, compare every F value it prints with the oracle.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from bpmax_b200 import workloads as W

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
LETTERS = "ACGU"


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    from bpmax_b200 import api

    exe = str(tmp_path_factory.mktemp("shim") / "shim_harness")
    libdir = os.path.dirname(api.LIB_PATH)
    subprocess.run(["g++", "-O2", "-o", exe, os.path.join(HERE, "shim_harness.cpp"), f"-L{libdir}", "-lbpmax_gpu",
                    f"-Wl,-rpath,{libdir}"], check=True)
    return exe


@pytest.mark.parametrize("M,N,T,seed,weights", [
    (11, 21, 8, 41, None),                     # the reference's hard-coded weights (shim default)
    (9, 40, 16, 42, W.random_weights(42)),     # weights set through bpmax_gpu_shim_set_weights
])
def test_dropin_shim_links_like_reference_wrapper(harness, tmp_path, oracle_mod, M, N, T, seed, weights):
    s1, s2 = W.pair(M, N, seed)
    inp = " ".join(map(str, list(s1) + list(s2)))
    out = str(tmp_path / "F.bin")
    wargs = [repr(float(x)) for x in weights] if weights is not None else []
    r = subprocess.run([harness, str(M), str(N), str(T), out, *wargs], input=inp, capture_output=True, text=True,
                       check=True)
    Fr = np.fromfile(out, dtype=np.float32)
    w = W.REFERENCE_WEIGHTS if weights is None else np.asarray(weights, dtype=np.float32)
    Fo, _, _ = oracle_mod.fill(s1, s2, w)
    mask = oracle_mod.reference_written_mask(M, N, T)
    mine = oracle_mod.to_reference_layout(Fo, M, N, T)
    assert np.array_equal(bits(mine[mask]), bits(Fr[mask]))
    assert f"F(0,{M - 1},0,{N - 1})" in r.stdout


def test_shim_rejects_bad_weights():
    from bpmax_b200 import api

    L = api.load_library()
    bad = np.array([1.0] * 11 + [-0.5], dtype=np.float32)
    assert L.bpmax_gpu_shim_set_weights(bad.ctypes.data) == 1
    assert L.bpmax_gpu_shim_set_weights(None) == 1
    assert L.bpmax_gpu_shim_set_weights(W.REFERENCE_WEIGHTS.ctypes.data) == 0


def _need_cli(oracle_mod):
    if not oracle_mod.cli_available():
        pytest.skip("the reference's CLI wrapper was not built (its sources were absent at build time)")


@pytest.mark.parametrize("M,N,T,seed", [(20, 33, 16, 71), (13, 64, 32, 72)])
def test_reference_cli_reads_sequence_files(tmp_path, oracle_mod, M, N, T, seed):
    """The reference's CLI, unmodified, on FASTA-like sequence files (its ReadSequencesFromFiles),
    filling through this library: the printed score F(0,M-1,0,N-1) is the oracle's."""
    _need_cli(oracle_mod)
    s1, s2 = W.pair(M, N, seed)
    f1, f2 = tmp_path / "seq1.fa", tmp_path / "seq2.fa"
    f1.write_text(">strand1\n" + "".join(LETTERS[b] for b in s1) + "\n")
    f2.write_text(">strand2 test\n" + "".join(LETTERS[b] for b in s2[:10]) + "\n" +
                  "".join(LETTERS[b] for b in s2[10:]).lower() + "\n")
    r = subprocess.run([oracle_mod._REF_CLI, str(M), str(N), str(T), "3", "8", str(f1), str(f2)],
                       capture_output=True, text=True, check=True, timeout=300)
    assert r.stdout.count("[SUCCESS]") == 2, r.stdout  # both sequences came from the files
    m = re.search(rf"F\(0, {M - 1}, 0, {N - 1}\)=\s*(\S+)", r.stdout)
    assert m, r.stdout
    Fo, _, _ = oracle_mod.fill(s1, s2, W.REFERENCE_WEIGHTS)
    assert float(m.group(1)) == oracle_mod.score(Fo, M, N)


def test_reference_cli_check_build_prints_every_cell(oracle_mod):
    """The wrapper's -DCHECKING -DNO_PROMPT build: sequences as letters on stdin, every logical F
    value printed with %0.2f after the run; all of them equal the oracle's."""
    _need_cli(oracle_mod)
    M, N, T = 9, 19, 8
    s1, s2 = W.pair(M, N, 73)
    inp = "".join(LETTERS[b] for b in s1) + "".join(LETTERS[b] for b in s2)
    r = subprocess.run([oracle_mod._REF_CLI_CHECK, str(M), str(N), str(T), "3", "8"], input=inp,
                       capture_output=True, text=True, check=True, timeout=300)
    lines = r.stdout.splitlines()
    start = next(i for i, l in enumerate(lines) if l.startswith("Execution time")) + 1
    got = lines[start:]
    Fo, _, _ = oracle_mod.fill(s1, s2, W.REFERENCE_WEIGHTS)
    exp = [f"{Fo[oracle_mod.cell(M, a, b), c, d]:0.2f}" for a in range(M) for b in range(a, M)
           for c in range(N) for d in range(c, N)]
    assert got == exp
