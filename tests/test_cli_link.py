"""The reference's own CLI wrapper links against libbpmax_gpu.so (no GPU needed).

oracle/Makefile compiles the unmodified V3/bpmax-wrapper.c and V3/external_functions.c (where the
reference sources exist) against the GPU library instead of the reference's CPU objects. Without a
GPU the linked program must reach the library's bpmax() and fail loudly: there is no CPU fallback.
"""
import subprocess

import pytest


def test_reference_cli_links_and_refuses_without_gpu(tmp_path, oracle_mod):
    import torch

    if oracle_mod.reference_root() is None:
        pytest.skip("the reference sources are not present")
    oracle_mod.build(["cli"])
    assert oracle_mod.cli_available()
    ldd = subprocess.run(["ldd", oracle_mod._REF_CLI], capture_output=True, text=True).stdout
    assert "libbpmax_gpu.so" in ldd and "not found" not in ldd
    und = subprocess.run(["nm", "-u", oracle_mod._REF_CLI], capture_output=True, text=True).stdout
    assert "_Z5bpmaxllllllllPiS_PPPPPPf" in und  # bpmax() comes from the GPU library
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU tests run the program")
    f1, f2 = tmp_path / "a.fa", tmp_path / "b.fa"
    f1.write_text(">a\nACGUACGUACGU\n")
    f2.write_text(">b\nGGCAUCGAUCGA\n")
    r = subprocess.run([oracle_mod._REF_CLI, "12", "12", "8", "3", "8", str(f1), str(f2)], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode != 0
    assert "no usable CUDA device" in r.stderr
