"""C ABI checks that need no GPU: the library loads, exports every function include/*.h declares
plus the reference's C++ bpmax() symbol, and refuses to run without a B200 (no CPU fallback)."""
import ctypes
import subprocess

import pytest

from bpmax_b200 import api


def test_library_exports_header_functions():
    L = api.load_library()
    names = api.header_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(L, n), n


def test_library_exports_reference_bpmax_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", api.LIB_PATH], capture_output=True, text=True).stdout
    # void bpmax(long, long, long, long, long, long, long, long, int*, int*, float******)
    assert "_Z5bpmaxllllllllPiS_PPPPPPf" in out


def test_engine_refuses_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.BpmaxError) as e:
        api.Engine(0)
    assert e.value.status == 4


def test_status_strings():
    L = api.load_library()
    assert L.bpmax_gpu_status_string(0) == b"ok"
    assert L.bpmax_gpu_status_string(5) == b"device wait timed out"
