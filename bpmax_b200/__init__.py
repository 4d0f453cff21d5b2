"""B200-native BPMax fill engine: hand-written sm_100a CUDA kernels behind a C ABI
(include/bpmax_gpu.h, library bpmax_b200/libbpmax_gpu.so) with a thin ctypes mirror."""
from .api import BpmaxError, Engine, load_library  # noqa: F401
from . import workloads  # noqa: F401

__all__ = ["Engine", "BpmaxError", "load_library", "workloads"]
