"""salsaa_b200 — B200-native (sm_100a) SALSAA prover hot path.

The compute lives in libsalsaa_gpu.so (CUDA kernels behind the C ABI of
include/salsaa_gpu.h).  This package only loads it and mirrors the
reference's host interface; there is no CPU fallback: if the library is
missing or no GPU is visible, the calls raise.
"""
import ctypes
import os

from .params import PRESETS, SalsaaParams, make_params, preset  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsalsaa_gpu.so")
_lib = None


def lib():
    """The loaded libsalsaa_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libsalsaa_gpu.so is not built; run `python -m salsaa_b200.build`")
        from . import _abi
        _lib = _abi.bind(ctypes.CDLL(LIB_PATH))
    return _lib
