"""ctypes binding of include/chatcarlo_b200_unet.h (libccunet.so).

No fallback: a missing library raises NativeLibraryError, and every call
that returns an error code raises CCError with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from ._native import CCError, NativeLibraryError

LIB_PATH = Path(os.environ.get("CHATCARLO_B200_UNET_LIB") or
                Path(__file__).resolve().parent / "lib" / "libccunet.so")

EXPORTED = [
    "ccu_version", "ccu_last_error", "ccu_status", "ccu_conv3d", "ccu_conv3d_head", "ccu_conv3d_wgrad",
    "ccu_bias_grad",
    "ccu_avgpool", "ccu_pool_backward", "ccu_up_reduce", "ccu_head", "ccu_input", "ccu_adam", "ccu_adam_clipped",
    "ccu_packed_weight_elems", "ccu_pack_weights", "ccu_set_conv_path", "ccu_set_wgrad_path", "ccu_set_conv_ring",
    "ccu_set_conv_group", "ccu_zero", "ccu_gemm_test",
]

P = C.c_void_p
F = C.POINTER(C.c_float)
I = C.c_int
LL = C.c_longlong

_SIGS = {
    "ccu_version": ([], I),
    "ccu_last_error": ([], C.c_char_p),
    "ccu_status": ([C.POINTER(C.c_uint), I], I),
    "ccu_conv3d": ([P, I, P, I, I, I, I, I, P, P, I, I, P, I, P, P, P], I),
    "ccu_conv3d_head": ([P, I, I, I, I, I, P, P, P, P, P, P, I, P], I),
    "ccu_conv3d_wgrad": ([P, I, P, I, I, I, I, I, P, I, P, I, P], I),
    "ccu_bias_grad": ([P, LL, I, P, P], I),
    "ccu_avgpool": ([P, I, I, I, I, I, P, P], I),
    "ccu_pool_backward": ([P, P, I, I, I, I, I, P, P], I),
    "ccu_up_reduce": ([P, P, I, I, I, I, I, P, P], I),
    "ccu_head": ([P, P, P, P, P, C.c_float, LL, P, P, P, P, P], I),
    "ccu_input": ([P, P, P, I, P, LL, P, P], I),
    "ccu_adam": ([P, P, P, P, LL, C.c_float, C.c_float, C.c_float, C.c_float, I, C.c_float, P], I),
    "ccu_adam_clipped": ([P, P, P, P, LL, C.c_float, C.c_float, C.c_float, C.c_float, I, C.c_float, P, C.c_float,
                          P], I),
    "ccu_packed_weight_elems": ([I, I], LL),
    "ccu_pack_weights": ([P, I, I, P, P, P], I),
    "ccu_set_conv_path": ([I], I),
    "ccu_set_wgrad_path": ([I], I),
    "ccu_set_conv_ring": ([I], I),
    "ccu_set_conv_group": ([I], I),
    "ccu_zero": ([P, LL, P], I),
    "ccu_gemm_test": ([P, P, P, I, I, I, I, I, P], I),
}

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise NativeLibraryError(f"{LIB_PATH} not found; run `python -m chatcarlo_b200.build`")
        _lib = C.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGS.items():
            fn = getattr(_lib, name)
            fn.argtypes = args
            fn.restype = res
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        raise CCError(rc, lib().ccu_last_error().decode())


def status(reset: bool = True) -> int:
    s = C.c_uint()
    check(lib().ccu_status(C.byref(s), int(reset)))
    return int(s.value)
