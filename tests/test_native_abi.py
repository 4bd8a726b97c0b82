"""The C-ABI library loads on a machine without a GPU and exports every
entry point that include/chatcarlo_b200.h declares."""
import ctypes as C
import re
from pathlib import Path

import pytest

from chatcarlo_b200 import _native as N

HEADER = Path(__file__).resolve().parent.parent / "include" / "chatcarlo_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cc_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(N.EXPORTED)


@pytest.mark.parametrize("path", [N.LIB_PATH, N.FP64_LIB_PATH])
def test_library_exports_every_declared_symbol(path):
    lib = C.CDLL(str(path))
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_version_and_error_string_without_gpu():
    lib = N.lib()
    assert lib.cc_version() == 1
    assert isinstance(lib.cc_last_error(), bytes)


def test_invalid_arguments_are_rejected_before_any_device_work():
    lib = N.lib()
    assert lib.cc_ctx_create(0, None) == N.CC_E_INVALID
    assert lib.cc_scene_create(None, None, 0, 0, None, None, None) == N.CC_E_INVALID
    assert lib.cc_transport_photons(None, None, None, None, 0, None, None, None, 0, 0, 1,
                                    None, None, None, None, None) == N.CC_E_INVALID
    with pytest.raises(ValueError):
        N.check(N.CC_E_ENERGY_RANGE)


UNET_HEADER = HEADER.parent / "chatcarlo_b200_unet.h"


def test_denoiser_library_exports_every_declared_symbol():
    from chatcarlo_b200 import _unet_native as U
    text = re.sub(r"/\*.*?\*/", "", UNET_HEADER.read_text(), flags=re.S)
    declared = sorted(set(re.findall(r"\b(ccu_[a-z0-9_]+)\s*\(", text)))
    assert declared == sorted(U.EXPORTED)
    lib = U.lib()
    assert not [f for f in declared if not hasattr(lib, f)]
    assert lib.ccu_version() == 1
    # invalid sizes are rejected on the host
    assert lib.ccu_conv3d(None, 16, None, 0, 1, 8, 8, 8, None, None, 16, 1, None, 16, None, None, None) == -1
    assert lib.ccu_gemm_test(None, None, None, 100, 16, 64, 0, 0, None) == -1


def test_kernel_path_setters_reject_unknown_paths_without_gpu():
    from chatcarlo_b200 import _unet_native as U
    lib = U.lib()
    assert lib.ccu_set_wgrad_path(2) == -1
    assert lib.ccu_set_wgrad_path(-1) == -1
    assert lib.ccu_set_wgrad_path(0) == 0
    assert lib.ccu_set_conv_path(5) == -1
    # the weight gradient checks its arguments on the host
    assert lib.ccu_conv3d_wgrad(None, 16, None, 0, 1, 8, 8, 8, None, 16, None, 1, None) == -1
