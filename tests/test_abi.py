"""CPU tests of the C ABI boundary: both libraries load and export every entry point that
include/ironav_inter.h declares; without a CUDA device the CUDA library refuses to create a context
with HardwareUnavailable (no silent fallback); the Python binding's structure layouts match the C ones."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

from ironav_b200 import build
from ironav_b200.inter import EXPORTS, MBRESULT_DTYPE, MBSTATE_DTYPE, InterStage, IronavError, cuda_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ironav_inter.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ironav_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert sorted(EXPORTS) == declared_functions()


def test_cuda_library_exports_every_declared_symbol():
    build.build_cuda()
    lib = ctypes.CDLL(build.CUDA_LIB)
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_oracle_exports_every_declared_symbol(oracle_lib):
    missing = [f for f in declared_functions() if not hasattr(oracle_lib, f)]
    assert not missing, missing


def test_struct_layouts():
    assert MBSTATE_DTYPE.itemsize == 72
    assert MBRESULT_DTYPE.itemsize == 104
    assert MBRESULT_DTYPE.fields["cost"][1] == 20
    assert MBRESULT_DTYPE.fields["mvs"][1] == 24
    assert MBRESULT_DTYPE.fields["sad_px"][1] == 92


def test_host_helpers_agree_between_libraries(oracle_lib):
    lib = cuda_library()
    for q in range(0, 64):
        assert lib.ironav_lambda(q) == oracle_lib.ironav_lambda(q)
        assert lib.ironav_skip_threshold(q) == oracle_lib.ironav_skip_threshold(q)
    for v in range(-3000, 3000, 7):
        assert lib.ironav_se_bits(v) == oracle_lib.ironav_se_bits(v)
    assert lib.ironav_version().startswith(b"cuda-sm_100a")


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the behaviour without a CUDA device")
def test_no_device_means_hardware_unavailable():
    with pytest.raises(IronavError) as e:
        InterStage(64, 48)
    assert e.value.status == 8


def test_invalid_arguments_on_the_oracle(oracle_lib):
    with pytest.raises(IronavError) as e:
        InterStage(63, 48, lib=oracle_lib)
    assert e.value.status == 3
    with pytest.raises(IronavError):
        InterStage(64, 48, nslices=4, lib=oracle_lib)  # more bands than macroblock rows
    with pytest.raises(IronavError):
        InterStage(64, 48, nslices=2, band_rows=[0, 0, 3], lib=oracle_lib)
    st = InterStage(64, 48, lib=oracle_lib)
    with pytest.raises(IronavError):
        st.begin_p_picture(26)  # no reference picture yet
