"""The C-ABI library builds for sm_100a and exports every entry point that
include/oa_gpu.h declares (no compute calls: no GPU here)."""
import ctypes
import os
import re
import shutil

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "oa_gpu.h")).read()
    return sorted(set(re.findall(r"\b(oa_gpu_\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib_path():
    from openatom_b200 import build
    if not os.path.exists(build.LIB) and shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"):
        pytest.skip("no nvcc and no prebuilt library")
    return build.build()


def test_header_lists_entry_points():
    syms = header_symbols()
    assert "oa_gpu_init" in syms and "oa_gpu_state_fft_fwd" in syms and len(syms) >= 15


def test_library_exports_all_header_symbols(lib_path):
    lib = ctypes.CDLL(lib_path)
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header(lib_path):
    from openatom_b200.gpu import SIGNATURES
    assert set(header_symbols()) <= set(SIGNATURES)


def test_no_cpu_fallback_without_gpu(lib_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from openatom_b200.gpu import CPContext
    from openatom_b200.system import make_system
    with pytest.raises(RuntimeError):
        CPContext(make_system("w2"), "fp64")
