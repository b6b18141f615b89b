"""The C-ABI library loads and exports every symbol of include/ccsd_gpu.h (no GPU needed)."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "ccsd_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ccsd_gpu_\w+)\s*\(", text)))


def test_header_declares_the_et_entry_points():
    names = _declared()
    for n in ("ccsd_gpu_omega", "ccsd_gpu_jacobian", "ccsd_gpu_jacobian_transpose", "ccsd_gpu_energy",
              "ccsd_gpu_set_amplitudes", "ccsd_gpu_solve_gs", "ccsd_gpu_create", "ccsd_gpu_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from et_b200 import ccsd
    lib = ccsd.load_library()
    for name in _declared():
        assert hasattr(lib, name), name
        assert name in ccsd.SIGNATURES, f"python binding missing for {name}"


def test_create_without_device_fails_loudly():
    """No silent CPU path: without an sm_100 device the context cannot be created."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from et_b200 import CCSD, CCSDGPUError
    with pytest.raises(CCSDGPUError):
        CCSD(2, 3, 4)


def test_invalid_dimensions_rejected():
    from et_b200 import ccsd
    lib = ccsd.load_library()
    ctx = ctypes.c_void_p()
    rc = lib.ccsd_gpu_create(0, 3, 4, None, ctypes.byref(ctx))
    assert rc == -1 and not ctx.value
    assert b"positive" in lib.ccsd_gpu_last_error(None)
