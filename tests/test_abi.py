"""The C-ABI library loads and exports every function include/ddg.h declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ddg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_api():
    names = declared("ddg.h")
    for need in ("ddg_solver_create", "ddg_solve_batch", "ddg_solve_batch_seeded", "ddg_solve_device",
                 "ddg_solve_strain", "ddg_last_error"):
        assert need in names


def test_library_exports_every_declared_symbol(ddg):
    lib = ctypes.CDLL(ddg.library_path())
    missing = [n for n in declared("ddg.h") if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_errors(ddg):
    lib = ddg.load_library()
    assert b"sm_100a" in lib.ddg_version()
    import numpy as np
    bad = np.zeros(4, np.uint64)
    assert lib.ddg_check_deal(bad.ctypes.data) != 0
    assert b"size" in lib.ddg_last_error()


def test_no_cpu_fallback_without_device(ddg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(ddg.DDGError):
        ddg.Solver(lanes=128)


def test_config_checked_before_any_device_call(ddg):
    """Out-of-range configuration is refused with its own message (no device needed)."""
    with pytest.raises(ddg.DDGError, match="free_pack"):
        ddg.Solver(free_pack=33)
    with pytest.raises(ddg.DDGError, match="tt_log2"):
        ddg.Solver(tt_log2=30)
