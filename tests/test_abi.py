"""The C-ABI library loads and exports every function include/ddg.h declares, and the
Python binding's structs match the header's layout."""
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


def test_struct_layouts_match_the_header(ddg, tmp_path):
    """The ctypes mirrors of ddg_config and ddg_stats have the C header's size and every
    field at the header's offset (a C program built against include/ddg.h prints them)."""
    import subprocess
    structs = {"ddg_config": ddg._Config, "ddg_stats": ddg._Stats}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "ddg.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for name, _ in py._fields_:
            lines.append(f'  printf("{cname}.{name} %zu\\n", offsetof({cname}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(ln.split() for ln in subprocess.run([str(exe)], capture_output=True, text=True,
                                                    check=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for name, _ in py._fields_:
            assert int(got[f"{cname}.{name}"]) == getattr(py, name).offset, f"{cname}.{name}"
