"""The 12-byte signature-entry TT (-DDDG_TT_SIG; the reference's -DDD_TT_SIG build,
src/dd.h:74-85,352-437), a speed option that is not strictly exact (a wrong hit needs two
keys with the same tag and the same 64-bit hash). Against fixtures made by the reference
compiled with its signature entries: the stage machine compiled the same way searches the
reference's nodes job for job on the CPU, and libddg_sig.so does on the GPU."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import NATIVE, ROOT, load_golden

P = ctypes.c_void_p
CSRC = os.path.join(ROOT, "dds_gpu_b200", "csrc")
FIXTURES = ["sig_k6_120.npz", "sig_k9_120.npz", "sig_k13_5.npz"]


@pytest.fixture(scope="module")
def sig_replay():
    src = os.path.join(NATIVE, "host_replay.cpp")
    out = os.path.join(NATIVE, "_build", "libreplay_sig.so")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-fPIC", "-shared", "-Wno-unknown-pragmas", "-DDDG_TT_SIG",
                    "-I" + CSRC, "-o", out + ".tmp", src], check=True)
    os.replace(out + ".tmp", out)
    return ctypes.CDLL(out)


@pytest.mark.parametrize("name", FIXTURES)
def test_signature_entries_on_host(sig_replay, name):
    g = load_golden(name)
    h = np.ascontiguousarray(g["hands"])
    n = h.shape[0]
    out = np.zeros(n * 20, np.int32)
    nodes = np.zeros(n * 5, np.uint64)
    assert sig_replay.replay_solve(h.ctypes.data_as(P), ctypes.c_longlong(n), 10, 5, 0, None, 8,
                                   out.ctypes.data_as(P), nodes.ctypes.data_as(P), None) == 0
    assert (out.reshape(n, 5, 4) == g["tricks"]).all()
    assert (nodes == g["nodes_jpd5"]).all()


@pytest.mark.gpu
def test_signature_entries_on_gpu(ddg):
    import torch
    lib = ddg.load_library(ddg.SIG_LIB_PATH)
    assert b"signature" in lib.ddg_version()
    for name in FIXTURES:
        g = load_golden(name)
        n = g["hands"].shape[0]
        s = ddg.Solver(tt_log2=10, lanes=4096, library=lib)
        try:
            d_h = torch.from_numpy(g["hands"].view(np.int64)).cuda()
            d_o = torch.empty(n * 20, dtype=torch.uint8, device="cuda")
            d_n = torch.zeros(n * 5, dtype=torch.int64, device="cuda")
            s.solve_device(d_h.data_ptr(), n, d_o.data_ptr(), 0, d_n.data_ptr())
            assert (d_o.cpu().numpy().reshape(n, 5, 4) == g["tricks"]).all(), name
            assert (d_n.cpu().numpy().view(np.uint64) == g["nodes_jpd5"]).all(), name
        finally:
            s.close()
