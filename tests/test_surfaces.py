"""The drop-in surfaces a caller of the reference uses, run as that caller would:
- a C++ program written against include/dd_solve.hpp (the reference's src/dd.h call
  shapes: dd_solve_strain, dd_solve_strain_guess, dd_ns_tricks, dd_ns_tricks_from);
- the dd_gpu command line, random mode (gpu/gpu_main.cu:307,340 output lines) and Pgx
  FILE.npy mode (gpu/gpu_main.cu:176-188) on a file of this project's seeded deals and the
  reference's tables, written in the dataset's layout;
- the dd_stream command line in stdin mode: 32-byte records in, 28-byte records out, every
  input index exactly once (gpu/stream_main.cu:289-332).
CPU tests build the programs and pin the Pgx writer to the reference's own reader."""
import ctypes
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import NATIVE, ROOT, load_golden
import pgx_np

LIB_DIR = os.path.join(ROOT, "dds_gpu_b200", "_lib")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libddref.so")
LIGHT_13 = [1, 3, 15, 17, 22]  # full deals of k13_24 whose largest job is < 600k nodes


@pytest.fixture(scope="module")
def caller(ddg):
    """tests/native/dd_solve_caller.cpp compiled against include/dd_solve.hpp and libddg.so."""
    src = os.path.join(NATIVE, "dd_solve_caller.cpp")
    out = os.path.join(NATIVE, "_build", "dd_solve_caller")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), "-o", out,
                    src, "-L" + LIB_DIR, "-lddg", "-Wl,-rpath," + LIB_DIR], check=True)
    return out


def test_caller_builds(caller):
    assert os.access(caller, os.X_OK)


def test_pgx_writer_roundtrip():
    g = load_golden("k13_24.npz")
    arr = pgx_np.encode(g["hands"], g["tricks"])
    assert arr.shape == (2, 24, 4) and arr.dtype == np.int32
    h, t = pgx_np.decode(arr)
    assert (h == g["hands"]).all() and (t == g["tricks"]).all()
    with pytest.raises(ValueError):
        pgx_np.encode(load_golden("k6_120.npz")["hands"][:2], g["tricks"][:2])  # not full deals


def test_pgx_writer_matches_reference_reader(tmp_path):
    """A file written by pgx_np is read back by the reference's own decoder (src/npy.h)
    with the same deals and tables."""
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref not built (the reference's sources are not here)")
    ref = ctypes.CDLL(REF_SO)
    P = ctypes.c_void_p
    ref.ref_pgx_load.argtypes = [ctypes.c_char_p, ctypes.c_long, ctypes.c_long, P, P]
    g = load_golden("k13_24.npz")
    path = str(tmp_path / "deals.npy")
    pgx_np.write(path, g["hands"], g["tricks"])
    hands = np.zeros((24, 4), np.uint64)
    tricks = np.zeros(24 * 20, np.int32)
    assert ref.ref_pgx_load(path.encode(), 3, 21, hands[3:].ctypes.data, tricks[60:].ctypes.data) == 0
    assert (hands[3:] == g["hands"][3:]).all()
    assert (tricks[60:].reshape(21, 5, 4) == g["tricks"][3:]).all()


def _full_light_deals():
    """Full deals whose hardest job is light: k13_24's, and the 13-card deals of the
    uneven-hardness fixture (some of them skewed)."""
    a = load_golden("k13_24.npz")
    m = load_golden("mixed_300.npz")
    k = np.array([bin(int(x[0])).count("1") for x in m["hands"]])
    mx = m["nodes_jpd5"].astype(np.int64).reshape(-1, 5).max(axis=1)
    sel = np.where((k == 13) & (mx < 3_000_000))[0]
    hands = np.concatenate([a["hands"][LIGHT_13], m["hands"][sel]])
    tricks = np.concatenate([a["tricks"][LIGHT_13], m["tricks"][sel]])
    return hands, tricks


@pytest.mark.gpu
def test_cpp_header_caller(caller, tmp_path):
    g = load_golden("k7_120.npz")
    n = 6
    path = tmp_path / "deals.bin"
    path.write_bytes(np.ascontiguousarray(g["hands"][:n]).tobytes())
    r = subprocess.run([caller, str(path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    want = g["tricks"][:n].reshape(-1)
    for key in ("strain", "guess", "ns", "ns_from", "deals"):
        assert (np.array(out[key]) == want).all(), key
    # one strain per call, fresh TT generation: the reference's node count of that job
    assert (np.array(out["strain_nodes"]) == g["nodes_jpd5"][: n * 5].astype(np.int64)).all()


@pytest.mark.gpu
def test_ns_tricks_api(ddg, gpu_solver):
    g = load_golden("k8_120.npz")
    for i in range(3):
        for strain in (0, 4):
            for leader in range(4):
                decl = (leader + 3) & 3
                t = int(g["tricks"][i, strain, decl])
                want = t if decl % 2 == 0 else 13 - t
                for guess in (0, 7, 13):
                    assert gpu_solver.ns_tricks(g["hands"][i], strain, leader, guess) == want
                    assert gpu_solver.ns_tricks(g["hands"][i], strain, leader, guess, stepping=True) == want
    with pytest.raises(ddg.DDGError):
        gpu_solver.ns_tricks(g["hands"][0], 0, 4)


@pytest.mark.gpu
def test_dd_gpu_random_mode(ddg):
    exe = os.path.join(LIB_DIR, "dd_gpu")
    env = dict(os.environ, THREADS="8192")
    r = subprocess.run([exe, "6", "300", "10", "300"], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert re.search(r"^GPU: [0-9.]+s, [0-9]+ deals/s \([0-9]+ strain-solves/s\), [0-9]+ nodes/solve$", r.stdout, re.M)
    assert re.search(r"^0 wrong of 6000 checked$", r.stdout, re.M)
    bad = subprocess.run([exe, "14", "10"], capture_output=True, text=True, timeout=60)
    assert bad.returncode == 2


@pytest.mark.gpu
def test_dd_gpu_pgx_file_mode(ddg, tmp_path):
    hands, tricks = _full_light_deals()
    n = len(hands)
    path = str(tmp_path / "deals.npy")
    pgx_np.write(path, hands, tricks)
    exe = os.path.join(LIB_DIR, "dd_gpu")
    r = subprocess.run([exe, path, "0", str(n), "10"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    assert re.search(rf"^0 wrong of {n * 20} checked$", r.stdout, re.M), r.stdout
    # a table entry changed in the file is reported and fails the run (exit 1)
    t2 = tricks.copy()
    t2[2, 4, 1] = (int(t2[2, 4, 1]) + 1) % 14
    pgx_np.write(path, hands, t2)
    r = subprocess.run([exe, path, "2", "1", "10"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 1 and re.search(r"^1 wrong of 20 checked$", r.stdout, re.M), r.stdout
    r = subprocess.run([exe, path, str(n), "5"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1  # range outside the file


@pytest.mark.gpu
def test_dd_stream_stdin_mode(ddg):
    g = load_golden("k7_120.npz")
    exe = os.path.join(LIB_DIR, "dd_stream")
    env = dict(os.environ, THREADS="4096", SLOTS="64")
    r = subprocess.run([exe], input=np.ascontiguousarray(g["hands"]).tobytes(), capture_output=True, timeout=600,
                       env=env)
    assert r.returncode == 0, r.stderr.decode()
    out = np.frombuffer(r.stdout, dtype=np.uint8)
    assert out.size == 120 * 28
    rec = out.reshape(-1, 28)
    idx = rec[:, :8].copy().view(np.uint64).reshape(-1)
    assert sorted(idx.tolist()) == list(range(120))  # every input index exactly once
    got = np.empty((120, 5, 4), np.uint8)
    got[idx.astype(np.int64)] = rec[:, 8:].reshape(-1, 5, 4)
    assert (got == g["tricks"]).all()
