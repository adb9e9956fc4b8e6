import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
NATIVE = os.path.join(ROOT, "tests", "native")
sys.path.insert(0, ROOT)
sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


def _stale(out, srcs):
    return not os.path.exists(out) or any(os.path.getmtime(s) > os.path.getmtime(out) for s in srcs)


@pytest.fixture(scope="session")
def replay_lib():
    """The product's stage machine compiled for the host (tests/native/host_replay.cpp)."""
    import ctypes
    src = os.path.join(NATIVE, "host_replay.cpp")
    csrc = os.path.join(ROOT, "dds_gpu_b200", "csrc")
    out = os.path.join(NATIVE, "_build", "libreplay.so")
    deps = [src] + [os.path.join(csrc, f) for f in os.listdir(csrc) if f.endswith(".cuh")]
    if _stale(out, deps):
        os.makedirs(os.path.dirname(out), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-fPIC", "-shared", "-Wno-unknown-pragmas",
                        "-I" + csrc, "-o", out + ".tmp", src], check=True)
        os.replace(out + ".tmp", out)
    return ctypes.CDLL(out)


@pytest.fixture(scope="session")
def ddg():
    """The product package with its library built."""
    from dds_gpu_b200 import build
    build.build()
    import dds_gpu_b200
    dds_gpu_b200.load_library()
    return dds_gpu_b200


@pytest.fixture(scope="session")
def gpu_solver(ddg):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: GPU tests need a B200")
    s = ddg.Solver(tt_log2=10, jobs_per_deal=5, lanes=16384)
    yield s
    s.close()
