"""ddg_solve_static, the entry point that allocates nothing (a static device array is its
working memory): same tables as the pooled solver's ddg_solve_device, on two calls in a
row over the same scratch; oversize requests are refused. Collected last on purpose, so it
also runs after every other GPU test has used the device."""
import ctypes

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def static_fn(ddg):
    lib = ddg.load_library()
    f = lib.ddg_solve_static
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return lib, f


def run_static(ddg, hands):
    import torch
    lib, f = static_fn(ddg)
    n = hands.shape[0]
    d_h = torch.from_numpy(np.ascontiguousarray(hands).view(np.int64)).cuda()
    d_o = torch.empty(n * 20, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    rc = f(d_h.data_ptr(), n, d_o.data_ptr(), None)  # legacy default stream
    assert rc == 0, lib.ddg_last_error()
    torch.cuda.synchronize()
    return d_o.cpu().numpy().reshape(n, 5, 4)


def test_static_matches_pooled_solver_twice(ddg):
    a = load_golden("k6_120.npz")
    b = load_golden("k8_120.npz")
    s = ddg.Solver(tt_log2=10, jobs_per_deal=5, lanes=2048, block=256, min_blocks=2)
    try:
        want_a = s.solve(a["hands"])
        want_b = s.solve(b["hands"])
    finally:
        s.close()
    assert (want_a == a["tricks"]).all() and (want_b == b["tricks"]).all()
    import torch
    first = run_static(ddg, a["hands"])   # first call on the device
    free_before, _ = torch.cuda.mem_get_info()
    second = run_static(ddg, b["hands"])  # a second call in a row on the same scratch
    again = run_static(ddg, a["hands"])   # and the first deals once more
    free_after, _ = torch.cuda.mem_get_info()
    assert (first == want_a).all()
    assert (second == want_b).all()
    assert (again == want_a).all()
    # the inputs and outputs are the caller's (allocated in run_static before each call and
    # returned to torch's cache after it); the calls themselves take no device memory (a
    # scratch of this size, 42.6 MB, would show; torch's cache grows by 2 MB segments)
    assert free_before - free_after < (8 << 20)


def test_static_refuses_oversize_and_accepts_empty(ddg):
    lib, f = static_fn(ddg)
    assert f(None, 0, None, None) == 0
    assert f(ctypes.c_void_p(16), (1 << 20) + 1, ctypes.c_void_p(16), None) != 0
    assert b"at most" in lib.ddg_last_error()
    assert f(None, 4, None, None) != 0
