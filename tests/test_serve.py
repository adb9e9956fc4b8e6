"""The serving load generator (dds_gpu_b200/serve.py): its seeded deal mix, and on the GPU a
short run of Poisson arrivals through a stream whose every finished deal is checked
against the reference's CPU solver (oracle/_ref, else the C restatement) here in the
harness: continuous batching must not change a table."""
import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT

P = ctypes.c_void_p


def cpu_reference():
    ref = os.path.join(ROOT, "oracle", "_ref", "libddref.so")
    if os.path.exists(ref):
        lib = ctypes.CDLL(ref)

        def solve(h):
            n = h.shape[0]
            out = np.zeros(n * 20, np.int32)
            assert lib.ref_solve_batch(h.ctypes.data_as(P), ctypes.c_long(n), 10, 8, out.ctypes.data_as(P), None) == 0
            return out.reshape(n, 5, 4)
        return solve
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "libddoracle.so"))
    lib.ddo_solve_batch.restype = ctypes.c_longlong
    lib.ddo_solve_batch.argtypes = [P, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P]

    def solve(h):
        n = h.shape[0]
        out = np.zeros(n * 20, np.int32)
        lib.ddo_solve_batch(h.ctypes.data, n, 10, 8, 5, None, out.ctypes.data, None)
        return out.reshape(n, 5, 4)
    return solve


def test_mix_is_seeded_and_shaped(ddg):
    from dds_gpu_b200 import serve
    h, k = serve.mix_deals(7, 2000)
    h2, k2 = serve.mix_deals(7, 2000)
    assert (h == h2).all() and (k == k2).all()
    assert 0.66 < (k == 13).mean() < 0.74
    assert set(k[k < 13].tolist()) == {7, 8, 9, 10}
    assert all(ddg.check_deal(x) for x in h[:200])
    assert all(bin(int(x[0])).count("1") == kk for x, kk in zip(h, k))


def test_arrival_times(ddg):
    """A backlog of `prefill` deals at t = 0, then Poisson arrivals at the asked rate, sorted
    and inside the window; the same seed gives the same schedule."""
    from dds_gpu_b200 import serve
    a = serve.arrival_times(20.0, 300.0, seed=5, prefill=150)
    assert (a[:150] == 0).all() and (a[150:] > 0).all() and (np.diff(a) >= 0).all() and a[-1] < 300.0
    assert abs((len(a) - 150) / 300.0 - 20.0) < 20.0 * 0.06  # 6,000 expected: within ~5 sigma
    gaps = np.diff(a[150:])
    assert abs(gaps.mean() - 1 / 20.0) < 0.05 / 20.0 * 5 and abs(gaps.std() / gaps.mean() - 1) < 0.1
    assert (serve.arrival_times(20.0, 300.0, seed=5, prefill=150) == a).all()
    assert len(serve.arrival_times(20.0, 300.0, seed=5)) == len(a) - 150


@pytest.mark.gpu
def test_poisson_stream_matches_reference(ddg):
    from dds_gpu_b200 import serve
    s = ddg.Solver(tt_log2=10, jobs_per_deal=5, lanes=16384)
    try:
        r = serve.run_rate(s, rate=6.0, seconds=8.0, drain_s=20.0, sample_every=1, seed=11)
    finally:
        s.close()
    assert r["arrived"] > 20 and r["admitted"] == r["arrived"]
    hands, ks = serve.mix_deals(11, r["arrived"])
    idx = sorted(r["sample"])
    assert len(idx) >= r["arrived"] * 0.3  # the endings and the easier full deals finished
    got = np.array([r["sample"][i] for i in idx], dtype=np.int32).reshape(-1, 5, 4)
    want = cpu_reference()(np.ascontiguousarray(hands[idx]))
    assert (got == want).all()
    assert r["latency_ms"]["p50"] is not None


@pytest.mark.gpu
def test_guided_stream_matches_reference(ddg):
    """The learned guide inside a stream (seeds and root leads computed as deals are
    submitted, while the persistent solve kernel runs): same tables as the reference."""
    import torch
    from dds_gpu_b200 import guide as ddg_guide
    from dds_gpu_b200 import serve
    params = ddg_guide.load_weights()
    if params is None:
        pytest.skip("no guide weights file")
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    full = ddg.Solver(tt_log2=10, jobs_per_deal=5)
    g = ddg.Guide(device=0, max_rows=4096, params=params)
    try:
        with pytest.raises(ddg.DDGError):  # no SM left for the guide's kernels
            ddg.Stream(full, ring_slots=64, guide=g)
        full.close()
        s = ddg.Solver(tt_log2=10, jobs_per_deal=5, lanes=(sms - 2) * 512)
        try:
            r = serve.run_rate(s, rate=6.0, seconds=8.0, drain_s=20.0, sample_every=1, seed=12, guide=g)
        finally:
            s.close()
    finally:
        g.close()
        full.close()
    hands, _ = serve.mix_deals(12, r["arrived"])
    idx = sorted(r["sample"])
    assert len(idx) >= r["arrived"] * 0.3
    got = np.array([r["sample"][i] for i in idx], dtype=np.int32).reshape(-1, 5, 4)
    assert (got == cpu_reference()(np.ascontiguousarray(hands[idx]))).all()
