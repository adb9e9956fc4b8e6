"""B200-native exact double-dummy solver.

A ctypes binding of the C ABI in ``include/ddg.h`` (``_lib/libddg.so``, built by
``python -m dds_gpu_b200.build``). The library runs the search only on the GPU: there is no
CPU fallback, and a missing library or device is an error.

Card model (the reference's, src/dd.h:13-14): hand = uint64 with bit suit*16+rank, suits
S,H,D,C, ranks 2..A = 0..12; seats N,E,S,W; strains C,D,H,S,NT. Results are
``tricks[deal, strain, declarer]`` (uint8; 255 = not solved).
"""
import ctypes
import os

import numpy as np

__all__ = ["Solver", "Stream", "Guide", "DDGError", "make_deals", "make_deals_mixed", "check_deal", "library_path", "load_library"]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_lib", "libddg.so")
# the same library built with bounds checks on every stack, TT and task index (tests)
CHECK_LIB_PATH = os.path.join(_HERE, "_lib", "libddg_check.so")
# the same library with 12-byte signature TT entries (the reference's DD_TT_SIG option): a
# bucket of 256 bytes instead of 320, any number of relevant cards stored, not strictly
# exact (a wrong hit needs two keys with the same tag and 64-bit hash)
SIG_LIB_PATH = os.path.join(_HERE, "_lib", "libddg_sig.so")
_lib = None
_libs = {}


class DDGError(RuntimeError):
    """A libddg call failed; the message is ddg_last_error()."""


class _Config(ctypes.Structure):
    _fields_ = [("tt_log2", ctypes.c_int), ("lanes", ctypes.c_int), ("block", ctypes.c_int),
                ("jobs_per_deal", ctypes.c_int), ("device", ctypes.c_int), ("schedule", ctypes.c_int),
                ("min_blocks", ctypes.c_int), ("time_limit_s", ctypes.c_double),
                ("mem_fraction", ctypes.c_double), ("help", ctypes.c_int), ("free_below", ctypes.c_int),
                ("free_steps", ctypes.c_int), ("phase_spread", ctypes.c_int),
                ("cheap_limit", ctypes.c_int), ("help_share_tt", ctypes.c_int), ("flat_moves", ctypes.c_int),
                ("free_pack", ctypes.c_int)]


class _Stats(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_uint64), ("tt_probes", ctypes.c_uint64), ("tt_hits", ctypes.c_uint64),
                ("tt_stores", ctypes.c_uint64), ("tt_bytes", ctypes.c_uint64),
                ("enter_exit", ctypes.c_uint64 * 7), ("phase_warps", ctypes.c_uint64 * 5),
                ("phase_items", ctypes.c_uint64 * 5), ("phase_cycles", ctypes.c_uint64 * 5),
                ("free_rounds", ctypes.c_uint64), ("free_cycles", ctypes.c_uint64),
                ("iterations", ctypes.c_uint64),
                ("tasks", ctypes.c_uint64),
                ("jobs_done", ctypes.c_int64),
                ("kernel_ms", ctypes.c_double), ("lanes", ctypes.c_int), ("grid", ctypes.c_int),
                ("block", ctypes.c_int), ("tt_entry_reads", ctypes.c_uint64)]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if isinstance(v, ctypes.Array) else v
        return d


P = ctypes.c_void_p


def library_path():
    return _LIB_PATH


def load_library(path=None):
    """Loads libddg.so (once; `path` = another build of it, e.g. CHECK_LIB_PATH). Raises
    DDGError when it has not been built."""
    global _lib
    if path is None and _lib is not None:
        return _lib
    path = path or _LIB_PATH
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise DDGError(f"{path} is missing: build it with `python -m dds_gpu_b200.build`")
    lib = ctypes.CDLL(path)
    lib.ddg_version.restype = ctypes.c_char_p
    lib.ddg_last_error.restype = ctypes.c_char_p
    lib.ddg_config_default.argtypes = [ctypes.POINTER(_Config)]
    lib.ddg_solver_create.argtypes = [ctypes.POINTER(_Config), ctypes.POINTER(P)]
    lib.ddg_solver_destroy.argtypes = [P]
    lib.ddg_solver_lanes.argtypes = [P]
    lib.ddg_solver_bytes.argtypes = [P]
    lib.ddg_solver_bytes.restype = ctypes.c_int64
    lib.ddg_solver_nodes.argtypes = [P]
    lib.ddg_solver_nodes.restype = ctypes.c_uint64
    lib.ddg_solver_set_job_times.argtypes = [P, P]
    lib.ddg_solver_set_job_starts.argtypes = [P, P]
    lib.ddg_solve_batch.argtypes = [P, P, ctypes.c_int64, P, ctypes.POINTER(_Stats)]
    lib.ddg_solve_batch_seeded.argtypes = [P, P, ctypes.c_int64, P, P, ctypes.POINTER(_Stats)]
    lib.ddg_solve_device.argtypes = [P, P, ctypes.c_int64, P, P, P, P, ctypes.POINTER(_Stats)]
    lib.ddg_solve_graph.argtypes = [P, P, ctypes.c_int64, P, P, P, ctypes.POINTER(_Stats)]
    lib.ddg_solve_device_ex.argtypes = [P, P, ctypes.c_int64, P, P, P, P, P, P, ctypes.POINTER(_Stats)]
    lib.ddg_solve_begin.argtypes = [P, P, ctypes.c_int64, P, P, P]
    lib.ddg_solve_begin_ex.argtypes = [P, P, ctypes.c_int64, P, P, P, P]
    lib.ddg_solve_continue.argtypes = [P, ctypes.c_double, P, P, P, ctypes.POINTER(_Stats),
                                       ctypes.POINTER(ctypes.c_int)]
    lib.ddg_solve_strain.argtypes = [P, P, ctypes.c_int, P, P]
    lib.ddg_ns_tricks.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_int)]
    lib.ddg_stream_open.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.POINTER(P)]
    lib.ddg_stream_open_guided.argtypes = [P, ctypes.c_int, ctypes.c_double, P, ctypes.POINTER(P)]
    lib.ddg_stream_submit.argtypes = [P, P, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    lib.ddg_stream_poll.argtypes = [P, P, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    lib.ddg_stream_in_flight.argtypes = [P]
    lib.ddg_stream_in_flight.restype = ctypes.c_int64
    lib.ddg_stream_capacity.argtypes = [P]
    lib.ddg_stream_capacity.restype = ctypes.c_int64
    lib.ddg_stream_close.argtypes = [P, ctypes.c_int, ctypes.POINTER(_Stats)]
    lib.ddg_guide_param_count.restype = ctypes.c_int64
    lib.ddg_guide_create.argtypes = [ctypes.c_int, ctypes.c_int, P, ctypes.POINTER(P)]
    lib.ddg_guide_destroy.argtypes = [P]
    lib.ddg_guide_destroy.restype = None
    lib.ddg_guide_get_params.argtypes = [P, P]
    lib.ddg_guide_set_params.argtypes = [P, P]
    lib.ddg_guide_train_step.argtypes = [P, P, P, P, P, ctypes.c_int, ctypes.c_float, P, P]
    lib.ddg_guide_predict.argtypes = [P, P, ctypes.c_int64, P, P]
    lib.ddg_check_deal.argtypes = [P]
    lib.ddg_make_deals.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, P]
    lib.ddg_make_deals.restype = None
    lib.ddg_make_deals_mixed.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, P]
    lib.ddg_make_deals_mixed.restype = None
    _libs[path] = lib
    if path == _LIB_PATH:
        _lib = lib
    return lib


def _check(last_error, rc):
    """Raises DDGError with the library's message (its own ddg_last_error) for rc != 0."""
    if rc != 0:
        raise DDGError(f"ddg error {rc}: {last_error().decode()}")


def make_deals(seed, first, n, k=13):
    """Seeded deals [first, first+n) with k cards per hand: (n, 4) uint64 (ddg_make_deals)."""
    out = np.zeros((n, 4), dtype=np.uint64)
    if n:
        load_library().ddg_make_deals(ctypes.c_uint64(seed), first, n, k, out.ctypes.data)
    return out


def make_deals_mixed(seed, first, n, k_min=5, k_max=13, skew=0.3):
    """Uneven-hardness deals (ddg_make_deals_mixed): K ~ U{k_min..k_max}, a share `skew`
    with a 7-10 card suit facing a void. (n, 4) uint64."""
    out = np.zeros((n, 4), dtype=np.uint64)
    if n:
        load_library().ddg_make_deals_mixed(ctypes.c_uint64(seed), first, n, k_min, k_max, skew, out.ctypes.data)
    return out


def check_deal(hands4):
    h = np.ascontiguousarray(hands4, dtype=np.uint64)
    return load_library().ddg_check_deal(h.ctypes.data) == 0


class Solver:
    """A solver pool on one GPU (ddg_solver_create): per-lane TTs and stacks in HBM."""

    def __init__(self, tt_log2=10, lanes=0, block=0, jobs_per_deal=5, device=0, schedule=0,
                 time_limit_s=0.0, mem_fraction=0.85, min_blocks=0, help=0, free_below=0, free_steps=0,
                 phase_spread=0, cheap_limit=0, library=None, help_share_tt=0, flat_moves=0, free_pack=0):
        lib = library or load_library()
        cfg = _Config()
        lib.ddg_config_default(ctypes.byref(cfg))
        cfg.tt_log2, cfg.lanes, cfg.block = tt_log2, lanes, block
        cfg.jobs_per_deal, cfg.device, cfg.schedule = jobs_per_deal, device, schedule
        cfg.min_blocks = min_blocks
        cfg.help = help
        cfg.free_below, cfg.free_steps = free_below, free_steps
        cfg.phase_spread = phase_spread
        cfg.cheap_limit = cheap_limit
        cfg.help_share_tt = help_share_tt
        cfg.flat_moves = flat_moves
        cfg.free_pack = free_pack
        cfg.time_limit_s, cfg.mem_fraction = time_limit_s, mem_fraction
        self._lib = lib
        self._h = P()
        _check(lib.ddg_last_error, lib.ddg_solver_create(ctypes.byref(cfg), ctypes.byref(self._h)))
        self.config = {name: getattr(cfg, name) for name, _ in cfg._fields_}
        blk = block or 512
        self.block_shape = f"{blk}, {min_blocks or (2 if blk == 256 else 1)}"
        self.jobs_per_deal = jobs_per_deal
        self.last_stats = None

    @property
    def lanes(self):
        return self._lib.ddg_solver_lanes(self._h)

    @property
    def nbytes(self):
        return self._lib.ddg_solver_bytes(self._h)

    def close(self):
        if self._h:
            self._lib.ddg_solver_destroy(self._h)
            self._h = P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, hands, seeds=None):
        """Tricks (n, 5, 4) uint8 for deals (n, 4) uint64 in host memory; `seeds`: optional
        NS-trick seeds (n, 5, 4) for the stepping search."""
        h = np.ascontiguousarray(hands, dtype=np.uint64).reshape(-1, 4)
        n = h.shape[0]
        out = np.empty((n, 5, 4), dtype=np.uint8)
        st = _Stats()
        if seeds is None:
            _check(self._lib.ddg_last_error, self._lib.ddg_solve_batch(self._h, h.ctypes.data, n, out.ctypes.data, ctypes.byref(st)))
        else:
            sd = np.ascontiguousarray(seeds, dtype=np.int8).reshape(n, 20)
            _check(self._lib.ddg_last_error, self._lib.ddg_solve_batch_seeded(self._h, h.ctypes.data, n, sd.ctypes.data,
                                                    out.ctypes.data, ctypes.byref(st)))
        self.last_stats = st.as_dict()
        return out

    def solve_device(self, d_hands, n, d_out, d_seeds=0, d_job_nodes=0, stream=0, d_hints=0, d_best=0):
        """Device-pointer form (ddg_solve_device / _ex): integer addresses of device buffers;
        d_hints / d_best = the guide's root leads in and best leads out (n*20 int8)."""
        st = _Stats()
        _check(self._lib.ddg_last_error, self._lib.ddg_solve_device_ex(self._h, P(d_hands), n, P(d_seeds or None), P(d_hints or None),
                                             P(d_out), P(d_best or None), P(d_job_nodes or None),
                                             P(stream or None), ctypes.byref(st)))
        self.last_stats = st.as_dict()
        return self.last_stats

    def begin(self, d_hands, n, d_out, d_seeds=0, stream=0, d_hints=0):
        """Starts a resumable solve on device buffers (ddg_solve_begin_ex)."""
        _check(self._lib.ddg_last_error, self._lib.ddg_solve_begin_ex(self._h, P(d_hands), n, P(d_seeds or None), P(d_hints or None),
                                            P(d_out), P(stream or None)))

    def resume(self, seconds, hands_host=0, out_host=0, stream=0):
        """Runs the resumable solve for at most `seconds` (ddg_solve_continue); returns
        (finished, stats of the slice)."""
        st = _Stats()
        fin = ctypes.c_int(0)
        _check(self._lib.ddg_last_error, self._lib.ddg_solve_continue(self._h, seconds, P(hands_host or None), P(out_host or None),
                                            P(stream or None), ctypes.byref(st), ctypes.byref(fin)))
        self.last_stats = st.as_dict()
        return bool(fin.value), self.last_stats

    def solve_graph(self, d_hands, n, d_out, d_seeds=0, stream=0):
        """The batch solve as a replayed CUDA graph (ddg_solve_graph)."""
        st = _Stats()
        _check(self._lib.ddg_last_error, self._lib.ddg_solve_graph(self._h, P(d_hands), n, P(d_seeds or None), P(d_out), P(stream or None),
                                         ctypes.byref(st)))
        self.last_stats = st.as_dict()
        return self.last_stats

    def set_job_times(self, d_job_end_ns, d_job_start_ns=None):
        """Device buffers (integer addresses, n*jobs_per_deal uint64) for job completion
        times and, when given, the times the jobs were taken (0 = unused)."""
        _check(self._lib.ddg_last_error, self._lib.ddg_solver_set_job_times(self._h, P(d_job_end_ns or None)))
        if d_job_start_ns is not None:
            _check(self._lib.ddg_last_error, self._lib.ddg_solver_set_job_starts(self._h, P(d_job_start_ns or None)))

    def solve_strain(self, hands4, strain, ns4=None):
        """One strain of one deal, declarers N,E,S,W (the reference's dd_solve_strain)."""
        h = np.ascontiguousarray(hands4, dtype=np.uint64).reshape(4)
        out = np.zeros(4, dtype=np.int32)
        s4 = None if ns4 is None else np.ascontiguousarray(ns4, dtype=np.int32)
        _check(self._lib.ddg_last_error, self._lib.ddg_solve_strain(self._h, h.ctypes.data, strain,
                                          None if s4 is None else s4.ctypes.data, out.ctypes.data))
        return [int(x) for x in out]

    def ns_tricks(self, hands4, strain, leader, guess=7, stepping=False):
        """NS tricks with `leader` on lead (the reference's dd_ns_tricks, or dd_ns_tricks_from
        with stepping=True, starting at `guess`)."""
        h = np.ascontiguousarray(hands4, dtype=np.uint64).reshape(4)
        v = ctypes.c_int(0)
        _check(self._lib.ddg_last_error, self._lib.ddg_ns_tricks(self._h, h.ctypes.data, strain, leader, guess, 1 if stepping else 0,
                                       ctypes.byref(v)))
        return v.value


class Stream:
    """Continuous batching on one solver (ddg_stream_*): submit deals while others are on
    the GPU, poll 28-byte records (index, 20 tricks) as deals finish, out of order."""

    def __init__(self, solver, ring_slots=0, idle_timeout_s=0.0, guide=None):
        """`guide`: a Guide on the solver's device whose seeds and root leads steer every
        deal's search (the solver then needs at most (SMs - 2) * block lanes)."""
        self._lib = solver._lib
        self._h = P()
        _check(self._lib.ddg_last_error,
               self._lib.ddg_stream_open_guided(solver._h, ring_slots, idle_timeout_s,
                                                guide._h if guide is not None else None, ctypes.byref(self._h)))
        self._guide = guide  # kept alive while the stream uses it
        self.stats = None

    @property
    def in_flight(self):
        return self._lib.ddg_stream_in_flight(self._h)

    @property
    def capacity(self):
        return self._lib.ddg_stream_capacity(self._h)

    def submit(self, hands):
        """Submits deals (n, 4) uint64 in order; returns how many were admitted (a prefix)."""
        h = np.ascontiguousarray(hands, dtype=np.uint64).reshape(-1, 4)
        acc = ctypes.c_int64(0)
        _check(self._lib.ddg_last_error, self._lib.ddg_stream_submit(self._h, h.ctypes.data, h.shape[0], ctypes.byref(acc)))
        return acc.value

    def poll(self, max_records=65536):
        """Finished deals: (indices uint64 (k,), tricks uint8 (k, 5, 4))."""
        buf = np.empty(max_records * 28, dtype=np.uint8)
        got = ctypes.c_int64(0)
        _check(self._lib.ddg_last_error, self._lib.ddg_stream_poll(self._h, buf.ctypes.data, max_records, ctypes.byref(got)))
        rec = buf[: got.value * 28].reshape(-1, 28)
        return rec[:, :8].copy().view(np.uint64).reshape(-1), rec[:, 8:].reshape(-1, 5, 4).copy()

    def close(self, drain=True):
        """Ends the stream; drain=True waits for every submitted deal, False drops them."""
        if self._h:
            st = _Stats()
            h, self._h = self._h, P()
            _check(self._lib.ddg_last_error, self._lib.ddg_stream_close(h, 1 if drain else 0, ctypes.byref(st)))
            self.stats = st.as_dict()
        return self.stats

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Guide:
    """The learned guide (ddg_guide_*): an MLP trained and run on the GPU by libddg's own
    tensor-core kernels; predicts NS-trick seeds and root leads for the solver."""

    def __init__(self, device=0, max_rows=4096, params=None):
        self._lib = load_library()
        self._h = P()
        p = None
        if params is not None:
            p = np.ascontiguousarray(params, dtype=np.float32).reshape(-1)
            if p.size != self.param_count():
                raise DDGError(f"guide parameters: {p.size} values, {self.param_count()} expected")
        _check(self._lib.ddg_last_error, self._lib.ddg_guide_create(device, max_rows, p.ctypes.data if p is not None else None,
                                          ctypes.byref(self._h)))
        self.max_rows = max_rows

    @staticmethod
    def param_count():
        return int(load_library().ddg_guide_param_count())

    def close(self):
        if self._h:
            self._lib.ddg_guide_destroy(self._h)
            self._h = P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        out = np.empty(self.param_count(), dtype=np.float32)
        _check(self._lib.ddg_last_error, self._lib.ddg_guide_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32).reshape(-1)
        _check(self._lib.ddg_last_error, self._lib.ddg_guide_set_params(self._h, p.ctypes.data))

    def step(self, d_hands, d_tricks20, d_best20, rows, lr, want_grad=False):
        """One training step on example indices `rows` (deal*20 + strain*4 + declarer);
        returns (mean loss, trick-head hits, labelled rows, gradients or None)."""
        r = np.ascontiguousarray(rows, dtype=np.int64)
        stats = np.zeros(3, dtype=np.float32)
        grad = np.empty(self.param_count(), dtype=np.float32) if want_grad else None
        _check(self._lib.ddg_last_error, self._lib.ddg_guide_train_step(self._h, P(d_hands), P(d_tricks20), P(d_best20), r.ctypes.data,
                                              r.size, lr, stats.ctypes.data,
                                              grad.ctypes.data if grad is not None else None))
        return float(stats[0]), float(stats[1]), float(stats[2]), grad

    def predict(self, d_hands, n, d_seed20=0, d_hint20=0):
        _check(self._lib.ddg_last_error, self._lib.ddg_guide_predict(self._h, P(d_hands), n, P(d_seed20 or None), P(d_hint20 or None)))
