"""Batched sampling: many independent problems in one call.

``sample_batch`` takes host arrays and anneals every problem's states in place
(``b200sa_sample_batch``).  ``Plan`` keeps the packed problems resident on the
device and runs on device buffers (torch CUDA tensors), the form used for
repeated runs and by the autograd layer.  Each read equals the reference run
with ``num_samples=1`` and that read's seed.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _lib
from .workloads import Instance

MODES = {"persistent": _lib.MODE_PERSISTENT, "plain": _lib.MODE_PLAIN, "graph": _lib.MODE_GRAPH,
         "plain_tuned": _lib.MODE_PLAIN_TUNED}
CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy


def _proposal_code(p: str) -> int:
    c = p.lower()
    if c == "gibbs":
        return _lib.GIBBS
    if c == "metropolis":
        return _lib.METROPOLIS
    raise ValueError(f"Unknown proposal_acceptance_criteria: {p}")


class _Packed:
    """ctypes problem array plus the numpy buffers it points into."""

    def __init__(self, problems: Sequence[Instance], need_states: bool,
                 energies: list | None = None):
        self.keep = []
        self.arr = (_lib.Problem * max(len(problems), 1))()
        self.energies = energies if energies is not None else []
        for i, p in enumerate(problems):
            h = np.ascontiguousarray(p.h, dtype=np.float64)
            u = np.ascontiguousarray(p.u, dtype=np.int32)
            v = np.ascontiguousarray(p.v, dtype=np.int32)
            J = np.ascontiguousarray(p.J, dtype=np.float64)
            betas = np.ascontiguousarray(p.betas, dtype=np.float64)
            seeds = np.ascontiguousarray(p.seeds, dtype=np.uint64)
            if not (u.shape == v.shape == J.shape):
                raise ValueError("coupler vectors have mismatched lengths")
            R = p.num_reads
            if seeds.shape != (R,):
                raise ValueError(f"problem {i}: need one seed per read")
            st = p.states
            if need_states:
                if st.dtype != np.int8 or not st.flags.c_contiguous or st.shape != (R, p.n):
                    raise ValueError(f"problem {i}: states must be C-contiguous int8 (R, n)")
            if energies is None:
                self.energies.append(np.zeros(R, dtype=np.float64))
            en = self.energies[i]
            self.keep += [h, u, v, J, betas, seeds, st, en]
            q = self.arr[i]
            q.num_vars = p.n
            q.h = h.ctypes.data
            q.num_couplers = J.shape[0]
            q.coupler_starts = u.ctypes.data
            q.coupler_ends = v.ctypes.data
            q.coupler_weights = J.ctypes.data
            q.num_reads = R
            q.states = st.ctypes.data if need_states else None
            q.energies = en.ctypes.data
            q.sweeps_per_beta = int(p.sweeps_per_beta)
            q.num_betas = betas.shape[0]
            q.beta_schedule = betas.ctypes.data
            q.seeds = seeds.ctypes.data
            q.varorder = _lib.RANDOM if p.randomize_order else _lib.SEQUENTIAL
            q.proposal = _proposal_code(p.proposal)


def sample_batch(problems: Sequence[Instance], mode: str = "persistent", device: int = 0,
                 stats: dict | None = None) -> list[np.ndarray]:
    """Anneal every problem's ``states`` in place; returns per-problem energies.

    ``stats`` (a dict) receives the run's counters and ``near_ties_per_read``,
    one array per problem with each read's near-tie count."""
    packed = _Packed(problems, need_states=True)
    L = _lib.load()
    st = _lib.Stats()
    ties = np.zeros(sum(p.num_reads for p in problems), dtype=np.uint32)
    st.read_near_ties = ties.ctypes.data
    err = _lib.errbuf()
    rc = L.b200sa_sample_batch(packed.arr, len(problems), MODES[mode], int(device),
                               ctypes.byref(st), err, len(err))
    _lib.check(rc, err)
    if stats is not None:
        stats.update(st.as_dict())
        offs = np.cumsum([0] + [p.num_reads for p in problems])
        stats["near_ties_per_read"] = [ties[offs[i]:offs[i + 1]] for i in range(len(problems))]
    return packed.energies


class Plan:
    """Problems packed once and kept on the device.

    ``run`` anneals device buffers: ``states_in`` / ``states_out`` are int8
    CUDA tensors of ``total_state`` elements (problem after problem, each
    ``R x n`` row-major) and ``energies`` a float64 CUDA tensor of
    ``total_reads`` elements.
    """

    def __init__(self, problems: Sequence[Instance], device: int = 0):
        self._packed = _Packed(problems, need_states=False)
        self._lib = _lib.load()
        self.handle = ctypes.c_void_p()
        err = _lib.errbuf()
        rc = self._lib.b200sa_plan_create(self._packed.arr, len(problems), int(device),
                                          ctypes.byref(self.handle), err, len(err))
        _lib.check(rc, err)
        k = len(problems) + 1
        so = np.zeros(k, dtype=np.int64)
        ro = np.zeros(k, dtype=np.int64)
        self._lib.b200sa_plan_layout(self.handle, so.ctypes.data, ro.ctypes.data)
        self.state_offsets = so
        self.read_offsets = ro
        self.total_state = int(so[-1])
        self.total_reads = int(ro[-1])
        self.device = int(device)
        self.attempts = int(sum(p.attempts for p in problems))

    def run(self, states_in, states_out, energies, seeds=None, mode: str = "persistent",
            stream=None, sync: bool = True, per_read: bool = False) -> dict:
        """Anneal on the device.  Arguments are CUDA tensors (or raw device
        pointers as ints).  Returns the run's counters when ``sync``; with
        ``per_read`` also ``near_ties_per_read`` (one count per read, at the
        plan's read offsets)."""
        def ptr(x):
            if x is None:
                return None
            return x if isinstance(x, int) else x.data_ptr()
        st = _lib.Stats()
        ties = None
        if per_read and sync:
            ties = np.zeros(self.total_reads, dtype=np.uint32)
            st.read_near_ties = ties.ctypes.data
        err = _lib.errbuf()
        s = None
        if stream is not None:
            s = stream if isinstance(stream, int) else stream.cuda_stream
            if s == 0:  # the legacy default stream: pass cudaStreamLegacy, not NULL
                s = CUDA_STREAM_LEGACY
        rc = self._lib.b200sa_plan_run(self.handle, MODES[mode], ptr(states_in),
                                       ptr(states_out), ptr(energies), ptr(seeds), s,
                                       1 if sync else 0, ctypes.byref(st), err, len(err))
        _lib.check(rc, err)
        out = st.as_dict()
        if ties is not None:
            out["near_ties_per_read"] = ties
        return out

    def set_weights(self, problem: int, h, J):
        """Replace problem ``problem``'s fields and coupler weights (COO order
        as given at creation); structure, schedule and seeds are kept."""
        h = np.ascontiguousarray(h, dtype=np.float64)
        J = np.ascontiguousarray(J, dtype=np.float64)
        err = _lib.errbuf()
        rc = self._lib.b200sa_plan_set_weights(self.handle, int(problem), h.ctypes.data,
                                               J.ctypes.data, err, len(err))
        _lib.check(rc, err)

    def set_weights_device(self, h_cat, J_cat, stream=None):
        """Replace the fields and coupler weights of every problem from device
        tensors (float64 CUDA tensors: all problems' h concatenated, and all
        problems' J in COO order concatenated), enqueued on ``stream``."""
        for x in (h_cat, J_cat):
            if x.dtype.itemsize != 8 or not x.is_cuda or not x.is_contiguous():
                raise ValueError("h_cat and J_cat must be contiguous float64 CUDA tensors")
        s = None
        if stream is not None:
            s = stream if isinstance(stream, int) else stream.cuda_stream
            if s == 0:
                s = CUDA_STREAM_LEGACY
        err = _lib.errbuf()
        rc = self._lib.b200sa_plan_set_weights_device(self.handle, h_cat.data_ptr(),
                                                      J_cat.data_ptr(), s, err, len(err))
        _lib.check(rc, err)

    def autotune(self, cache_path: str | None = None, force: bool = False) -> list[dict]:
        """Measure launch configurations per size bucket and keep the fastest
        for persistent / graph runs (results are unchanged).  Choices are
        cached in ``cache_path``.  Returns one dict per non-empty bucket."""
        cap = 64
        rep = (_lib.TuneEntry * cap)()
        err = _lib.errbuf()
        path = cache_path.encode() if cache_path else None
        rc = self._lib.b200sa_plan_autotune(self.handle, path, _lib.TUNE_FORCE if force else 0,
                                            rep, cap, err, len(err))
        _lib.check(rc, err)
        return [rep[i].as_dict() for i in range(min(rc, cap))]

    def bucket_report(self) -> list[dict]:
        """Per size bucket of the last persistent or graph run: reads,
        attempts, flips, passes, the state-access model bytes, the launch's
        device time (ms) and its shape.  Waits for the run."""
        cap = 64
        rep = (_lib.BucketReport * cap)()
        err = _lib.errbuf()
        rc = self._lib.b200sa_plan_bucket_report(self.handle, rep, cap, err, len(err))
        _lib.check(rc, err)
        return [rep[i].as_dict() for i in range(min(rc, cap))]

    def close(self):
        if self.handle:
            self._lib.b200sa_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
