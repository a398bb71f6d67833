"""ctypes binding of libb200sa.so (C ABI in include/b200sa.h).

The library is built in-tree by ``dwave-samplers_b200/build.py``.  There is no
fallback: if the library is missing or cannot load, every sampling call
raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libb200sa.so")

OK = 0
EINVAL = -1
ECUDA = -2
ENOMEM = -3
ENODEV = -4
ETIMEOUT = -5
ERANGE = -6

GIBBS = 0
METROPOLIS = 1
SEQUENTIAL = 0
RANDOM = 1

MODE_PERSISTENT = 0
MODE_PLAIN = 1
MODE_GRAPH = 2
MODE_PLAIN_TUNED = 3
TUNE_FORCE = 1

EXPORTS = (
    "b200sa_sample",
    "b200sa_sample_batch",
    "b200sa_plan_create",
    "b200sa_plan_layout",
    "b200sa_plan_run",
    "b200sa_plan_destroy",
    "b200sa_version",
    "b200sa_check_acceptance",
    "b200sa_sample_noalloc",
    "b200sa_edge_moments",
    "b200sa_random_states",
    "b200sa_plan_set_weights",
    "b200sa_plan_set_weights_device",
    "b200sa_plan_autotune",
    "b200sa_plan_bucket_report",
    "b200sa_steepest_descent",
    "b200sa_rotor_anneal",
    "b200sa_path_anneal",
)


class Stats(ctypes.Structure):
    _fields_ = [
        ("reads", ctypes.c_int64),
        ("attempts", ctypes.c_int64),
        ("flips", ctypes.c_int64),
        ("near_ties", ctypes.c_int64),
        ("passes", ctypes.c_int64),
        ("kernel_ms", ctypes.c_double),
        ("launches", ctypes.c_int64),
        ("read_near_ties", ctypes.c_void_p),  # input: optional per-read uint32 array
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_
                if name != "read_near_ties"}


class Problem(ctypes.Structure):
    _fields_ = [
        ("num_vars", ctypes.c_int32),
        ("h", ctypes.c_void_p),
        ("num_couplers", ctypes.c_int64),
        ("coupler_starts", ctypes.c_void_p),
        ("coupler_ends", ctypes.c_void_p),
        ("coupler_weights", ctypes.c_void_p),
        ("num_reads", ctypes.c_int32),
        ("states", ctypes.c_void_p),
        ("energies", ctypes.c_void_p),
        ("sweeps_per_beta", ctypes.c_int32),
        ("num_betas", ctypes.c_int32),
        ("beta_schedule", ctypes.c_void_p),
        ("seeds", ctypes.c_void_p),
        ("varorder", ctypes.c_int32),
        ("proposal", ctypes.c_int32),
    ]


class MomentsProblem(ctypes.Structure):
    _fields_ = [
        ("num_vars", ctypes.c_int32),
        ("num_couplers", ctypes.c_int64),
        ("num_reads", ctypes.c_int32),
        ("states", ctypes.c_void_p),
        ("coupler_starts", ctypes.c_void_p),
        ("coupler_ends", ctypes.c_void_p),
        ("sum_s", ctypes.c_void_p),
        ("sum_ss", ctypes.c_void_p),
    ]


class TuneEntry(ctypes.Structure):
    _fields_ = [
        ("bucket", ctypes.c_int32),
        ("kind", ctypes.c_int32),
        ("max_n", ctypes.c_int32),
        ("items", ctypes.c_int64),
        ("staging", ctypes.c_int32),
        ("warps_per_cta", ctypes.c_int32),
        ("ctas_per_sm", ctypes.c_int32),
        ("registers", ctypes.c_int32),
        ("attempts_per_s", ctypes.c_double),
        ("from_cache", ctypes.c_int32),
        ("candidates", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BucketReport(ctypes.Structure):
    _fields_ = [
        ("bucket", ctypes.c_int32),
        ("kind", ctypes.c_int32),
        ("max_n", ctypes.c_int32),
        ("reads", ctypes.c_int64),
        ("attempts", ctypes.c_int64),
        ("flips", ctypes.c_int64),
        ("passes", ctypes.c_int64),
        ("model_bytes", ctypes.c_double),
        ("ms", ctypes.c_double),
        ("staging", ctypes.c_int32),
        ("warps_per_cta", ctypes.c_int32),
        ("grid", ctypes.c_int32),
        ("registers", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


INTERRUPT_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p)

_lib = None


def load() -> ctypes.CDLL:
    """Load the CUDA library, failing loudly when it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is not built; run `python dwave-samplers_b200/build.py`")
    L = ctypes.CDLL(LIB_PATH)
    c = ctypes
    L.b200sa_sample.restype = c.c_int
    L.b200sa_sample.argtypes = [
        c.c_int32, c.c_void_p, c.c_int64, c.c_void_p, c.c_void_p, c.c_void_p,
        c.c_int32, c.c_void_p, c.c_void_p, c.c_int32, c.c_int32, c.c_void_p,
        c.c_void_p, c.c_int32, c.c_int32, c.c_int32, INTERRUPT_FN, c.c_void_p,
        c.c_int32, c.POINTER(Stats), c.c_char_p, c.c_size_t]
    L.b200sa_sample_batch.restype = c.c_int
    L.b200sa_sample_batch.argtypes = [
        c.POINTER(Problem), c.c_int32, c.c_int32, c.c_int32, c.POINTER(Stats),
        c.c_char_p, c.c_size_t]
    L.b200sa_plan_create.restype = c.c_int
    L.b200sa_plan_create.argtypes = [
        c.POINTER(Problem), c.c_int32, c.c_int32, c.POINTER(c.c_void_p),
        c.c_char_p, c.c_size_t]
    L.b200sa_plan_layout.restype = c.c_int
    L.b200sa_plan_layout.argtypes = [c.c_void_p, c.c_void_p, c.c_void_p]
    L.b200sa_plan_run.restype = c.c_int
    L.b200sa_plan_run.argtypes = [
        c.c_void_p, c.c_int32, c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p,
        c.c_void_p, c.c_int32, c.POINTER(Stats), c.c_char_p, c.c_size_t]
    L.b200sa_plan_destroy.restype = c.c_int
    L.b200sa_plan_destroy.argtypes = [c.c_void_p]
    L.b200sa_check_acceptance.restype = c.c_int
    L.b200sa_check_acceptance.argtypes = [c.c_int64, c.c_uint64, c.c_int32, c.c_void_p,
                                          c.c_char_p, c.c_size_t]
    L.b200sa_sample_noalloc.restype = c.c_int
    L.b200sa_sample_noalloc.argtypes = [
        c.c_int32, c.c_void_p, c.c_int64, c.c_void_p, c.c_void_p, c.c_void_p, c.c_int32,
        c.c_void_p, c.c_void_p, c.c_void_p, c.c_int32, c.c_int32, c.c_void_p, c.c_void_p,
        c.c_int32, c.c_int32, c.c_int32, c.c_void_p, c.c_void_p, c.POINTER(c.c_int64),
        c.c_char_p, c.c_size_t]
    L.b200sa_edge_moments.restype = c.c_int
    L.b200sa_edge_moments.argtypes = [c.POINTER(MomentsProblem), c.c_int32, c.c_int32,
                                      c.c_void_p, c.c_char_p, c.c_size_t]
    L.b200sa_random_states.restype = c.c_int
    L.b200sa_random_states.argtypes = [c.c_uint64, c.c_uint64, c.c_int64, c.c_int64, c.c_int32,
                                       c.c_void_p, c.c_int32, c.c_void_p, c.c_char_p, c.c_size_t]
    L.b200sa_plan_set_weights.restype = c.c_int
    L.b200sa_plan_set_weights.argtypes = [c.c_void_p, c.c_int32, c.c_void_p, c.c_void_p,
                                          c.c_char_p, c.c_size_t]
    L.b200sa_plan_set_weights_device.restype = c.c_int
    L.b200sa_plan_set_weights_device.argtypes = [c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p,
                                                 c.c_char_p, c.c_size_t]
    L.b200sa_plan_autotune.restype = c.c_int
    L.b200sa_plan_autotune.argtypes = [c.c_void_p, c.c_char_p, c.c_int32, c.POINTER(TuneEntry),
                                       c.c_int32, c.c_char_p, c.c_size_t]
    L.b200sa_plan_bucket_report.restype = c.c_int
    L.b200sa_plan_bucket_report.argtypes = [c.c_void_p, c.POINTER(BucketReport), c.c_int32,
                                            c.c_char_p, c.c_size_t]
    L.b200sa_steepest_descent.restype = c.c_int
    L.b200sa_steepest_descent.argtypes = [
        c.c_int32, c.c_void_p, c.c_int64, c.c_void_p, c.c_void_p, c.c_void_p, c.c_int32,
        c.c_void_p, c.c_void_p, c.c_void_p, c.c_int32, c.c_uint32, c.c_int32, c.c_char_p,
        c.c_size_t]
    L.b200sa_rotor_anneal.restype = c.c_int
    L.b200sa_rotor_anneal.argtypes = [
        c.c_int32, c.c_void_p, c.c_int64, c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p,
        c.c_int32, c.c_void_p, c.c_void_p, c.c_int32, c.c_int32, c.c_void_p, c.c_void_p,
        c.c_void_p, c.c_int32, c.c_int32, c.c_int32, c.c_void_p, c.c_int32, c.c_int32,
        c.POINTER(c.c_int64), c.c_char_p, c.c_size_t]
    L.b200sa_path_anneal.restype = c.c_int
    L.b200sa_path_anneal.argtypes = [
        c.c_int32, c.c_void_p, c.c_int64, c.c_void_p, c.c_void_p, c.c_void_p, c.c_int32,
        c.c_void_p, c.c_void_p, c.c_int32, c.c_int32, c.c_void_p, c.c_void_p, c.c_double,
        c.c_int32, c.c_int32, c.c_void_p, c.c_int32, c.c_int32, c.c_int32, c.c_void_p,
        c.c_void_p, c.c_int64, c.c_void_p, c.c_int64, c.c_void_p, c.c_int32, c.c_int32,
        c.c_int32, c.POINTER(c.c_int64), c.c_char_p, c.c_size_t]
    L.b200sa_version.restype = c.c_char_p
    L.b200sa_version.argtypes = []
    _lib = L
    return L


class CapacityError(RuntimeError):
    """A fixed device capacity (break lists of path-integral annealing) was
    exceeded; calling again with a larger capacity succeeds."""


def check(rc: int, err: ctypes.Array) -> int:
    """Map a negative return code to the matching Python exception."""
    if rc >= 0:
        return rc
    msg = err.value.decode(errors="replace") if err is not None else ""
    if rc == EINVAL:
        raise ValueError(msg or "invalid argument")
    if rc == ENOMEM:
        raise MemoryError(msg or "out of memory")
    if rc == ETIMEOUT:
        raise TimeoutError(msg or "device wait timed out")
    if rc == ERANGE:
        raise CapacityError(msg or "capacity exceeded")
    raise RuntimeError(f"b200sa error {rc}: {msg}")


def errbuf() -> ctypes.Array:
    return ctypes.create_string_buffer(512)
