"""Drop-in for the reference's Cython binding.

``simulated_annealing`` keeps the signature, argument meaning, return value
and error behaviour of ``dwave/samplers/sa/simulated_annealing.pyx:45-197``
(dwave-samplers 1.8.0), and runs the sweep on the B200 through the C ABI.

Seeding.  The reference seeds one xorshift128+ stream per call and continues
it across reads (``cpu_sa.cpp:283-284``), which forces reads to run one after
another.  Here, by default (``rng_stream="per_read"``), read ``r`` is seeded
with ``seed + r`` (mod 2**64), or with ``seeds[r]`` when given, and equals the
reference run with ``num_samples=1`` and that seed, bit for bit.
``rng_stream="shared"`` reproduces the reference's multi-read stream exactly
(reads then run one after another on one warp).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

__all__ = ["simulated_annealing", "per_read_seeds"]


def per_read_seeds(seed: int, num_reads: int) -> np.ndarray:
    """Seeds ``seed + r`` (mod 2**64) for reads ``r = 0 .. num_reads-1``."""
    base = np.uint64(int(seed) % (1 << 64))
    with np.errstate(over="ignore"):
        return base + np.arange(num_reads, dtype=np.uint64)


def _as_c_array(x, dtype, name):
    try:
        return np.ascontiguousarray(np.asarray(x, dtype=dtype))
    except (TypeError, ValueError) as e:
        raise TypeError(f"{name}: {e}") from None


def simulated_annealing(num_samples, h, coupler_starts, coupler_ends,
                        coupler_weights, sweeps_per_beta, beta_schedule, seed,
                        states_numpy, randomize_order=False,
                        proposal_acceptance_criteria="Metropolis",
                        interrupt_function=None, *, seeds=None,
                        rng_stream="per_read", device=0, stats=None):
    """Anneal ``states_numpy`` in place and return ``(samples, energies)``.

    Parameters follow ``simulated_annealing.pyx:45-130``; the keyword-only
    extras are ``seeds`` (one uint64 seed per read), ``rng_stream``
    ("per_read" or "shared"), ``device`` and ``stats`` (a dict that receives
    the run's counters: attempts, flips, near_ties, passes, kernel_ms, and
    ``near_ties_per_read``, one count per completed read: a read with a
    nonzero count made an exp() decision so close to its threshold that the
    host libm could have decided it differently; every other read is
    bit-exact with the reference).

    Returns views ``states_numpy[:num]`` and ``energies[:num]``, ``num`` being
    the number of reads completed (fewer when ``interrupt_function`` stops the
    run), as ``simulated_annealing.pyx:189``.
    """
    num_vars = len(h)

    # simulated_annealing.pyx:134-136
    if num_samples * num_vars == 0:
        annealed_states = np.empty((num_samples, num_vars), dtype=np.int8)
        return annealed_states, np.zeros(num_samples, dtype=np.double)

    # The Cython signature types states_numpy as int8[:, ::1].
    if not isinstance(states_numpy, np.ndarray):
        raise TypeError("states_numpy must be a numpy.ndarray")
    if states_numpy.dtype != np.int8:
        raise ValueError(
            f"Buffer dtype mismatch, expected 'int8_t' but got '{states_numpy.dtype}'")
    if states_numpy.ndim != 2:
        raise ValueError(f"Buffer has wrong number of dimensions (expected 2, got {states_numpy.ndim})")
    if not states_numpy.flags.c_contiguous:
        raise ValueError("ndarray is not C-contiguous")
    num_samples = int(num_samples)
    if states_numpy.shape[0] < num_samples or states_numpy.shape[1] != num_vars:
        raise ValueError(
            f"states_numpy has shape {states_numpy.shape}; expected ({num_samples}, {num_vars})")

    hh = _as_c_array(h, np.float64, "h")
    cs = _as_c_array(coupler_starts, np.int32, "coupler_starts")
    ce = _as_c_array(coupler_ends, np.int32, "coupler_ends")
    cw = _as_c_array(coupler_weights, np.float64, "coupler_weights")
    if not (cs.shape[0] == ce.shape[0] == cw.shape[0]):
        # cpu_sa.cpp:276-279 throws "coupler vectors have mismatched lengths"
        raise ValueError("coupler vectors have mismatched lengths")
    betas = _as_c_array(beta_schedule, np.float64, "beta_schedule")
    sweeps_per_beta = int(sweeps_per_beta)

    # simulated_annealing.pyx:152: `cdef unsigned long long _seed = seed`
    seed = int(seed)
    if seed < 0:
        raise OverflowError("can't convert negative value to unsigned PY_LONG_LONG")
    if seed >= 1 << 64:
        raise OverflowError("Python int too large to convert to C unsigned long long")

    varorder = _lib.RANDOM if randomize_order else _lib.SEQUENTIAL
    crit = proposal_acceptance_criteria.lower()
    if crit == "gibbs":
        proposal = _lib.GIBBS
    elif crit == "metropolis":
        proposal = _lib.METROPOLIS
    else:
        raise ValueError(f"Unknown proposal_acceptance_criteria: {proposal_acceptance_criteria}")

    if rng_stream == "shared":
        if seeds is not None:
            raise ValueError("seeds cannot be combined with rng_stream='shared'")
        seed_arr = np.array([seed], dtype=np.uint64)
    elif rng_stream == "per_read":
        if seeds is None:
            seed_arr = per_read_seeds(seed, num_samples)
        else:
            seed_arr = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64))
            if seed_arr.shape != (num_samples,):
                raise ValueError("seeds must have one entry per read")
    else:
        raise ValueError("rng_stream must be 'per_read' or 'shared'")

    energies = np.empty(num_samples, dtype=np.float64)

    # simulated_annealing.pyx:192-197: an exception in the callback interrupts.
    cb = _lib.INTERRUPT_FN()
    if interrupt_function is not None:
        def _poll(_ctx):
            try:
                return 1 if interrupt_function() else 0
            except Exception:
                return 1
        cb = _lib.INTERRUPT_FN(_poll)

    L = _lib.load()
    st = _lib.Stats()
    read_ties = np.zeros(num_samples, dtype=np.uint32)
    st.read_near_ties = read_ties.ctypes.data
    err = _lib.errbuf()
    rc = L.b200sa_sample(
        num_vars, hh.ctypes.data, cw.shape[0], cs.ctypes.data, ce.ctypes.data,
        cw.ctypes.data, num_samples, states_numpy.ctypes.data, energies.ctypes.data,
        sweeps_per_beta, betas.shape[0], betas.ctypes.data, seed_arr.ctypes.data,
        seed_arr.shape[0], varorder, proposal, cb, None, int(device),
        ctypes.byref(st), err, len(err))
    num = _lib.check(rc, err)
    if stats is not None:
        stats.update(st.as_dict())
        stats["near_ties_per_read"] = read_ties[:num]
    return states_numpy[:num], energies[:num]
