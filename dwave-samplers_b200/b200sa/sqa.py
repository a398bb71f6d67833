"""The reference's SQA samplers on the B200.

* :func:`simulated_annealing` -- rotor-model annealing, with the signature and
  return values of ``dwave/samplers/sqa/rotormc_annealing.pyx:54-236``
  (``b200sa_rotor_anneal``).
* :func:`path_annealing` -- path-integral Monte Carlo annealing, with the
  signature and return values of ``dwave/samplers/sqa/pimc_annealing.pyx:45-283``
  (``b200sa_path_anneal``).

Every sample equals the reference's (states and energies bit for bit,
statistics, break positions).  Seeding follows
:func:`b200sa.simulated_annealing`: by default sample r is annealed with seed
``seed + r`` (samples run in parallel, each equal to a reference call with
``num_samples=1``); ``rng_stream="shared"`` continues one stream over the
samples exactly as one reference call does.

``interrupt_function`` is called after the samples are annealed, once per
sample in order, and the results are cut after the first sample for which it
returns true.  This matches the reference's returned samples; the reference
instead polls between samples.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

__all__ = ["simulated_annealing", "path_annealing", "PROPOSALS"]

PROPOSALS = {"GibbsNonErgodic": 0, "MetropolisNonErgodic": 1, "MetropolisUniform": 2,
             "MetropolisTF": 3}


def simulated_annealing(num_samples, h, coupler_starts, coupler_ends, coupler_weights,
                        trans_fields, sweeps_per_beta, Hp_field, Hd_field, seed, states_numpy,
                        randomize_order, proposal_acceptance_criteria, schedule_sample_interval,
                        interrupt_function=None, *, rng_stream: str = "per_read",
                        device: int = 0):
    """Returns ``(states, energies, statistics)`` as the reference binding."""
    num_vars = len(h)
    if num_samples * num_vars == 0:  # rotormc_annealing.pyx:161-164
        return (np.empty((num_samples, num_vars), dtype=np.uint8),
                np.zeros(num_samples, dtype=np.double), np.empty(0, dtype=np.uint8))
    if proposal_acceptance_criteria not in PROPOSALS:
        raise ValueError('Unknown proposal_acceptance_criteria')
    if (not isinstance(states_numpy, np.ndarray) or states_numpy.dtype != np.uint8
            or states_numpy.ndim != 2 or not states_numpy.flags.c_contiguous
            or states_numpy.shape != (num_samples, num_vars)):
        raise ValueError("states_numpy must be a C-contiguous uint8 array "
                         "(num_samples, num_variables)")
    if seed < 0:
        raise OverflowError("can't convert negative value to unsigned long long")
    hh = np.ascontiguousarray(h, dtype=np.float64)
    cs = np.ascontiguousarray(coupler_starts, dtype=np.int32)
    ce = np.ascontiguousarray(coupler_ends, dtype=np.int32)
    cw = np.ascontiguousarray(coupler_weights, dtype=np.float64)
    tf = np.ascontiguousarray(trans_fields, dtype=np.float64)
    hp = np.ascontiguousarray(Hp_field, dtype=np.float64)
    hd = np.ascontiguousarray(Hd_field, dtype=np.float64)
    if not (len(cs) == len(ce) == len(cw)):
        raise ValueError("coupler vectors have mismatched lengths")
    if len(tf) != num_vars or len(hd) < len(hp):
        raise ValueError("trans_fields must have num_variables entries and Hd_field at "
                         "least as many as Hp_field")
    if rng_stream == "shared":
        seeds = np.array([seed], dtype=np.uint64)
    elif rng_stream == "per_read":
        with np.errstate(over="ignore"):
            seeds = np.uint64(seed) + np.arange(num_samples, dtype=np.uint64)
    else:
        raise ValueError("rng_stream must be 'per_read' or 'shared'")
    interval = int(schedule_sample_interval)
    if interval:
        stat_size = (num_samples, 1 + (len(hp) - 1) // interval, num_vars)
    else:
        stat_size = (num_samples, 1, 1)  # as the reference allocates it
    statistics = np.zeros(stat_size, dtype=np.uint8)
    energies = np.empty(num_samples, dtype=np.float64)
    near = ctypes.c_int64(0)
    err = _lib.errbuf()
    rc = _lib.load().b200sa_rotor_anneal(
        num_vars, hh.ctypes.data, len(cw), cs.ctypes.data, ce.ctypes.data, cw.ctypes.data,
        tf.ctypes.data, int(num_samples), states_numpy.ctypes.data, energies.ctypes.data,
        int(sweeps_per_beta), len(hp), hp.ctypes.data, hd.ctypes.data, seeds.ctypes.data,
        len(seeds), 1 if randomize_order else 0, PROPOSALS[proposal_acceptance_criteria],
        statistics.ctypes.data if interval else None, interval, int(device),
        ctypes.byref(near), err, len(err))
    _lib.check(rc, err)
    num = num_samples
    if interrupt_function is not None:
        for k in range(num_samples):
            if interrupt_function():
                num = k + 1
                break
    return states_numpy[:num], energies[:num], statistics[:num]


def _breaks_capacity(hd) -> int:
    """Default bound on the breaks of a variable and the proposals of one
    update: more than ten standard deviations above Poisson(max Gamma)."""
    finite = np.abs(hd[np.isfinite(hd)])
    g = float(finite.max()) if finite.size else 0.0
    return int(min(1e6, np.ceil((g + 10.0 * np.sqrt(g) + 16.0) / 4.0) * 4.0))


def path_annealing(num_samples, h, coupler_starts, coupler_ends, coupler_weights,
                   sweeps_per_beta, Hp_field, Hd_field, Gamma, chain_coupler_strength,
                   qubits_per_chain, qubits_per_update, seed, states_numpy, project_inputs,
                   project_outputs, num_breaks_numpy, breaks_in_numpy, breaks_buffer_out_numpy,
                   schedule_sample_interval, interrupt_function=None, *,
                   rng_stream: str = "per_read", break_capacity: int = 0, device: int = 0):
    """Returns ``(states, energies, statistics, num_breaks, breaks_buffer_out)``
    as the reference binding.

    ``Gamma`` is accepted and unused, as in the reference (the schedule sets
    the transverse field of every step).  The schedule has ``len(Hd_field)``
    steps (the reference's loop); ``Hp_field`` must have at least as many
    entries.  ``break_capacity`` bounds the breaks of a variable and the
    proposals of one update on the device; 0 picks one from the largest
    transverse field and doubles it (up to four times) when it is exceeded.
    """
    num_vars = len(h)
    if num_samples * num_vars == 0:  # pimc_annealing.pyx:185-191
        return (np.empty((num_samples, num_vars), dtype=np.int8),
                np.zeros(num_samples, dtype=np.double), np.empty(0, dtype=np.int8),
                np.empty((num_samples, num_vars), dtype=np.int8), np.empty(0, dtype=np.int8))

    def c_array(a, dtype, ndim, name):
        if (not isinstance(a, np.ndarray) or a.dtype != dtype or a.ndim != ndim
                or not a.flags.c_contiguous):
            raise ValueError(f"{name} must be a C-contiguous {ndim}D {np.dtype(dtype).name} array")
        return a

    c_array(states_numpy, np.int8, 2, "states_numpy")
    c_array(num_breaks_numpy, np.intc, 2, "num_breaks_numpy")
    c_array(breaks_in_numpy, np.intc, 1, "breaks_in_numpy")
    c_array(breaks_buffer_out_numpy, np.intc, 1, "breaks_buffer_out_numpy")
    if states_numpy.shape != (num_samples, num_vars) or num_breaks_numpy.shape != states_numpy.shape:
        raise ValueError("states_numpy and num_breaks_numpy must have shape "
                         "(num_samples, num_variables)")
    if not 0 <= seed < 2**32:
        raise OverflowError("seed must fit an unsigned 32-bit integer")
    hh = np.ascontiguousarray(h, dtype=np.float64)
    cs = np.ascontiguousarray(coupler_starts, dtype=np.int32)
    ce = np.ascontiguousarray(coupler_ends, dtype=np.int32)
    cw = np.ascontiguousarray(coupler_weights, dtype=np.float64)
    hd = np.ascontiguousarray(Hd_field, dtype=np.float64)
    hp = np.ascontiguousarray(Hp_field, dtype=np.float64)
    if not (len(cs) == len(ce) == len(cw)):
        raise ValueError("coupler vectors have mismatched lengths")
    if len(hp) < len(hd):
        raise ValueError("Hp_field must have at least as many entries as Hd_field")
    hp = np.ascontiguousarray(hp[:len(hd)])
    if rng_stream == "shared":
        seeds = np.array([seed], dtype=np.uint32)
    elif rng_stream == "per_read":
        seeds = ((int(seed) + np.arange(num_samples, dtype=np.uint64)) % 2**32).astype(np.uint32)
    else:
        raise ValueError("rng_stream must be 'per_read' or 'shared'")
    interval = int(schedule_sample_interval)
    if interval:
        stat_size = (num_samples, 1 + (len(hd) - 1) // interval, num_vars)
    else:
        stat_size = (num_samples, 1, 1)  # as the reference allocates it
    statistics = np.zeros(stat_size, dtype=np.int8)
    energies = np.empty(num_samples, dtype=np.float64)
    capacity = int(break_capacity) or _breaks_capacity(hd)
    retries = 0 if break_capacity else 4
    while True:
        near = ctypes.c_int64(0)
        err = _lib.errbuf()
        rc = _lib.load().b200sa_path_anneal(
            num_vars, hh.ctypes.data, len(cw), cs.ctypes.data, ce.ctypes.data, cw.ctypes.data,
            int(num_samples), states_numpy.ctypes.data, energies.ctypes.data,
            int(sweeps_per_beta), len(hd), hp.ctypes.data, hd.ctypes.data,
            float(chain_coupler_strength), int(qubits_per_chain), int(qubits_per_update),
            seeds.ctypes.data, len(seeds), 1 if project_inputs else 0,
            1 if project_outputs else 0, num_breaks_numpy.ctypes.data,
            breaks_in_numpy.ctypes.data, len(breaks_in_numpy),
            breaks_buffer_out_numpy.ctypes.data, len(breaks_buffer_out_numpy),
            statistics.ctypes.data if interval else None, interval, capacity, int(device),
            ctypes.byref(near), err, len(err))
        if rc == _lib.ERANGE and retries:
            retries -= 1
            capacity *= 2
            continue
        _lib.check(rc, err)
        break
    num = num_samples
    if interrupt_function is not None:
        for k in range(num_samples):
            if interrupt_function():
                num = k + 1
                break
    return (states_numpy[:num], energies[:num], statistics[:num], num_breaks_numpy[:num],
            breaks_buffer_out_numpy)
