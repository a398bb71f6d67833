"""Rotor-model annealing (the reference's SQA rotor Monte Carlo) on the B200.

:func:`simulated_annealing` has the signature and return values of
``dwave/samplers/sqa/rotormc_annealing.pyx:54-236`` and calls
``b200sa_rotor_anneal``; every sample equals the reference's (states and
energies bit for bit, statistics).  Seeding follows
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

__all__ = ["simulated_annealing", "PROPOSALS"]

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
