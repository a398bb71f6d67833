"""Steepest descent on the B200: the drop-in for ``dwave.samplers.greedy``.

* :func:`steepest_gradient_descent` has the signature and return values of
  the reference's Cython binding (``dwave/samplers/greedy/descent.pyx:22-112``)
  and calls ``b200sa_steepest_descent``; every sample equals the reference's
  result (states, energies bit for bit, step counts).
* :class:`SteepestDescentSolver` mirrors the reference's
  ``SteepestDescentSolver.sample`` (``greedy/sampler.py:137-318``:
  ``num_reads``, ``initial_states``, ``initial_states_generator``, ``seed``,
  ``large_sparse_opt``) without dimod, in the manner of
  :class:`b200sa.sampler.SimulatedAnnealingSampler`.
* :class:`SteepestDescentComposite` runs a child sampler and then descends
  from its samples (``greedy/composite.py:60-82``): annealing followed by
  descent to the nearest local minima.

Descent from a state with a self-loop of positive weight can cycle for ever
in the reference; here each sample stops after ``max_steps`` flips and a
``TimeoutError`` is raised.
"""
from __future__ import annotations

import ctypes
from numbers import Integral
from time import perf_counter_ns
from typing import Optional

import numpy as np

from . import _lib
from .sampler import SampleSet, SimulatedAnnealingSampler, _as_problem, dimod

__all__ = ["steepest_gradient_descent", "SteepestDescentSolver", "SteepestDescentSampler",
           "SteepestDescentComposite"]


def steepest_gradient_descent(num_samples, linear_biases, coupler_starts, coupler_ends,
                              coupler_weights, states_numpy, large_sparse_opt=False, *,
                              max_steps: int = 0, device: int = 0):
    """Steepest descent from every row of ``states_numpy`` (C-contiguous int8,
    num_samples x num_variables, overwritten).  Returns ``(states_numpy,
    energies, num_steps)`` as the reference binding does."""
    num_vars = len(linear_biases)
    if num_samples == 0 or num_vars == 0:  # descent.pyx:83-88
        states = np.empty((num_samples, num_vars), dtype=np.int8)
        return states, np.zeros(num_samples, dtype=np.double), np.zeros(num_samples, dtype=np.uint32)
    if (not isinstance(states_numpy, np.ndarray) or states_numpy.dtype != np.int8
            or states_numpy.ndim != 2 or not states_numpy.flags.c_contiguous):
        raise ValueError("states_numpy must be a C-contiguous 2D int8 numpy array")
    if states_numpy.shape != (num_samples, num_vars):
        raise ValueError("states_numpy must have shape (num_samples, num_variables)")
    h = np.ascontiguousarray(linear_biases, dtype=np.float64)
    cs = np.ascontiguousarray(coupler_starts, dtype=np.int32)
    ce = np.ascontiguousarray(coupler_ends, dtype=np.int32)
    cw = np.ascontiguousarray(coupler_weights, dtype=np.float64)
    if not (len(cs) == len(ce) == len(cw)):
        raise ValueError("coupler vectors have mismatched lengths")
    energies = np.empty(num_samples, dtype=np.float64)
    num_steps = np.empty(num_samples, dtype=np.uint32)
    err = _lib.errbuf()
    rc = _lib.load().b200sa_steepest_descent(
        num_vars, h.ctypes.data, len(cw), cs.ctypes.data, ce.ctypes.data, cw.ctypes.data,
        int(num_samples), states_numpy.ctypes.data, energies.ctypes.data, num_steps.ctypes.data,
        1 if large_sparse_opt else 0, int(max_steps), int(device), err, len(err))
    _lib.check(rc, err)
    return states_numpy, energies, num_steps


def _rows_from_sampleset(sampleset, problem):
    """Initial states from a sample set (ours or dimod's), in the problem's
    variable order."""
    variables = list(sampleset.variables)
    index = {x: i for i, x in enumerate(variables)}
    cols = [index[x] for x in problem.variables]
    return np.asarray(sampleset.record.sample)[:, cols]


class SteepestDescentSolver:
    """Steepest descent with the reference solver's interface."""

    def __init__(self, device: int = 0):
        self.device = device
        self.parameters = {'num_reads': [], 'initial_states': [],
                           'initial_states_generator': ['initial_states_generators'],
                           'seed': [], 'large_sparse_opt': ['large_sparse_opt_values']}
        self.properties = {'initial_states_generators': ('none', 'tile', 'random'),
                           'large_sparse_opt_values': (True, False)}

    sample_ising = SimulatedAnnealingSampler.sample_ising
    sample_qubo = SimulatedAnnealingSampler.sample_qubo

    def sample(self, bqm, num_reads: Optional[int] = None, initial_states=None,
               initial_states_generator: str = "random", seed: Optional[int] = None,
               large_sparse_opt: bool = False, **kwargs):
        timestamp_preprocess = perf_counter_ns()
        if kwargs:
            raise TypeError("unknown parameter(s): " + ", ".join(sorted(kwargs)))
        problem = _as_problem(bqm)
        if seed is None:
            seed = np.random.randint(2**31)
        elif not isinstance(seed, Integral):
            raise TypeError("'seed' should be None or an integer between 0 and 2^32 - 1")
        elif not (0 <= seed < 2**32):
            raise ValueError("'seed' should be an integer between 0 and 2^32 - 1")
        if initial_states is not None and hasattr(initial_states, "record"):
            initial_states = _rows_from_sampleset(initial_states, problem)
        init = SimulatedAnnealingSampler._initial_states(
            problem, num_reads, initial_states, initial_states_generator, seed)
        timestamp_sample = perf_counter_ns()
        samples, energies, num_steps = steepest_gradient_descent(
            init.shape[0], problem.h, problem.u, problem.v, problem.J, init,
            large_sparse_opt, device=self.device)
        timestamp_postprocess = perf_counter_ns()
        if problem.vartype == "BINARY":
            out = ((np.asarray(samples) + 1) // 2).astype(np.int8)
        else:
            out = np.asarray(samples)
        energies = energies + problem.offset
        if dimod is not None:
            response = dimod.SampleSet.from_samples(
                (out, problem.variables), energy=energies, num_steps=num_steps,
                vartype=dimod.BINARY if problem.vartype == "BINARY" else dimod.SPIN)
        else:
            response = SampleSet(out, problem.variables, energies, {}, problem.vartype)
            response.num_steps = num_steps
        response.info.update(dict(timing=dict(
            preprocessing_ns=timestamp_sample - timestamp_preprocess,
            sampling_ns=timestamp_postprocess - timestamp_sample,
            postprocessing_ns=perf_counter_ns() - timestamp_postprocess)))
        return response


SteepestDescentSampler = SteepestDescentSolver


class SteepestDescentComposite:
    """Runs ``child_sampler``, then steepest descent from its samples."""

    def __init__(self, child_sampler, device: int = 0):
        self.children = [child_sampler]
        self.device = device

    @property
    def child(self):
        return self.children[0]

    @property
    def parameters(self):
        return self.child.parameters.copy()

    @property
    def properties(self):
        return {'child_properties': self.child.properties.copy()}

    def sample(self, bqm, **parameters):
        sampleset = self.child.sample(bqm, **parameters)
        return SteepestDescentSolver(self.device).sample(bqm, initial_states=sampleset)

    sample_ising = SimulatedAnnealingSampler.sample_ising
    sample_qubo = SimulatedAnnealingSampler.sample_qubo
