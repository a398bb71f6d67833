"""SQA sampler front ends on the B200: ``PathIntegralAnnealingSampler`` and
``RotorModelAnnealingSampler``.

Mirrors ``dwave/samplers/sqa/sampler.py`` (dwave-samplers 1.8.0): the same
``sample`` keyword arguments, validation and error messages, schedule
construction (``Hp_field`` from ``beta_range`` / ``num_sweeps`` /
``beta_schedule_type``, ``Hd_field`` zero by default; ``sampler.py:374-447``
and ``:980-1063``), break-buffer sizing (``:456-494``), the rotor model's
projections between spins and angles (``:941-966``, ``:1103-1109``) and the
``info`` keys.  Unknown keyword arguments are ignored, as there.

As in :mod:`b200sa.sampler` (problems, initial states and the result set work
the same way, with dimod optional): sample r runs with seed ``seed + r`` on
the GPU, where the reference continues one generator over the samples.
"""
from __future__ import annotations

from numbers import Integral
from time import perf_counter_ns
from typing import Optional, Sequence

import numpy as np

from .sampler import SampleSet, SimulatedAnnealingSampler, _as_problem, dimod, ising_beta_range
from .sqa import path_annealing, simulated_annealing as rotor_annealing

__all__ = ["PathIntegralAnnealingSampler", "RotorModelAnnealingSampler"]


def _check_seed(seed):
    """Seed policy of ``sampler.py:326-339``."""
    if seed is None:
        return int(np.random.randint(2**31))
    if not isinstance(seed, Integral):
        raise TypeError("'seed' should be None or an integer between 0 and 2^32 "
                        "- 1: value = {}".format(seed))
    if not (0 <= seed < 2**31):
        raise ValueError("'seed' should be an integer between 0 and 2^32 - 1: "
                         "value = {}".format(seed))
    return int(seed)


def _check_sweeps_per_beta(num_sweeps_per_beta):
    if not isinstance(num_sweeps_per_beta, Integral):
        raise TypeError("'num_sweeps_per_beta' should be a positive integer: value = {}"
                        .format(num_sweeps_per_beta))
    if num_sweeps_per_beta < 1:
        raise ValueError("'num_sweeps_per_beta' should be a positive integer: value = {}"
                         .format(num_sweeps_per_beta))


def build_fields(problem, beta_range, num_sweeps, num_sweeps_per_beta, beta_schedule_type,
                 Hp_field, Hd_field, zero_sweeps_empty=False):
    """The problem (``Hp_field``) and driver (``Hd_field``) schedules of the SQA
    samplers; returns (beta_range, Hp_field, Hd_field).  ``zero_sweeps_empty``:
    ``num_sweeps == 0`` gives an empty schedule (the rotor sampler)."""
    if beta_schedule_type == "custom":
        if Hp_field is None:
            raise ValueError("'Hp_field' must be provided for beta_schedule_type = 'custom': "
                             "value is None")
        try:
            Hp_field = np.array(Hp_field, dtype=float)
        except Exception:
            raise ValueError("Hp_field cannot be case as a numpy array of dtype=float")
        if num_sweeps is not None and num_sweeps != len(Hp_field) * num_sweeps_per_beta:
            raise ValueError("'num_sweeps' should be set to None, or a value consistent with "
                             "'Hp_field' and 'num_sweeps_per_beta' for 'beta_schedule_type' = "
                             "'custom': value = ".format(num_sweeps))
        if beta_range is not None and (beta_range[0] != Hp_field[0]
                                       or beta_range[-1] != Hp_field[-1]):
            raise ValueError("'beta_range' should be set to None, or a value consistent with "
                             "'Hp_field', for 'beta_schedule_type'='custom'.")
        if len(Hp_field) and np.min(Hp_field) < 0:
            raise ValueError("'Hp_field' cannot include negative values.")
    elif zero_sweeps_empty and num_sweeps == 0:
        Hp_field = np.zeros(0)
    else:
        if Hp_field is not None:
            raise ValueError("'Hp_field' must be set to None for 'beta_schedule_type' not "
                             "equal to 'custom'")
        if num_sweeps is None:
            num_sweeps = 100
        num_betas, rem = divmod(num_sweeps, num_sweeps_per_beta)
        if rem > 0 or num_betas < 0:
            raise ValueError("'num_sweeps' must be a positive value divisible by "
                             "'num_sweeps_per_beta'.")
        if beta_range is None:
            beta_range = ising_beta_range(problem.linear, problem.quadratic)
        elif len(beta_range) != 2 or min(beta_range) < 0:
            raise ValueError("'beta_range' should be a 2-tuple, or 2 element list of positive "
                             "numbers. The latter value is the target value.")
        if num_betas == 1:
            Hp_field = np.array([beta_range[-1]], dtype=float)
        elif beta_schedule_type == "linear":
            Hp_field = np.linspace(*beta_range, num=num_betas)
        elif beta_schedule_type == "geometric":
            if min(beta_range) <= 0:
                raise ValueError("'beta_range' must contain non-zero values for "
                                 "'beta_schedule_type' = 'geometric'")
            Hp_field = np.geomspace(*beta_range, num=num_betas)
        else:
            raise ValueError("Beta schedule type {} not implemented".format(beta_schedule_type))
    num_betas = len(Hp_field)
    if Hd_field is None:
        Hd_field = np.zeros(num_betas)
    else:
        Hd_field = np.array(Hd_field, dtype=float)
        if len(Hd_field) < num_betas:
            raise ValueError("Hd_field incompatible with Hp_field")
    return beta_range, np.asarray(Hp_field, dtype=float), Hd_field


def _check_interval(schedule_sample_interval, Hp_field):
    if schedule_sample_interval is None:
        return 0
    if schedule_sample_interval > len(Hp_field) or schedule_sample_interval < 1:
        raise ValueError("schedule_sample_interval is incompatible with Hp_field")
    return int(schedule_sample_interval)


def _response(problem, spins, energies, info, timestamps, json_keys, make_json):
    """Result set in the problem's vartype, with the reference's info keys."""
    if make_json:
        info["beta_range"] = np.array(info["beta_range"]).tolist()
        for k in json_keys:
            if k in info:
                info[k] = np.asarray(info[k]).tolist()
    if problem.vartype == "BINARY":
        out = ((np.asarray(spins) + 1) // 2).astype(np.int8)
    else:
        out = np.asarray(spins)
    energies = energies + problem.offset
    if dimod is not None:
        response = dimod.SampleSet.from_samples(
            (out, problem.variables), energy=energies, info=info,
            vartype=dimod.BINARY if problem.vartype == "BINARY" else dimod.SPIN)
    else:
        response = SampleSet(out, problem.variables, energies, info, problem.vartype)
    t0, t1, t2 = timestamps
    response.info.update(dict(timing=dict(preprocessing_ns=t1 - t0, sampling_ns=t2 - t1,
                                          postprocessing_ns=perf_counter_ns() - t2)))
    return response


class _SQASampler:
    def __init__(self, device: int = 0):
        self.device = device
        self.parameters = {
            "beta_range": [], "num_reads": [], "num_sweeps": [], "num_sweeps_per_beta": [],
            "beta_schedule_type": ["beta_schedule_options"], "seed": [],
            "interrupt_function": [], "initial_states": [], "initial_states_generator": [],
        }
        self.properties = {"beta_schedule_options": ("linear", "geometric", "custom")}

    sample_ising = SimulatedAnnealingSampler.sample_ising
    sample_qubo = SimulatedAnnealingSampler.sample_qubo


class PathIntegralAnnealingSampler(_SQASampler):
    """Path-integral Monte Carlo annealing of a binary quadratic model
    (``sqa/sampler.py:33-569``) on :func:`b200sa.sqa.path_annealing`."""

    def sample(self, bqm, *, beta_range=None, num_reads: Optional[int] = None,
               num_sweeps: Optional[int] = None, num_sweeps_per_beta: int = 1,
               beta_schedule_type: str = "geometric", seed: Optional[int] = None,
               Hp_field: Optional[Sequence[float]] = None,
               Hd_field: Optional[Sequence[float]] = None, Gamma: float = 1,
               chain_coupler_strength: float = 1, qubits_per_chain: int = 1,
               qubits_per_update: int = 1, initial_states=None,
               initial_states_generator: str = "random",
               make_info_json_serializable: bool = False, project_states=(True, True),
               num_breaks: Optional[np.ndarray] = None, breaks_in: Optional[np.ndarray] = None,
               breaks_buffer_out: Optional[np.ndarray] = None,
               schedule_sample_interval: Optional[int] = None, interrupt_function=None,
               **kwargs):
        t0 = perf_counter_ns()
        problem = _as_problem(bqm)
        seed = _check_seed(seed)
        init = SimulatedAnnealingSampler._initial_states(
            problem, num_reads, initial_states, initial_states_generator, seed)
        num_reads = init.shape[0]
        n = len(problem.variables)
        if interrupt_function and not callable(interrupt_function):
            raise TypeError("'interrupt_function' should be a callable")
        _check_sweeps_per_beta(num_sweeps_per_beta)
        beta_range, Hp_field, Hd_field = build_fields(
            problem, beta_range, num_sweeps, num_sweeps_per_beta, beta_schedule_type,
            Hp_field, Hd_field)
        num_betas = len(Hp_field)
        # Break buffers, sampler.py:456-494.
        if num_breaks is None:
            num_breaks = np.zeros(shape=init.shape, dtype=np.intc)
        elif num_breaks.shape != init.shape:
            raise ValueError("Path integral initialization is inconsistent")
        if breaks_in is None:
            breaks_in = np.zeros(max(1, int(np.sum(num_breaks))))
        breaks_in = np.ascontiguousarray(breaks_in, dtype=np.intc)
        if breaks_buffer_out is None:
            if not project_states[1]:
                patterns = num_reads * n
                if num_betas > 0:
                    need = int((1 + Hd_field[-1]) * (patterns + np.log(patterns)) + 1000)
                else:
                    need = int(np.sum(num_breaks))
            else:
                need = 1
            breaks_buffer_out = np.zeros(need, dtype=np.intc)
        breaks_buffer_out = np.ascontiguousarray(breaks_buffer_out, dtype=np.intc)
        num_breaks = np.ascontiguousarray(num_breaks, dtype=np.intc)
        interval = _check_interval(schedule_sample_interval, Hp_field)
        t1 = perf_counter_ns()
        samples, energies, statistics, num_breaks, breaks_buffer_out = path_annealing(
            num_reads, problem.h, problem.u, problem.v, problem.J, num_sweeps_per_beta,
            Hp_field, Hd_field, Gamma, chain_coupler_strength, qubits_per_chain,
            qubits_per_update, seed, init, project_states[0], project_states[1], num_breaks,
            breaks_in, breaks_buffer_out, interval, interrupt_function, device=self.device)
        t2 = perf_counter_ns()
        info = {"beta_range": beta_range, "beta_schedule_type": beta_schedule_type}
        if interval > 0:
            info["statistics"] = statistics
        if not project_states[1]:
            info["num_breaks"] = num_breaks
            total = int(np.sum(num_breaks))
            if breaks_buffer_out.size >= total:
                info["complete_break_specification"] = True
                info["break_positions"] = breaks_buffer_out[:total]
            else:
                info["complete_break_specification"] = False
                info["break_positions"] = breaks_buffer_out
        return _response(problem, samples, energies, info, (t0, t1, t2),
                         ("statistics", "num_breaks", "break_positions"),
                         make_info_json_serializable)


class RotorModelAnnealingSampler(_SQASampler):
    """Rotor-model annealing of a binary quadratic model (``sqa/sampler.py:572-1132``)
    on :func:`b200sa.sqa.simulated_annealing`.  Spins map to angles 0 (+1) and
    128 (-1); returned angles are projected to spins with probability
    (1 + cos(theta)) / 2 of +1, from ``numpy.random.default_rng(seed)``; the
    energies are the rotor model's."""

    def sample(self, bqm, *, beta_range=None, num_reads: Optional[int] = None,
               num_sweeps: Optional[int] = None, num_sweeps_per_beta: int = 1,
               beta_schedule_type: str = "geometric", seed: Optional[int] = None,
               Hp_field: Optional[Sequence[float]] = None,
               Hd_field: Optional[Sequence[float]] = None, initial_states=None,
               initial_states_generator: str = "random",
               make_info_json_serializable: bool = False, project_states=(False, True),
               schedule_sample_interval: Optional[int] = None, randomize_order: bool = False,
               proposal_acceptance_criteria: str = "MetropolisUniform", trans_fields=None,
               interrupt_function=None, **kwargs):
        t0 = perf_counter_ns()
        problem = _as_problem(bqm)
        n = len(problem.variables)
        if trans_fields is None:
            trans_fields = np.ones(n)
        elif isinstance(trans_fields, (list, tuple, np.ndarray)):
            if len(trans_fields) != n:
                raise ValueError("bqm.num_variables and trans_fields lengths incompatible")
            trans_fields = np.array(trans_fields)
        else:
            trans_fields = trans_fields * np.ones(n)
        seed = _check_seed(seed)
        prng = np.random.default_rng(seed)
        if isinstance(initial_states, np.ndarray):
            if num_reads is None:
                num_reads = initial_states.shape[0]
            if (num_reads, n) != initial_states.shape:
                raise ValueError("Shape of initial_states specified as"
                                 "ndarray should match (num_reads, num_vars)")
            states = initial_states
        else:
            states = SimulatedAnnealingSampler._initial_states(
                problem, num_reads, initial_states, initial_states_generator, seed)
            num_reads = states.shape[0]
        if states.dtype == np.uint8:
            if project_states[0]:  # sampler.py:941-951
                states = np.ascontiguousarray(
                    128 * (np.cos(np.pi * (states / 128))
                           < 1 - 2 * prng.random(size=states.shape)), dtype=np.uint8)
            else:
                states = np.ascontiguousarray(states)
        else:
            if not set(np.unique(states)).issubset({-1, 1}):
                raise ValueError("initial_states dtype is neither np.uint8 nor consistent with "
                                 "spins {-1, 1}")
            states = np.ascontiguousarray(64 - 64 * states, dtype=np.uint8)
        if interrupt_function and not callable(interrupt_function):
            raise TypeError("'interrupt_function' should be a callable")
        _check_sweeps_per_beta(num_sweeps_per_beta)
        beta_range, Hp_field, Hd_field = build_fields(
            problem, beta_range, num_sweeps, num_sweeps_per_beta, beta_schedule_type,
            Hp_field, Hd_field, zero_sweeps_empty=True)
        interval = _check_interval(schedule_sample_interval, Hp_field)
        t1 = perf_counter_ns()
        samples, energies, statistics = rotor_annealing(
            num_reads, problem.h, problem.u, problem.v, problem.J, trans_fields,
            num_sweeps_per_beta, Hp_field, Hd_field, seed, states, randomize_order,
            proposal_acceptance_criteria, interval, interrupt_function, device=self.device)
        t2 = perf_counter_ns()
        info = {"beta_range": beta_range, "beta_schedule_type": beta_schedule_type}
        if interval > 0:
            info["statistics"] = statistics
        if not project_states[1]:
            info["rotor_states"] = samples.copy()
        spins = np.array(1 - 2 * (np.cos(np.pi * samples / 128)
                                  < 1 - 2 * prng.random(size=samples.shape)), dtype=np.int8)
        return _response(problem, spins, energies, info, (t0, t1, t2),
                         ("statistics", "rotor_states"), make_info_json_serializable)
