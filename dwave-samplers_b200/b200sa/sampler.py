"""SimulatedAnnealingSampler front end on the B200 sweep.

Mirrors ``dwave/samplers/sa/sampler.py`` (dwave-samplers 1.8.0): the same
``sample`` keyword arguments, validation and error messages
(``sampler.py:321-461``), the same beta-schedule construction
(``sampler.py:373-426``) and default beta range (``sampler.py:467-600``),
``parameters`` / ``properties`` (``sampler.py:138-154``) and the ``Neal``
alias (``sampler.py:464``).

dimod is optional.  Problems are given as a ``dimod.BinaryQuadraticModel``
when dimod is installed, or as any object with ``linear`` (variable -> bias),
``quadratic`` ((u, v) -> bias), ``offset`` and ``vartype`` ("SPIN" or
"BINARY"), or through :meth:`sample_ising` / :meth:`sample_qubo`.  The result is
a ``dimod.SampleSet`` when dimod is importable, else a :class:`SampleSet` with
the same ``record`` fields (sample, energy, num_occurrences), ``variables``,
``info`` and ``first``.

Variable and coupler order come from the problem's own iteration order (dimod
orders them through ``to_numpy_vectors``, which is not reproduced here), and
random initial states are drawn with ``numpy.random.RandomState(seed)``; read
r is annealed with seed ``seed + r`` (see ``b200sa.simulated_annealing``).
"""
from __future__ import annotations

import math
import warnings
from collections import defaultdict, namedtuple
from numbers import Integral
from time import perf_counter_ns
from typing import Optional, Sequence

import numpy as np

from .simulated_annealing import simulated_annealing

__all__ = ["SimulatedAnnealingSampler", "Neal", "SampleSet", "default_beta_range",
           "ising_beta_range"]

try:  # optional
    import dimod  # type: ignore
except ImportError:  # pragma: no cover - dimod is absent in this environment
    dimod = None


class _Record(namedtuple("_Record", ["sample", "energy", "num_occurrences"])):
    pass


class SampleSet:
    """Minimal stand-in for ``dimod.SampleSet`` (used when dimod is absent)."""

    def __init__(self, samples, variables, energies, info, vartype):
        self.record = _Record(np.asarray(samples), np.asarray(energies, dtype=np.float64),
                              np.ones(len(energies), dtype=np.int64))
        self.variables = list(variables)
        self.info = dict(info)
        self.vartype = vartype

    def __len__(self):
        return len(self.record.energy)

    @property
    def first(self):
        i = int(np.argmin(self.record.energy))
        Sample = namedtuple("Sample", ["sample", "energy", "num_occurrences"])
        return Sample(dict(zip(self.variables, self.record.sample[i].tolist())),
                      float(self.record.energy[i]), 1)

    def samples(self):
        return [dict(zip(self.variables, row.tolist())) for row in self.record.sample]

    def data_vectors(self):
        return {"energy": self.record.energy, "num_occurrences": self.record.num_occurrences}


class _IsingProblem:
    """Problem in SPIN form: variable order, h, COO couplers, offset."""

    def __init__(self, linear, quadratic, offset, vartype):
        vartype = str(getattr(vartype, "name", vartype)).upper()
        if vartype not in ("SPIN", "BINARY"):
            raise ValueError(f"unknown vartype {vartype}")
        variables = list(linear)
        for (a, b) in quadratic:
            for x in (a, b):
                if x not in linear and x not in variables:
                    variables.append(x)
        index = {x: i for i, x in enumerate(variables)}
        n = len(variables)
        h = np.zeros(n)
        for x, bias in linear.items():
            h[index[x]] += float(bias)
        pairs = [(index[a], index[b], float(w)) for (a, b), w in quadratic.items()]
        offset = float(offset)
        if vartype == "BINARY":
            # x = (s + 1) / 2:  a x -> a/2 s + a/2;  b x y -> b/4 (s t + s + t + 1)
            hs = h / 2.0
            offset += float(np.sum(h)) / 2.0
            for i, j, w in pairs:
                hs[i] += w / 4.0
                hs[j] += w / 4.0
                offset += w / 4.0
            h = hs
            pairs = [(i, j, w / 4.0) for i, j, w in pairs]
        self.variables = variables
        self.h = h
        self.u = np.array([p[0] for p in pairs], dtype=np.int32)
        self.v = np.array([p[1] for p in pairs], dtype=np.int32)
        self.J = np.array([p[2] for p in pairs], dtype=np.float64)
        self.offset = offset
        self.vartype = vartype
        self.linear = {x: self.h[index[x]] for x in variables}
        self.quadratic = {(variables[i], variables[j]): w for i, j, w in zip(self.u, self.v, self.J)}


def ising_beta_range(h: dict, J: dict, max_single_qubit_excitation_rate: float = 0.01,
                     scale_T_with_N: bool = True):
    """Default [hot, cold] beta of an Ising model (``sampler.py:467-600``).

    Hot: every spin flips with probability >= 1/2 under the worst-case
    effective field (sum of |biases| of the variable).  Cold: the probability
    of exciting any spin on the last sweep is about the target rate, with the
    smallest non-zero bias of each variable as its minimal gap.  A model whose
    biases are all zero gives [0.1, 1] with a warning.
    """
    if not 0 < max_single_qubit_excitation_rate < 1:
        raise ValueError('Targeted single qubit excitations rates must be in range (0,1)')
    total = defaultdict(float, {k: abs(b) for k, b in h.items()})
    smallest = {k: abs(b) for k, b in h.items() if abs(b) != 0}
    for (a, b), w in J.items():
        for k in (a, b):
            total[k] += abs(w)
            if w != 0:
                smallest[k] = min(abs(w), smallest[k]) if k in smallest else abs(w)
    if not smallest:
        warnings.warn('All bqm biases are zero (all energies are zero), this is likely a '
                      'value error. Temperature range is set arbitrarily to [0.1,1]. '
                      'Metropolis-Hastings update is non-ergodic.')
        return [0.1, 1]
    max_field = max(total.values(), default=0)
    hot = 1 if max_field == 0 else np.log(2) / (2 * max_field)
    values = np.array(list(smallest.values()), dtype=float)
    min_field = np.min(values)
    gaps = np.sum(min_field == values) if scale_T_with_N else 1
    cold = np.log(gaps / max_single_qubit_excitation_rate) / (2 * min_field)
    return [hot, cold]


def default_beta_range(bqm):
    """Default beta range of a problem in any vartype (``sampler.py:602-604``)."""
    p = _as_problem(bqm)
    return ising_beta_range(p.linear, p.quadratic)


def _as_problem(bqm) -> _IsingProblem:
    return _IsingProblem(dict(bqm.linear), dict(bqm.quadratic), getattr(bqm, "offset", 0.0),
                         getattr(bqm, "vartype", "SPIN"))


class SimulatedAnnealingSampler:
    """Simulated annealing on the B200 with the reference sampler's interface."""

    def __init__(self, device: int = 0):
        self.device = device
        self.parameters = {'beta_range': [], 'num_reads': [], 'num_sweeps': [],
                           'num_sweeps_per_beta': [],
                           'beta_schedule_type': ['beta_schedule_options'],
                           'beta_schedule': [], 'seed': [], 'interrupt_function': [],
                           'initial_states': [], 'initial_states_generator': [],
                           'randomize_order': [], 'proposal_acceptance_criteria': []}
        self.properties = {'beta_schedule_options': ('linear', 'geometric', 'custom')}

    # -- dimod-style mixins -------------------------------------------------
    def sample_ising(self, h, J, **kwargs):
        if not isinstance(h, dict):
            h = dict(enumerate(h))
        Q = type("Ising", (), {})()
        Q.linear, Q.quadratic, Q.offset, Q.vartype = h, J, 0.0, "SPIN"
        return self.sample(Q, **kwargs)

    def sample_qubo(self, Q, **kwargs):
        linear, quadratic = {}, {}
        for (a, b), w in Q.items():
            if a == b:
                linear[a] = linear.get(a, 0.0) + w
            else:
                linear.setdefault(a, 0.0)
                linear.setdefault(b, 0.0)
                quadratic[(a, b)] = quadratic.get((a, b), 0.0) + w
        B = type("Qubo", (), {})()
        B.linear, B.quadratic, B.offset, B.vartype = linear, quadratic, 0.0, "BINARY"
        return self.sample(B, **kwargs)

    # -- the sampler --------------------------------------------------------
    def sample(self, bqm, beta_range: Optional[Sequence[float]] = None,
               num_reads: Optional[int] = None, num_sweeps: Optional[int] = None,
               num_sweeps_per_beta: int = 1, beta_schedule_type: str = "geometric",
               seed: Optional[int] = None, interrupt_function=None,
               beta_schedule=None, initial_states=None,
               initial_states_generator: str = "random", randomize_order: bool = False,
               proposal_acceptance_criteria: str = 'Metropolis', **kwargs):
        timestamp_preprocess = perf_counter_ns()
        for k in kwargs:
            warnings.warn(f"Ignoring unknown kwarg: {k!r}", UserWarning)
        problem = _as_problem(bqm)
        n = len(problem.variables)

        # seed policy, sampler.py:331-340
        if seed is None:
            seed = np.random.randint(2**31)
        elif not isinstance(seed, Integral):
            raise TypeError("'seed' should be None or an integer between 0 and 2^32 "
                            "- 1: value = {}".format(seed))
        elif not (0 <= seed < 2**31):
            raise ValueError("'seed' should be an integer between 0 and 2^32 - 1: "
                             "value = {}".format(seed))

        init = self._initial_states(problem, num_reads, initial_states,
                                    initial_states_generator, seed)
        num_reads = init.shape[0]

        if interrupt_function and not callable(interrupt_function):
            raise TypeError("'interrupt_function' should be a callable")
        if not isinstance(num_sweeps_per_beta, Integral):
            raise TypeError("'num_sweeps_per_beta' should be a positive integer: value = {}"
                            .format(num_sweeps_per_beta))
        if num_sweeps_per_beta < 1:
            raise ValueError("'num_sweeps_per_beta' should be a positive integer: value = {}"
                             .format(num_sweeps_per_beta))
        beta_range, beta_schedule = build_schedule(
            problem, beta_range, num_sweeps, num_sweeps_per_beta, beta_schedule_type,
            beta_schedule)

        timestamp_sample = perf_counter_ns()
        run = {}
        samples, energies = simulated_annealing(
            num_reads, problem.h, problem.u, problem.v, problem.J, num_sweeps_per_beta,
            beta_schedule, seed, init, randomize_order, proposal_acceptance_criteria,
            interrupt_function, device=self.device, stats=run)
        timestamp_postprocess = perf_counter_ns()

        info = {"beta_range": beta_range, "beta_schedule_type": beta_schedule_type}
        # Reads whose exp() decisions all fell outside the 2^-48 band around
        # their thresholds are bit-exact with the reference; the others are
        # listed (expected: none).
        ties = run.get("near_ties_per_read", np.zeros(0, np.uint32))
        info["near_ties"] = int(ties.sum())
        info["near_tie_reads"] = np.flatnonzero(ties).tolist()
        if problem.vartype == "BINARY":
            out = ((np.asarray(samples) + 1) // 2).astype(np.int8)
        else:
            out = np.asarray(samples)
        energies = energies + problem.offset
        if dimod is not None:
            response = dimod.SampleSet.from_samples(
                (out, problem.variables), energy=energies, info=info,
                vartype=dimod.BINARY if problem.vartype == "BINARY" else dimod.SPIN)
        else:
            response = SampleSet(out, problem.variables, energies, info, problem.vartype)
        response.info.update(dict(timing=dict(
            preprocessing_ns=timestamp_sample - timestamp_preprocess,
            sampling_ns=timestamp_postprocess - timestamp_sample,
            postprocessing_ns=perf_counter_ns() - timestamp_postprocess)))
        return response

    @staticmethod
    def _initial_states(problem, num_reads, initial_states, generator, seed):
        """Initial states (num_reads x n int8 SPIN), following the semantics of
        the reference's ``initial_states`` / ``initial_states_generator``."""
        n = len(problem.variables)
        if generator not in ("none", "tile", "random"):
            raise ValueError("unknown initial_states_generator: {!r}".format(generator))
        if initial_states is None:
            given = np.empty((0, n), dtype=np.int8)
        else:
            if isinstance(initial_states, dict) or (
                    isinstance(initial_states, (list, tuple)) and initial_states
                    and isinstance(initial_states[0], dict)):
                rows = [initial_states] if isinstance(initial_states, dict) else initial_states
                given = np.array([[r[x] for x in problem.variables] for r in rows])
            else:
                given = np.atleast_2d(np.asarray(initial_states))
            if given.size and given.shape[1] != n:
                raise ValueError("initial_states have the wrong number of variables")
            if problem.vartype == "BINARY":
                given = 2 * given - 1
            given = given.astype(np.int8)
        if num_reads is None:
            num_reads = len(given) if len(given) else 1
        if num_reads < 1:
            raise ValueError("num_reads should be a positive integer")
        if len(given) >= num_reads:
            return np.ascontiguousarray(given[:num_reads])
        if generator == "none":
            raise ValueError("insufficient number of initial states given")
        if generator == "tile" and len(given):
            reps = -(-num_reads // len(given))
            return np.ascontiguousarray(np.tile(given, (reps, 1))[:num_reads])
        rng = np.random.RandomState(seed)
        extra = 2 * rng.randint(2, size=(num_reads - len(given), n)).astype(np.int8) - 1
        return np.ascontiguousarray(np.vstack([given, extra]).astype(np.int8))


def build_schedule(problem, beta_range, num_sweeps, num_sweeps_per_beta, beta_schedule_type,
                   beta_schedule):
    """The beta schedule of ``sampler.py:373-426``; returns (beta_range, schedule)."""
    if beta_schedule_type == "custom":
        if beta_schedule is None:
            raise ValueError("'beta_schedule' must be provided for beta_schedule_type = "
                             "'custom': value is None")
        try:
            beta_schedule = np.array(beta_schedule, dtype=float)
        except Exception:
            raise ValueError('beta_schedule cannot be case as a numpy array of dtype=float')
        if num_sweeps is not None and num_sweeps != len(beta_schedule) * num_sweeps_per_beta:
            raise ValueError("'num_sweeps' should be set to None, or a value consistent with "
                             "'beta_schedule' and 'num_sweeps_per_beta' for "
                             "'beta_schedule_type' = 'custom': value = ")
        if beta_range is not None and (beta_range[0] != beta_schedule[0]
                                       or beta_range[-1] != beta_schedule[-1]):
            raise ValueError("'beta_range' should be set to None, or a value consistent with "
                             "'beta_schedule', for 'beta_schedule_type'='custom'.")
        if np.min(beta_schedule) < 0:
            raise ValueError("'beta_schedule' cannot include negative values.")
        return beta_range, beta_schedule
    if beta_schedule is not None:
        raise ValueError("'beta_schedule' must be set to None for 'beta_schedule_type' not "
                         "equal to 'custom'")
    if num_sweeps is None:
        num_sweeps = 1000
    num_betas, rem = divmod(num_sweeps, num_sweeps_per_beta)
    if rem > 0 or num_betas < 0:
        raise ValueError("'num_sweeps' must be a non-negative value divisible by "
                         "'num_sweeps_per_beta'.")
    if beta_range is None:
        beta_range = ising_beta_range(problem.linear, problem.quadratic)
    elif len(beta_range) != 2 or min(beta_range) < 0:
        raise ValueError("'beta_range' should be a 2-tuple, or 2 element list of positive "
                         "numbers. The latter value is the target value.")
    if num_betas == 1:
        schedule = np.array([beta_range[-1]], dtype=float)
    elif beta_schedule_type == "linear":
        schedule = np.linspace(*beta_range, num=num_betas)
    elif beta_schedule_type == "geometric":
        if min(beta_range) <= 0:
            raise ValueError("'beta_range' must contain non-zero values for "
                             "'beta_schedule_type' = 'geometric'")
        schedule = np.geomspace(*beta_range, num=num_betas)
    else:
        raise ValueError("Beta schedule type {} not implemented".format(beta_schedule_type))
    return beta_range, schedule


Neal = SimulatedAnnealingSampler
