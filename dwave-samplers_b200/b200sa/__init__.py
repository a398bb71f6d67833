"""b200sa: the simulated-annealing sweep of dwave-samplers, on B200 (sm_100a).

Public surface (mirrors ``dwave.samplers.sa``):

* :func:`simulated_annealing` -- the Cython-level drop-in
  (``dwave/samplers/sa/simulated_annealing.pyx``).
* :func:`sample_batch`, :class:`Plan` -- many problems in one persistent launch.
"""
from .simulated_annealing import per_read_seeds, simulated_annealing
from .batch import Plan, sample_batch

__all__ = ["simulated_annealing", "per_read_seeds", "sample_batch", "Plan"]
__version__ = "0.1.0"
