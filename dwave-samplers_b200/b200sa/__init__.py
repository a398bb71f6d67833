"""b200sa: the simulated-annealing path of dwave-samplers, on B200 (sm_100a).

Public surface:

* :func:`simulated_annealing` -- the Cython-level drop-in
  (``dwave/samplers/sa/simulated_annealing.pyx``).
* :func:`sample_batch`, :class:`Plan` -- many problems in one persistent
  launch (graph replay, in-place weights, autotuning).
* :mod:`b200sa.shards` -- one batch split across several GPUs (threads of
  one process, or one rank per GPU under torch.distributed).
* :mod:`b200sa.sampler` -- ``SimulatedAnnealingSampler`` front end (dimod-free).
* :mod:`b200sa.greedy` -- steepest descent (``dwave.samplers.greedy``).
* :mod:`b200sa.sqa` -- ``dwave.samplers.sqa``'s two bindings: rotor-model
  annealing and path-integral Monte Carlo annealing; :mod:`b200sa.sqa_sampler`
  -- its two sampler classes (dimod-free).
* :mod:`b200sa.autograd`, :mod:`b200sa.bm` -- differentiable fixed-beta
  sampling and batched Boltzmann-machine learning.
"""
from .simulated_annealing import per_read_seeds, simulated_annealing
from .batch import Plan, sample_batch

__all__ = ["simulated_annealing", "per_read_seeds", "sample_batch", "Plan"]
__version__ = "0.6.0"
