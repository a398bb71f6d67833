"""Differentiable fixed-beta sampling (no reference counterpart).

For Ising models in the reference's convention (energy
``E(s) = sum_i h_i s_i + sum_c J_c s_u s_v``, ``cpu_sa.cpp:210-227``, and
acceptance ``exp(-beta dE)``, ``cpu_sa.cpp:154``) the log partition function
``log Z = log sum_s exp(-beta E(s))`` has

    d log Z / d h_i = -beta <s_i>,     d log Z / d J_c = -beta <s_u(c) s_v(c)>.

:class:`LogPartition` wraps fixed-beta sampling on the B200 (every read bit
identical to the reference run with that read's seed) as an autograd
``Function``: its forward draws the samples, its backward reduces them over
the couplers with the ``b200sa_edge_moments`` CUDA kernel and returns the two
expectations above scaled by ``-beta``.  The forward *value* is a placeholder
(zero): only the gradient of log Z is estimated.

When ``reads * num_vars`` exceeds ``memory_budget`` bytes the samples are not
kept: the backward re-runs the sampler from the stored seeds in chunks of
reads.  Initial states are then a deterministic function of ``init_seed`` (not
stored either), so the recomputed samples are bit-identical.

``models`` may hold many problems; sampling runs as one persistent batch and
the backward reduction as one launch over all of them.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import numpy as np
import torch

from . import _lib
from .batch import Plan
from .workloads import Instance


@dataclass
class IsingModel:
    """Structure of one model: size and couplers (COO, input order)."""
    num_vars: int
    u: np.ndarray  # int32 [m]
    v: np.ndarray  # int32 [m]

    @property
    def num_couplers(self) -> int:
        return int(self.u.shape[0])


def _mix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finalizer (a bijective 64-bit mixing function), vectorized."""
    with np.errstate(over="ignore"):
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return x ^ (x >> np.uint64(31))


def initial_states(init_seed: int, model_index: int, reads: int, n: int,
                   read0: int = 0) -> np.ndarray:
    """Uniform +-1 initial states as a counter-based hash of (seed, model,
    read, variable): any range of reads can be regenerated identically."""
    r = np.arange(read0, read0 + reads, dtype=np.uint64)[:, None]
    i = np.arange(n, dtype=np.uint64)[None, :]
    with np.errstate(over="ignore"):
        key = _mix64(np.uint64(init_seed) * np.uint64(0x9E3779B97F4A7C15)
                     + np.uint64(model_index) * np.uint64(0xD1B54A32D192ED03))
        x = _mix64(key ^ (r * np.uint64(0x100000001B3) + i))
    return np.where((x >> np.uint64(63)) != 0, 1, -1).astype(np.int8)


def device_initial_states(out: torch.Tensor, init_seed: int, model_index: int, read0: int,
                          reads: int, n: int, device: int = 0) -> torch.Tensor:
    """:func:`initial_states` generated on the GPU into ``out`` (int8 CUDA
    tensor of reads * n elements) by ``b200sa_random_states``."""
    if out.dtype != torch.int8 or not out.is_cuda or out.numel() != reads * n:
        raise ValueError("out must be an int8 CUDA tensor of reads * n elements")
    err = _lib.errbuf()
    rc = _lib.load().b200sa_random_states(
        int(init_seed), int(model_index), int(read0), int(reads), int(n), out.data_ptr(),
        int(device), torch.cuda.current_stream(out.device).cuda_stream, err, len(err))
    _lib.check(rc, err)
    return out


def read_seeds(seed: int, model_index: int, reads: int, read0: int = 0) -> np.ndarray:
    base = (np.uint64(seed) * np.uint64(1000003) + np.uint64(model_index) * np.uint64(1 << 40))
    with np.errstate(over="ignore"):
        return base + np.arange(read0, read0 + reads, dtype=np.uint64)


class ModelSampler:
    """Fixed-beta sampling of a fixed set of model structures.

    The models are packed into one plan once; every call writes the new
    fields and couplings into it (``b200sa_plan_set_weights``), generates the
    initial states on the GPU, uploads the per-read seeds and replays the
    plan's captured CUDA graph over the same device buffers.  Reads
    [read0, read0 + reads) of model k start from ``initial_states(init_seed,
    k, reads, n, read0)`` with seeds ``read_seeds(seed, k, reads, read0)``.
    """

    def __init__(self, models: Sequence[IsingModel], beta: float, sweeps: int, reads: int,
                 proposal: str = "Gibbs", device: int = 0, autotune: bool = False):
        self.models = list(models)
        self.reads = int(reads)
        self.device = int(device)
        dev = torch.device("cuda", self.device)
        insts = [Instance(
            np.zeros(m.num_vars), m.u, m.v, np.zeros(m.num_couplers),
            # shape only: the plan packs structure, the states are made on the GPU
            np.broadcast_to(np.zeros(1, np.int8), (self.reads, m.num_vars)),
            np.array([float(beta)]), int(sweeps), np.zeros(self.reads, np.uint64),
            proposal=proposal) for m in self.models]
        self.plan = Plan(insts, device=self.device)
        if autotune:
            # Launch shapes measured per size bucket (results do not depend on them).
            self.plan.autotune(None)
        self.sin = torch.empty(max(self.plan.total_state, 1), dtype=torch.int8, device=dev)
        self.sout = torch.empty_like(self.sin)
        self.en = torch.empty(max(self.plan.total_reads, 1), dtype=torch.float64, device=dev)
        self.seeds = torch.empty(max(self.plan.total_reads, 1), dtype=torch.int64, device=dev)

    def sample(self, hs, Js, seed: int, init_seed: int, read0: int = 0) -> list[torch.Tensor]:
        """One int8 CUDA tensor (reads x n) per model; the tensors are views of
        the sampler's output buffer, overwritten by the next call.  ``hs`` /
        ``Js`` are per-model arrays (host or device)."""
        dev = self.sin.device
        cat = lambda xs: torch.cat([torch.as_tensor(x, dtype=torch.float64).reshape(-1).to(dev)
                                    for x in xs]) if len(xs) else torch.zeros(0, dtype=torch.float64,
                                                                              device=dev)
        return self.sample_cat(cat(hs), cat(Js), seed, init_seed, read0)

    def sample_cat(self, h_cat: torch.Tensor, J_cat: torch.Tensor, seed: int, init_seed: int,
                   read0: int = 0) -> list[torch.Tensor]:
        """As :meth:`sample`, with every model's fields and couplings given
        concatenated in two float64 CUDA tensors: they are written into the
        plan on the device (``b200sa_plan_set_weights_device``), with no host
        round trip."""
        dev = self.sin.device
        offs = self.plan.state_offsets
        stream = torch.cuda.current_stream(dev)
        h_cat = h_cat.detach().to(device=dev, dtype=torch.float64).contiguous()
        J_cat = J_cat.detach().to(device=dev, dtype=torch.float64).contiguous()
        if h_cat.numel() == 0:
            h_cat = torch.zeros(1, dtype=torch.float64, device=dev)
        if J_cat.numel() == 0:
            J_cat = torch.zeros(1, dtype=torch.float64, device=dev)
        self.plan.set_weights_device(h_cat, J_cat, stream=stream)
        seeds = np.concatenate([read_seeds(seed, k, self.reads, read0)
                                for k in range(len(self.models))])
        self.seeds[:seeds.shape[0]].copy_(torch.from_numpy(seeds.view(np.int64)))
        for k, mod in enumerate(self.models):
            device_initial_states(self.sin[int(offs[k]):int(offs[k + 1])], init_seed, k, read0,
                                  self.reads, mod.num_vars, self.device)
        self.plan.run(self.sin, self.sout, self.en, seeds=self.seeds, mode="graph",
                      stream=torch.cuda.current_stream(dev), sync=True)
        return [self.sout[int(offs[k]):int(offs[k + 1])].view(self.reads, m.num_vars)
                for k, m in enumerate(self.models)]

    def close(self):
        self.plan.close()


def sample_models(models: Sequence[IsingModel], hs: Sequence[np.ndarray],
                  Js: Sequence[np.ndarray], beta: float, sweeps: int, reads: int,
                  seed: int, init_seed: int, read0: int = 0, proposal: str = "Gibbs",
                  device: int = 0, sampler: ModelSampler | None = None) -> list[torch.Tensor]:
    """Fixed-beta sampling of every model (one persistent batch): reads
    [read0, read0 + reads) of each model, `sweeps` sweeps at `beta`.
    Returns one int8 CUDA tensor (reads x n) per model.  With `sampler` (a
    :class:`ModelSampler` built for these models, reads and settings) its
    plan and graph are reused; the results are the same."""
    own = sampler is None
    if own:
        sampler = ModelSampler(models, beta, sweeps, reads, proposal, device)
    try:
        out = sampler.sample(hs, Js, seed, init_seed, read0)
        return [x.clone() for x in out] if not own else out
    finally:
        if own:
            sampler.close()


def edge_moments(models: Sequence[IsingModel], samples: Sequence[torch.Tensor],
                 device: int = 0):
    """Integer sums over reads of s_i and of s_u s_v per coupler, for every
    model, in one launch of the moments kernel.  Returns lists of int64 CUDA
    tensors (n,) and (m,)."""
    dev = torch.device("cuda", device)
    keep = []
    arr = (_lib.MomentsProblem * max(len(models), 1))()
    sums_s, sums_ss = [], []
    for k, (mod, st) in enumerate(zip(models, samples)):
        st = st.contiguous()
        cu = torch.from_numpy(np.ascontiguousarray(mod.u, dtype=np.int32)).to(dev)
        cv = torch.from_numpy(np.ascontiguousarray(mod.v, dtype=np.int32)).to(dev)
        ss = torch.zeros(mod.num_vars, dtype=torch.int64, device=dev)
        sss = torch.zeros(max(mod.num_couplers, 1), dtype=torch.int64, device=dev)
        keep += [st, cu, cv]
        q = arr[k]
        q.num_vars = mod.num_vars
        q.num_couplers = mod.num_couplers
        q.num_reads = int(st.shape[0])
        q.states = st.data_ptr()
        q.coupler_starts = cu.data_ptr()
        q.coupler_ends = cv.data_ptr()
        q.sum_s = ss.data_ptr()
        q.sum_ss = sss.data_ptr()
        sums_s.append(ss)
        sums_ss.append(sss[:mod.num_couplers])
    err = _lib.errbuf()
    rc = _lib.load().b200sa_edge_moments(arr, len(models), device,
                                         torch.cuda.current_stream(dev).cuda_stream, err, len(err))
    _lib.check(rc, err)
    del keep
    return sums_s, sums_ss


def pool_sums(sum_s: Sequence[torch.Tensor], sum_ss: Sequence[torch.Tensor], group):
    """Moment sums added over the ranks of `group`: one all-reduce (NCCL
    between GPUs) of the concatenated int64 sums, so the pooled sums are
    exact and identical on every rank.  Returns new lists of the same shapes."""
    import torch.distributed as dist
    parts = list(sum_s) + list(sum_ss)
    flat = torch.cat([x.reshape(-1) for x in parts])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    out, i = [], 0
    for x in parts:
        out.append(flat[i:i + x.numel()].view(x.shape))
        i += x.numel()
    return out[:len(sum_s)], out[len(sum_s):]


class LogPartition(torch.autograd.Function):
    """``LogPartition.apply(h_cat, J_cat, spec)`` for a batch of models.

    ``h_cat`` / ``J_cat`` are the models' fields and couplings concatenated
    (float64, any device, may require grad); ``spec`` is a
    :class:`SamplingSpec`.  Returns a zero placeholder (log Z itself is not
    estimated); the forward's samples are left in ``spec.last_samples``
    (empty when they are recomputed in backward).  Backward returns
    ``-beta <s_i>`` and ``-beta <s_u s_v>`` per coupler; with ``spec.group``
    the moments are pooled over the group's ranks (:func:`pool_sums`) before
    the averages are taken.
    """

    @staticmethod
    def forward(ctx, h_cat, J_cat, spec):
        # The weights stay on the device: they are scattered into the plan by
        # a kernel (no copy to the host).
        dev = torch.device("cuda", spec.device)
        hd = h_cat.detach().to(device=dev, dtype=torch.float64).contiguous()
        Jd = J_cat.detach().to(device=dev, dtype=torch.float64).contiguous()
        keep = spec.reads * sum(m.num_vars for m in spec.models) <= spec.memory_budget
        samples = []
        if keep:
            samples = spec.sampler(spec.reads).sample_cat(hd, Jd, spec.seed, spec.init_seed,
                                                          spec.first_read)
        spec.last_samples = samples
        ctx.spec = spec
        ctx.hs, ctx.Js = hd, Jd
        ctx.samples = samples
        ctx.h_device, ctx.J_device = h_cat.device, J_cat.device
        return torch.zeros((), dtype=torch.float64, device=h_cat.device)

    @staticmethod
    def backward(ctx, g):
        spec = ctx.spec
        sum_s, sum_ss = spec.moments(ctx.hs, ctx.Js, ctx.samples)
        if spec.group is not None:
            sum_s, sum_ss = pool_sums(sum_s, sum_ss, spec.group)
        spec.last_moments = (sum_s, sum_ss)
        scale = -spec.beta / spec.total_reads
        gh = (torch.cat([x.to(torch.float64) for x in sum_s]) * scale).to(ctx.h_device)
        gJ = (torch.cat([x.to(torch.float64) for x in sum_ss]) * scale).to(ctx.J_device)
        return gh * g.to(ctx.h_device), gJ * g.to(ctx.J_device), None


@dataclass
class SamplingSpec:
    """Fixed-beta sampling settings for :class:`LogPartition`."""
    models: Sequence[IsingModel]
    beta: float = 1.0
    sweeps: int = 1000
    reads: int = 1024
    seed: int = 1
    init_seed: int = 2
    proposal: str = "Gibbs"
    memory_budget: int = 1 << 30   # bytes of samples kept for backward
    recompute_chunk: int = 256     # reads per chunk when recomputing
    device: int = 0
    autotune: bool = False         # measure launch shapes when a sampler is built
    last_samples: list = None      # set by LogPartition.forward
    last_moments: tuple = None     # set by LogPartition.backward
    samplers: dict = None          # reads per call -> ModelSampler (plan + graph reused)
    group: object = None           # torch.distributed group: each rank samples `reads` reads

    @property
    def first_read(self) -> int:
        """This rank's first read: with a group, rank k samples reads
        [k reads, (k + 1) reads) of the pooled set (their seeds and initial
        states), so the pooled moments equal one run of reads x ranks."""
        return 0 if self.group is None else torch.distributed.get_rank(self.group) * self.reads

    @property
    def total_reads(self) -> int:
        """Reads behind the (pooled) moments."""
        ranks = 1 if self.group is None else torch.distributed.get_world_size(self.group)
        return self.reads * ranks

    def sampler(self, reads: int) -> ModelSampler:
        """The spec's sampler for calls of `reads` reads (built on first use;
        later calls reuse its plan and captured graph)."""
        if self.samplers is None:
            self.samplers = {}
        if reads not in self.samplers:
            self.samplers[reads] = ModelSampler(self.models, self.beta, self.sweeps, reads,
                                                self.proposal, self.device, self.autotune)
        return self.samplers[reads]

    def split(self, h_cat, J_cat):
        hs, Js, i, j = [], [], 0, 0
        for m in self.models:
            hs.append(h_cat[i:i + m.num_vars])
            Js.append(J_cat[j:j + m.num_couplers])
            i += m.num_vars
            j += m.num_couplers
        return hs, Js

    def moments(self, h_cat, J_cat, samples):
        """Moment sums of the forward's samples, or of samples recomputed from
        the stored seeds (h_cat / J_cat: the concatenated weights, device)."""
        if samples:
            return edge_moments(self.models, samples, self.device)
        # Recompute from the stored seeds, chunk by chunk of reads.
        tot_s = tot_ss = None
        for r0 in range(0, self.reads, self.recompute_chunk):
            k = min(self.recompute_chunk, self.reads - r0)
            chunk = self.sampler(k).sample_cat(h_cat, J_cat, self.seed, self.init_seed,
                                               self.first_read + r0)
            s, ss = edge_moments(self.models, chunk, self.device)
            if tot_s is None:
                tot_s, tot_ss = s, ss
            else:
                tot_s = [a + b for a, b in zip(tot_s, s)]
                tot_ss = [a + b for a, b in zip(tot_ss, ss)]
        return tot_s, tot_ss


def log_partition(h_cat: torch.Tensor, J_cat: torch.Tensor, spec: SamplingSpec):
    """Differentiable placeholder for log Z (see :class:`LogPartition`)."""
    return LogPartition.apply(h_cat, J_cat, spec)
