"""One batch of problems split across several GPUs.

Reads are independent (each read has its own seed and initial state, the
per-read contract of ``dwave/samplers/sa/src/cpu_sa.cpp:321-358``), so a batch
shards without any exchange during sampling: the reads of every problem are
cut into chunks, the chunks are spread over the devices longest-first by their
cost (reads x sweeps x n) onto the least loaded device, every device anneals
its shard as one batch, and the results are gathered back into the callers'
arrays in problem and read order.  The result is byte for byte the result of
annealing the whole batch on one device.

* :func:`partition` / :func:`shard` / :func:`gather` -- the plan of the split
  and its two halves, pure host code.
* :func:`sample_batch_devices` -- one process driving several devices (one
  host thread per device; the C ABI is reentrant).
* :func:`sample_batch_distributed` -- one process per device under
  ``torch.distributed``: every rank computes the same partition, anneals its
  own shard and the shards are exchanged with one all-gather (or gathered on
  one rank).
"""
from __future__ import annotations

import copy
from typing import Callable, Sequence

import numpy as np

from .workloads import Instance

Chunk = tuple  # (problem index, first read, end read)


def _cost(p: Instance, reads: int) -> int:
    return reads * p.sweeps_per_beta * len(p.betas) * p.n


def partition(problems: Sequence[Instance], parts: int) -> list[list[Chunk]]:
    """Chunks of reads per part, balanced by cost.

    A problem whose cost exceeds a quarter of one part's share is cut into
    ``parts`` near-equal read ranges; smaller problems stay whole.  Chunks are
    taken longest first and each goes to the part with the least cost so far
    (ties to the lower part).  Deterministic in its inputs, so every rank of a
    distributed run computes the same partition."""
    if parts < 1:
        raise ValueError("parts must be at least 1")
    total = sum(_cost(p, p.num_reads) for p in problems)
    share = total / parts
    chunks = []
    for k, p in enumerate(problems):
        R = p.num_reads
        if R == 0:
            continue
        pieces = parts if (parts > 1 and _cost(p, R) > share / 4) else 1
        pieces = min(pieces, R)
        bounds = [R * i // pieces for i in range(pieces + 1)]
        for i in range(pieces):
            if bounds[i + 1] > bounds[i]:
                chunks.append((k, bounds[i], bounds[i + 1]))
    chunks.sort(key=lambda c: (-_cost(problems[c[0]], c[2] - c[1]), c[0], c[1]))
    load = [0] * parts
    out: list[list[Chunk]] = [[] for _ in range(parts)]
    for c in chunks:
        i = min(range(parts), key=lambda j: (load[j], j))
        out[i].append(c)
        load[i] += _cost(problems[c[0]], c[2] - c[1])
    for lst in out:
        lst.sort()
    return out


def shard(problems: Sequence[Instance], chunks: Sequence[Chunk]) -> list[Instance]:
    """The sub-problems of one part: each chunk as a problem holding its read
    range (a copy of those initial states and seeds)."""
    out = []
    for k, r0, r1 in chunks:
        q = copy.copy(problems[k])
        q.states = np.ascontiguousarray(problems[k].states[r0:r1])
        q.seeds = np.ascontiguousarray(np.asarray(problems[k].seeds)[r0:r1])
        out.append(q)
    return out


def gather(problems: Sequence[Instance], parts: Sequence[Sequence[Chunk]],
           results: Sequence[tuple]) -> list[np.ndarray]:
    """Writes every part's annealed states into ``problems[k].states`` (in
    place) and returns the energies per problem.  ``results[i]`` is part i's
    ``(states, energies)``: lists aligned with its chunks."""
    energies = [np.zeros(p.num_reads, dtype=np.float64) for p in problems]
    for chunks, (states, ens) in zip(parts, results):
        for (k, r0, r1), s, e in zip(chunks, states, ens):
            problems[k].states[r0:r1] = s
            energies[k][r0:r1] = e
    return energies


def _device_worker(device: int, mode: str):
    from .batch import sample_batch

    def run(sub: list[Instance]):
        ens = sample_batch(sub, mode=mode, device=device) if sub else []
        return [q.states for q in sub], list(ens)
    return run


def sample_batch_devices(problems: Sequence[Instance], devices: Sequence[int],
                         mode: str = "persistent") -> list[np.ndarray]:
    """Anneal the batch on several devices of this process (one host thread
    per device) and gather the results in place; returns energies per
    problem."""
    from concurrent.futures import ThreadPoolExecutor
    devices = list(devices)
    parts = partition(problems, len(devices))
    subs = [shard(problems, c) for c in parts]
    with ThreadPoolExecutor(len(devices)) as ex:
        futs = [ex.submit(_device_worker(d, mode), s) for d, s in zip(devices, subs)]
        results = [f.result() for f in futs]
    return gather(problems, parts, results)


def sample_batch_distributed(problems: Sequence[Instance], mode: str = "persistent",
                             group=None, dst: int | None = None, device: int | None = None,
                             worker: Callable | None = None) -> list[np.ndarray] | None:
    """One rank per device under ``torch.distributed`` (initialized by the
    caller; NCCL or gloo).  Every rank passes the same problems; each anneals
    its own shard (``worker(sub_problems) -> (states, energies)``, by default
    the batched sampler on ``device``, else the rank's current CUDA device),
    then the shards are exchanged: with ``dst=None`` every rank receives the
    whole result, else rank ``dst`` only (the others return None).  Results are
    written into ``problems[k].states`` on the receiving ranks."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = partition(problems, world)
    sub = shard(problems, parts[rank])
    if worker is None:
        if device is None:
            import torch
            device = torch.cuda.current_device()
        worker = _device_worker(device, mode)
    mine = worker(sub)
    if dst is None:
        results = [None] * world
        dist.all_gather_object(results, mine, group=group)
    else:
        results = [None] * world if rank == dst else None
        dist.gather_object(mine, results, dst=dst, group=group)
        if rank != dst:
            return None
    return gather(problems, parts, results)
